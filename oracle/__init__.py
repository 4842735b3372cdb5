"""CPU oracle for the periodic-orbit path — TEST INFRASTRUCTURE ONLY.

This package restates, in numpy/scipy, the reference algorithms the device
path replaces (operator assembly, the FCT deferred correction, the SuperLU
periodic-orbit GMRES solve and its transposed adjoint, the air-mass-balance
diagnostics).  Each function cites the reference file:line it follows.

Only the test suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or the timed CPU baseline.  The product package ``orbit_b200`` never
imports it and fails loudly when its CUDA library is missing.

Parity pinning: the restatement is checked against golden vectors that
``tests/golden/make_golden.py`` generated by running the reference itself
(ORBIT 1.0.4, SciPy SuperLU backend) on seeded synthetic grids.
"""
