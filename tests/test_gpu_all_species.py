"""solve_orbit_all_species (orbit/core/orbit.py:213-806) options on the device,
against the CPU oracle on the 5x8x9 golden grid (B200).

* end-of-bin couplings (``endbin_keys``): the target reads c_src[tau + 1];
* the LU cache: a second call reuses the first call's factors (its operators
  already released) and solves new emissions;
* seed orbits for a cyclic source pair: both species read the seeds;
* ``skip_solve_species`` with ``cached_orbits``: the cached orbit is returned
  as given and feeds the species downstream of it.
The coupled right-hand sides are formed on the device
(``orbit_source_coupling``); each result must match the oracle to 1e-9.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import golden_io
from oracle import assembly, orbit as oorbit

pytestmark = pytest.mark.gpu

Z = golden_io.load()
MET = golden_io.met_list(Z)
SPC = golden_io.species(Z)
N = MET[0].N


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _L(scale):
    d = SPC.sink_diag(MET)
    return [assembly.species_operator(assembly.transport_block(g), scale * d[t]) for t, g in enumerate(MET)]


def _oracle(L, e):
    lus = [oorbit.factor_one_bin(L[t]) for t in range(8)]
    o, _ = oorbit.solve_orbit_one_species(lus, [np.asarray(x) for x in e], tol=1e-12)
    return o


def _problem():
    L0, L1 = _L(1.0), _L(2.0)
    rate = 3e-5 * (1.0 + np.arange(N) / N)
    emis = np.zeros((8, 2 * N))
    emis[:, :N] = SPC.emis
    emis[:, N:] = 0.3 * SPC.emis
    return L0, L1, rate, emis


def test_endbin_coupling_reads_the_next_bin():
    from orbit_b200 import orbit as oorb
    L0, L1, rate, emis = _problem()
    K = [{(1, 0): sp.diags(-rate).tocsc()} for _ in range(8)]
    res = oorb.solve_orbit_all_species([[L0[t], L1[t]] for t in range(8)], K, emis, N, tol=1e-12,
                                       verbose=False, endbin_keys={(1, 0)})
    o0 = _oracle(L0, SPC.emis)
    e1 = [0.3 * SPC.emis[t] + rate * o0[t + 1] for t in range(8)]
    o1 = _oracle(L1, e1)
    assert _rel(np.stack(res["orbits"][0]), np.stack(o0)) < 1e-9
    assert _rel(np.stack(res["orbits"][1]), np.stack(o1)) < 1e-9


def test_lu_cache_reused_by_a_second_call():
    from orbit_b200 import orbit as oorb
    L0, L1, rate, emis = _problem()
    K = [{(1, 0): sp.diags(-rate).tocsc()} for _ in range(8)]
    Ls = [[L0[t], L1[t]] for t in range(8)]
    from orbit_b200.solve import umfpack_symbolic
    sym = umfpack_symbolic(L0[0], verbose=False)
    res = oorb.solve_orbit_all_species(Ls, K, emis, N, tol=1e-12, verbose=False, return_lu_cache=True,
                                       umfpack_sym=sym)
    assert set(res["lu_cache"]) == {0, 1}
    assert all(Ls[t][s] is None for t in range(8) for s in range(2))  # operators released
    res2 = oorb.solve_orbit_all_species(Ls, K, 2.0 * emis, N, tol=1e-12, verbose=False,
                                        lu_cache=res["lu_cache"], umfpack_sym=sym)
    o0 = _oracle(L0, 2.0 * SPC.emis)
    o1 = _oracle(L1, [0.6 * SPC.emis[t] + rate * o0[t] for t in range(8)])
    assert _rel(np.stack(res2["orbits"][0]), np.stack(o0)) < 1e-9
    assert _rel(np.stack(res2["orbits"][1]), np.stack(o1)) < 1e-9


def test_seed_orbits_break_a_cyclic_pair():
    from orbit_b200 import orbit as oorb
    L0, L1, rate, emis = _problem()
    K = [{(1, 0): sp.diags(-rate).tocsc(), (0, 1): sp.diags(-0.5 * rate).tocsc()} for _ in range(8)]
    rng = np.random.default_rng(12)
    seed = {0: [np.abs(rng.standard_normal(N)) * 1e-6 for _ in range(9)],
            1: [np.abs(rng.standard_normal(N)) * 1e-6 for _ in range(9)]}
    seed_copy = {s: [c.copy() for c in v] for s, v in seed.items()}
    res = oorb.solve_orbit_all_species([[L0[t], L1[t]] for t in range(8)], K, emis, N, tol=1e-12,
                                       verbose=False, seed_orbits=seed)
    o0 = _oracle(L0, [SPC.emis[t] + 0.5 * rate * seed[1][t] for t in range(8)])
    o1 = _oracle(L1, [0.3 * SPC.emis[t] + rate * seed[0][t] for t in range(8)])
    assert _rel(np.stack(res["orbits"][0]), np.stack(o0)) < 1e-9
    assert _rel(np.stack(res["orbits"][1]), np.stack(o1)) < 1e-9
    for s in (0, 1):  # the caller's seeds are not modified
        assert all(np.array_equal(a, b) for a, b in zip(seed[s], seed_copy[s]))


def test_skip_solve_returns_cached_orbit_and_feeds_downstream():
    from orbit_b200 import orbit as oorb
    L0, L1, rate, emis = _problem()
    K = [{(1, 0): sp.diags(-rate).tocsc()} for _ in range(8)]
    rng = np.random.default_rng(13)
    cached = {0: [np.abs(rng.standard_normal(N)) * 1e-6 for _ in range(9)]}
    res = oorb.solve_orbit_all_species([[L0[t], L1[t]] for t in range(8)], K, emis, N, tol=1e-12,
                                       verbose=False, skip_solve_species={0}, cached_orbits=cached)
    assert all(np.array_equal(a, b) for a, b in zip(res["orbits"][0], cached[0]))
    o1 = _oracle(L1, [0.3 * SPC.emis[t] + rate * cached[0][t] for t in range(8)])
    assert _rel(np.stack(res["orbits"][1]), np.stack(o1)) < 1e-9
