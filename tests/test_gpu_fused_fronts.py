"""One-CTA fronts of the numeric factorization (B200).

Supernodes with at most 64 pivots whose pivot-block inverses and panels fit
in shared memory are factored whole by one CTA (k_front); every other
supernode goes through the blocked DIAG / PANEL / UPDATE / INV / product /
Schur launches (and, in FP32, the tensor-core GEMMs).  Both paths compute the
same SQ, Pb, Qr and Schur complement, so chained solves through a
factorization with the one-CTA fronts and through one without them
(``ORBIT_B200_FUSED_MAX_N=0``) must agree to rounding: 1e-12 relative in
FP64 and 1e-5 in FP32, on a grid where both kinds of supernode occur.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _symbolic(shape, leaf, fused):
    from orbit_b200.symbolic import Symbolic
    old = os.environ.get("ORBIT_B200_FUSED_MAX_N")
    if not fused:
        os.environ["ORBIT_B200_FUSED_MAX_N"] = "0"
    try:
        return Symbolic(*shape, leaf_cells=leaf)
    finally:
        if old is None:
            os.environ.pop("ORBIT_B200_FUSED_MAX_N", None)
        else:
            os.environ["ORBIT_B200_FUSED_MAX_N"] = old


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-5)])
def test_fused_fronts_match_blocked_path(precision, tol):
    import torch
    from orbit_b200 import device, synthetic
    shape = (8, 22, 26)
    met = synthetic.make_met(5, *shape, cmfmc_frac=0.3)
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    n = 2
    sinks = []
    for k in range(n):
        spc = synthetic.make_species(40 + k, *shape)
        sinks += [torch.as_tensor(d, device="cuda") for d in spc.sink_diag(met)]
    sym_f = _symbolic(shape, 48, True)
    sym_b = _symbolic(shape, 48, False)
    assert sym_b.info["fused_fronts"] == 0
    assert 0 < sym_f.info["fused_fronts"] < sym_f.info["nsuper"] - 1  # both kinds present
    x = torch.as_tensor(np.random.default_rng(3).standard_normal((n, sym_f.N)), device="cuda")
    out = []
    for sym in (sym_f, sym_b):
        fb = device.FactorBatch(sym, n, precision)
        fb.numeric(T * n, sinks)
        out.append((fb.chain(x.clone(), refine=False).cpu().numpy(),
                    fb.chain(x.clone(), trans=True, refine=False).cpu().numpy()))
        fb.close()
    for a, b in zip(out[0], out[1]):
        assert np.abs(a - b).max() <= tol * np.abs(b).max()
