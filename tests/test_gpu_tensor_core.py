"""Tensor-core Schur complements of the FP32 factorization (B200).

FP32 factor batches send the Schur complement F22 -= L21 U12 of every
supernode with at least ``ORBIT_B200_TC_MIN_N`` pivots to the tcgen05 kernel
(split tf32 operands, fp32 accumulation in tensor memory); ``ORBIT_B200_TC=0``
keeps all of them on the CUDA-core GEMM.  On a small grid with the threshold
lowered so that most supernodes take the tensor-core path, the chained solves
through both factorizations must agree to FP32 rounding (1e-5 relative), must
not be bit-identical (the other kernel really ran), and both must match the
FP64 chain to 1e-5.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chain(sym, mets_T, sinks, precision, x, tc):
    from orbit_b200 import device
    old = os.environ.get("ORBIT_B200_TC")
    os.environ["ORBIT_B200_TC"] = tc
    try:
        fb = device.FactorBatch(sym, x.shape[0], precision)
        fb.numeric(mets_T * x.shape[0], sinks)
        y = fb.chain(x.clone(), refine=False).cpu().numpy()
        fb.close()
    finally:
        if old is None:
            del os.environ["ORBIT_B200_TC"]
        else:
            os.environ["ORBIT_B200_TC"] = old
    return y


def test_tensor_core_schur_matches_cuda_cores():
    import torch
    from orbit_b200 import device, synthetic
    from orbit_b200.symbolic import Symbolic
    rng = np.random.default_rng(11)
    nz, ny, nx = 10, 24, 28
    met = synthetic.make_met(11, nz, ny, nx)
    mets = [device.MetDevice(g) for g in met]
    T = [device.assemble_transport(m) for m in mets]
    n = 2
    sinks = []
    for k in range(n):
        spc = synthetic.make_species(20 + k, nz, ny, nx)
        sinks += [torch.as_tensor(d, device="cuda") for d in spc.sink_diag(met)]
    # no one-CTA fronts: every supernode with n >= 16 takes the tensor cores
    saved = {k: os.environ.get(k) for k in ("ORBIT_B200_TC_MIN_N", "ORBIT_B200_FUSED_MAX_N")}
    os.environ["ORBIT_B200_TC_MIN_N"] = "16"
    os.environ["ORBIT_B200_FUSED_MAX_N"] = "0"
    try:
        sym = Symbolic(nz, ny, nx, 32)
    finally:
        for k, v in saved.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    assert sym.info["fused_fronts"] == 0
    x = torch.as_tensor(rng.standard_normal((n, sym.N)), device="cuda")
    ref = _chain(sym, T, sinks, 64, x, "1")
    y_tc = _chain(sym, T, sinks, 32, x, "1")
    y_cc = _chain(sym, T, sinks, 32, x, "0")
    scale = np.abs(ref).max()
    d_tc = np.abs(y_tc - ref).max() / scale
    d_cc = np.abs(y_cc - ref).max() / scale
    d = np.abs(y_tc - y_cc).max() / scale
    assert d_tc < 1e-5 and d_cc < 1e-5, (d_tc, d_cc)
    assert 0.0 < d < 1e-5, d
