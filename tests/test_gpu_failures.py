"""Failure paths on the device, none of which faults or hangs the GPU:
a bounded wait that runs out (status read, context usable afterwards), a
zero pivot, and GMRES non-convergence (the reference's WARNING and return)."""
import numpy as np
import pytest

import golden_io

pytestmark = pytest.mark.gpu

Z = golden_io.load()
MET = golden_io.met_list(Z)
SPC = golden_io.species(Z)


def _batch(precision=64):
    import torch
    from orbit_b200 import device
    from orbit_b200.symbolic import Symbolic
    mets = [device.MetDevice(g) for g in MET]
    T = [device.assemble_transport(m) for m in mets]
    sinks = [torch.as_tensor(x, device="cuda") for x in SPC.sink_diag(MET)]
    fb = device.FactorBatch(Symbolic(MET[0].nz, MET[0].ny, MET[0].nx, leaf_cells=8), 1, precision)
    fb.numeric(T, sinks)
    return fb, T, sinks


def test_bounded_wait_times_out_and_context_stays_usable():
    import torch
    from orbit_b200 import _lib
    fb, _, _ = _batch()
    rc = _lib.lib().orbit_selftest_wait_timeout(fb._h, torch.cuda.current_stream().cuda_stream)
    assert rc == 4  # ORBIT_ERR_TIMEOUT
    v = torch.as_tensor(Z["mono_v"], device="cuda")[None]
    Mv = fb.chain(v).cpu().numpy()[0]
    assert np.abs(Mv - Z["mono_Mv"]).max() <= 1e-12 * np.abs(Z["mono_Mv"]).max()


def test_zero_pivot_reported():
    import torch
    from orbit_b200 import device, _lib
    from orbit_b200.symbolic import Symbolic
    g = MET[0]
    T = torch.zeros((7, g.N), dtype=torch.float64, device="cuda")
    T[0] = -1.0  # with dtau = 1, A = I + T has an exactly zero diagonal
    fb = device.FactorBatch(Symbolic(g.nz, g.ny, g.nx, leaf_cells=8), 1, 64)
    with pytest.raises(_lib.OrbitError) as ei:
        fb.numeric([T] * 8, None, dtau=1.0)
    assert ei.value.code == 5
    fb2, _, _ = _batch()  # the device is fine afterwards
    v = torch.as_tensor(Z["mono_v"], device="cuda")[None]
    assert np.all(np.isfinite(fb2.chain(v).cpu().numpy()))


def test_gmres_nonconvergence_warns_and_returns(capsys):
    import torch
    fb, _, _ = _batch()
    e = torch.as_tensor(SPC.emis, device="cuda")[None]
    orb, info = fb.solve(e, tol=1e-15, maxiter=1, restart=1)
    assert "WARNING: GMRES did not converge" in capsys.readouterr().out
    assert info[0, 4] == 0.0 and np.all(np.isfinite(orb.cpu().numpy()))
