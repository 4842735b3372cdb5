"""The allocation-free FCT entry point against the allocating one (B200).

orbit_fct_source_noalloc serves callers that cannot allocate device memory
where they apply the FCT correction (a host model that owns its whole device
budget through its own pool, or a time loop that must not stall on the
synchronization a cudaFree can cause); its scratch is a static device array
shared by all calls.  Calls in a row, with different inputs (limited and
unlimited), must each
match orbit_fct_source called through the same C ABI, to the 1e-12 relative
tolerance of the FCT parity tests; the second call also shows that nothing
left in the shared scratch by the first leaks into it.  This file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import golden_io

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_noalloc_fct_matches_allocating_entry_point():
    import torch
    from orbit_b200 import _lib, device

    z = golden_io.load()
    met = golden_io.met_list(z)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    c0 = torch.as_tensor(z["fct_c"], device="cuda")
    inputs = [
        (met[0], torch.stack([c0, 2.0 * c0]), 1),          # limited, two vectors
        (met[1], torch.stack([c0.flip(0), c0 * 0.5]), 1),  # another bin, new data
        (met[2], torch.stack([c0 * 3.0, c0.flip(0)]), 0),  # unlimited: no R+/R- pass
    ]
    for g, c, limited in inputs:
        md = device.MetDevice(g)
        c = c.contiguous()
        n_vec = c.shape[0]
        ref = torch.empty_like(c)
        out = torch.full_like(c, float("nan"))
        _lib.check(L.orbit_fct_source(md.nz, md.ny, md.nx, C.byref(md.struct), n_vec, _lib.ptr(c),
                                      10800.0, limited, _lib.ptr(ref), stream))
        _lib.check(L.orbit_fct_source_noalloc(md.nz, md.ny, md.nx, C.byref(md.struct), n_vec,
                                              _lib.ptr(c), 10800.0, limited, _lib.ptr(out), stream))
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert _rel(o, r) < 1e-12


def test_noalloc_fct_rejects_oversize_requests():
    import torch
    from orbit_b200 import _lib, device

    z = golden_io.load()
    md = device.MetDevice(golden_io.met_list(z)[0])
    L = _lib.lib()
    n_vec = (1 << 20) // md.N + 1
    c = torch.zeros((n_vec, md.N), dtype=torch.float64, device="cuda")
    d = torch.empty_like(c)
    rc = L.orbit_fct_source_noalloc(md.nz, md.ny, md.nx, C.byref(md.struct), n_vec, _lib.ptr(c),
                                    10800.0, 1, _lib.ptr(d), torch.cuda.current_stream().cuda_stream)
    assert rc == 1
    assert b"exceeds the static scratch limit" in L.orbit_last_error()
