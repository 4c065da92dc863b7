"""The allocation-free SGS entry point (fsl_dynamic_smagorinsky_noalloc).

It serves callers that cannot allocate device memory (their own allocator
owns the device memory, or they must not stall on cudaFree); it takes caller
buffers and uses a fixed static scratch array instead.  This file is
collected last on purpose: it runs after every other test, and also passes
alone in a fresh process.  The entry point is called through the C ABI and
must give the same SGS viscosity as the context-based fsl_dynamic_smagorinsky,
bit for bit (the tolerance of all plain-FP64 parity tests), on two calls in a
row with different inputs (the scratch keeps the previous call's contents).
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import random_state, spatial_params, temporal_params

pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.fsl_dynamic_smagorinsky_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                   C.c_double, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _context_mu(fsl, p, state):
    """Padded U (ghost layer filled) and mu from the context-based entry point."""
    d = fsl.Domain(p)
    d.upload_state(state)
    d.ghost_bc()
    d.dynamic_smagorinsky()
    U = np.stack([d.cells(0, v) for v in range(4)])
    mu = d.cells(3)
    d.close()
    return U, mu


@pytest.mark.parametrize("make_p", [lambda: spatial_params(L=24, H=16, D=12),
                                    lambda: temporal_params(L=32, H=16, D=16),
                                    # near the size limit, non-cubic: 66 x 34 x 34 padded cells
                                    lambda: temporal_params(L=64, H=32, D=32)])
def test_noalloc_matches_context_two_calls(make_p):
    import torch
    import freeshearlayer_b200 as fsl
    fn = _bind(fsl.lib())
    p = make_p()
    stream = torch.cuda.current_stream()
    for call, seed in enumerate((31, 32)):
        U_host, mu_ref = _context_mu(fsl, p, random_state(p, seed))
        U_dev = torch.from_numpy(np.ascontiguousarray(U_host)).cuda()
        mu_dev = torch.full(mu_ref.shape, float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = fn(U_dev.data_ptr(), mu_dev.data_ptr(), p["LEN"], p["HIG"], p["DEP"],
                p["deltaX"], p["deltaY"], p["deltaZ"], C.c_void_p(stream.cuda_stream))
        assert rc == 0, "call %d returned %d" % (call, rc)
        stream.synchronize()
        mu = mu_dev.cpu().numpy()
        assert np.count_nonzero(mu_ref) > 0
        assert np.array_equal(mu, mu_ref), "call %d: max |d| = %g" % (call, np.max(np.abs(mu - mu_ref)))


def test_noalloc_rejects_oversize():
    import torch
    import freeshearlayer_b200 as fsl
    fn = _bind(fsl.lib())
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    # (LEN+2)(HIG+2)(DEP+2) above FSL_NOALLOC_MAX_CELLS: rejected before any device work
    rc = fn(buf.data_ptr(), buf.data_ptr(), 128, 64, 64, 1.0, 1.0, 1.0, None)
    assert rc == -9


def test_noalloc_leaves_a_pending_error_to_its_owner():
    """A CUDA error left pending by the caller's earlier work (here a refused
    host-side allocation request, which touches no device) is reported as
    FSL_ERR_CUDA before any work starts, and stays pending for its owner."""
    import torch
    import freeshearlayer_b200 as fsl
    fn = _bind(fsl.lib())
    rt = C.CDLL("libcudart.so.12")  # the runtime instance the library shares
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaGetLastError.restype = C.c_int
    rt.cudaPeekAtLastError.restype = C.c_int
    p = temporal_params(L=16, H=8, D=8)
    U = torch.zeros(4 * 18 * 10 * 10, dtype=torch.float64, device="cuda")
    mu = torch.full((18 * 10 * 10,), 7.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert rt.cudaGetLastError() == 0
    ptr = C.c_void_p()
    assert rt.cudaMalloc(C.byref(ptr), 1 << 62) != 0  # far beyond any device: refused
    pending = rt.cudaPeekAtLastError()
    assert pending != 0
    rc = fn(U.data_ptr(), mu.data_ptr(), p["LEN"], p["HIG"], p["DEP"], p["deltaX"], p["deltaY"],
            p["deltaZ"], None)
    assert rc == -3
    assert rt.cudaGetLastError() == pending  # still the caller's, now cleared by its owner
    torch.cuda.synchronize()
    assert bool(torch.all(mu == 7.0))       # no work was queued
