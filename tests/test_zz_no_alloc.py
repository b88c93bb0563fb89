"""The allocation-free adjoint entry point, pfb_nufft_adj_noalloc, against the
workspace-taking pfb_nufft_adj.

pfb_nufft_adj_noalloc serves callers that cannot call cudaMalloc at apply time
(for example code inside a framework that owns all device memory through its
own pool, or a real-time loop with a fixed memory budget).  Its scratch is one
static device array shared by all calls, so these tests also check that a
second call in a row is not disturbed by what the first one left behind.
This file runs last in the suite and also passes on its own.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5  # same rel-L2 tolerance as the other parity tests


def _radial(nspokes, nread, N):
    ga = np.pi / ((1 + 5 ** 0.5) / 2)
    ang = np.arange(nspokes) * ga
    kr = (np.arange(nread) - nread // 2) / nread * N
    return np.stack([np.cos(ang)[:, None] * kr, np.sin(ang)[:, None] * kr], -1).astype(np.float32)


def _rel(a, b):
    a = a.detach().cpu().numpy().astype(np.complex128)
    b = b.detach().cpu().numpy().astype(np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _setup(N=64, nspokes=40, nread=128, B=4):
    import pyfourier_b200 as pf
    from pyfourier_b200 import _lib

    L = _lib.load()
    plan = pf.plan_nufft(torch.as_tensor(_radial(nspokes, nread, N)), (N, N), width=4, oversamp=2.0,
                         device="cuda:0")
    h = plan.interpolator.handle
    o = _lib.ApplyT()
    o.batch, o.ncoeff, o.nseg, o.norm, o.flags = B, 1, 1, _lib.PFB_NORM_NONE, 0
    return L, _lib, plan, h, o


def test_noalloc_adjoint_matches_workspace_adjoint_twice():
    L, _lib, plan, h, o = _setup()
    B, M = o.batch, plan.interpolator.total_samples
    nbytes = ctypes.c_size_t()
    # set-up: creates the cuFFT plan for B planes (this call may allocate)
    _lib.check(L.pfb_workspace_size(h, B, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda:0")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(0)
    for call in range(2):
        y = torch.as_tensor((rng.standard_normal((B, M)) + 1j * rng.standard_normal((B, M))).astype(np.complex64),
                            device="cuda:0")
        ref = torch.empty((B, 1, 64, 64), dtype=torch.complex64, device="cuda:0")
        out = torch.full_like(ref, float("nan"))
        _lib.check(L.pfb_nufft_adj(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                   ctypes.c_void_p(ws.data_ptr()), ws.numel(), stream))
        _lib.check(L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()),
                                           ctypes.c_void_p(out.data_ptr()), stream))
        torch.cuda.synchronize()
        assert torch.isfinite(out).all(), f"call {call}"
        assert _rel(out, ref) < TOL, f"call {call}"


def test_noalloc_rejects_requests_beyond_the_static_scratch():
    L, _lib, plan, h, o = _setup()
    # planes of 128^2 complex64 (128 KiB each): enough of them to exceed the 64 MiB array
    big = (64 << 20) // (128 * 128 * 8) + 8
    o.batch = big
    nbytes = ctypes.c_size_t()
    _lib.check(L.pfb_workspace_size(h, big, ctypes.byref(nbytes)))
    y = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    out = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.PFB_ERR_INVALID
    assert b"static" in L.pfb_last_error()


def test_noalloc_requires_cufft_plan_set_up():
    L, _lib, plan, h, o = _setup()
    o.batch = 7  # no pfb_workspace_size call for 7 planes on this plan
    y = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    out = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.PFB_ERR_INVALID
    assert b"pfb_workspace_size" in L.pfb_last_error()
