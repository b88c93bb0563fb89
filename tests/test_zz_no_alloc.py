"""The allocation-free adjoint entry point, pfb_nufft_adj_noalloc, called
through the C ABI and checked against the oracle and against the
workspace-taking pfb_nufft_adj.

pfb_nufft_adj_noalloc serves callers that cannot call cudaMalloc at apply time
(for example code inside a framework that owns all device memory through its
own pool, or a real-time loop with a fixed memory budget).  Its scratch is one
static device array shared by all calls, so every case makes two calls in a
row with different inputs: the second must not be disturbed by what the first
left behind.  The cases cover 2D and 3D plans, both norms, the accumulate flag,
and a subspace basis with B0 time segments, each sized to fit the 64 MiB array.
This file runs last in the suite and also passes on its own.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402

TOL = 1e-5  # same rel-L2 tolerance as the other parity tests


def _radial(nspokes, nread, N, rot=0.0):
    ga = np.pi / ((1 + 5 ** 0.5) / 2)
    ang = np.arange(nspokes) * ga + rot
    kr = (np.arange(nread) - nread // 2) / nread * N
    return np.stack([np.cos(ang)[:, None] * kr, np.sin(ang)[:, None] * kr], -1).astype(np.float32)


def _crandn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return orc.rel_l2(a, b)


def _case(name):
    """(coord, shape, plan keywords, batch, basis or None) of each case."""
    rng = np.random.default_rng(sum(map(ord, name)))
    if name == "2d":
        return _radial(40, 128, 64), (64, 64), dict(width=4, oversamp=2.0), 4, None
    if name == "3d-ortho":
        N = (24, 24, 24)
        coord = ((rng.random((30, 64, 3)) - 0.5) * 24).astype(np.float32)
        return coord, N, dict(width=4, oversamp=1.25), 3, None
    if name == "2d-basis-b0":
        N, F, K = 32, 5, 3
        coord = np.stack([_radial(6, 48, N, rot=0.2 * f) for f in range(F)])
        basis = np.linalg.qr(_crandn(rng, F, K))[0].astype(np.complex64)
        yy, xx = np.mgrid[:N, :N] / N - 0.5
        b0 = (150 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 80).astype(np.float32)
        kw = dict(width=4, oversamp=2.0, zmap=b0, L=4, nbins=40, dt=5e-3 / 48)
        return coord, (N, N), kw, 2, basis
    raise KeyError(name)


@pytest.mark.parametrize("name, norm, accumulate", [("2d", None, False), ("3d-ortho", "ortho", False),
                                                    ("2d", None, True), ("2d-basis-b0", None, False)])
def test_noalloc_adjoint_matches_oracle_and_workspace_adjoint_twice(name, norm, accumulate):
    import pyfourier_b200 as pf
    from pyfourier_b200 import _lib
    from pyfourier_b200._nufft import _Ctx, norm_code

    L = _lib.load()
    coord, shape, kw, B, basis = _case(name)
    gplan = pf.plan_nufft(torch.as_tensor(coord), shape, device="cuda:0", **kw)
    oplan = orc.plan_nufft(coord, shape, **kw)
    bt = torch.as_tensor(basis, device="cuda:0") if basis is not None else None
    ctx = _Ctx(gplan, bt, None, norm_code(norm))
    seg = (0, gplan.zmap_s_kernel.shape[0]) if gplan.zmap_s_kernel is not None else (0, 1)
    o = ctx.opts(B, seg, _lib.PFB_FLAG_ACCUMULATE if accumulate else 0)
    h = gplan.interpolator.handle
    nplanes = o.nseg * o.batch * o.ncoeff
    nbytes = ctypes.c_size_t()
    # set-up: the cuFFT plan for these planes (may allocate), then the no-alloc
    # entry point's own set-up call (batch 0: only the scratch address lookup)
    _lib.check(L.pfb_workspace_size(h, nplanes, ctypes.byref(nbytes)))
    o0 = ctx.opts(0, seg)
    _lib.check(L.pfb_nufft_adj_noalloc(h, ctypes.byref(o0), None, None,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    ws = ctx.workspace(o)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(1)
    M = gplan.interpolator.total_samples
    F = gplan.interpolator.nframes
    for call in range(2):
        yk = _crandn(rng, B, *coord.shape[:-1])
        y = torch.as_tensor(yk.reshape(B, M), device="cuda:0")
        prev = _crandn(rng, B, ctx.C, *shape) if accumulate else np.zeros((B, ctx.C, *shape), np.complex64)
        ref = torch.as_tensor(prev, device="cuda:0")
        out = torch.as_tensor(prev, device="cuda:0") if accumulate else torch.full_like(ref, float("nan"))
        _lib.check(L.pfb_nufft_adj(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()),
                                   ctypes.c_void_p(ref.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                   stream))
        _lib.check(L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()),
                                           ctypes.c_void_p(out.data_ptr()), stream))
        torch.cuda.synchronize()
        assert torch.isfinite(out).all(), f"call {call}"
        # the oracle takes k-space as (B, [F,] nviews, nsamples) and returns (B, [C,] *shape)
        yo = yk if F > 1 or basis is not None else yk.reshape(B, *coord.shape[:-1])
        xo = orc.nufft_adj(yo, oplan, basis=basis, norm=norm).reshape(B, ctx.C, *shape) + prev
        e_oracle, e_ws = _rel(out, xo), _rel(out, ref.cpu().numpy())
        assert e_oracle < TOL and e_ws < TOL, (call, e_oracle, e_ws)


def test_noalloc_rejects_requests_beyond_the_static_scratch():
    import pyfourier_b200 as pf
    from pyfourier_b200 import _lib

    L = _lib.load()
    plan = pf.plan_nufft(torch.as_tensor(_radial(40, 128, 64)), (64, 64), width=4, oversamp=2.0, device="cuda:0")
    h = plan.interpolator.handle
    o = _lib.ApplyT()
    # planes of 128^2 complex64 (128 KiB each): enough of them to exceed the 64 MiB array
    big = (64 << 20) // (128 * 128 * 8) + 8
    o.batch, o.ncoeff, o.nseg, o.norm, o.flags = big, 1, 1, _lib.PFB_NORM_NONE, 0
    nbytes = ctypes.c_size_t()
    _lib.check(L.pfb_workspace_size(h, big, ctypes.byref(nbytes)))
    y = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    out = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.PFB_ERR_INVALID
    assert b"static" in L.pfb_last_error()


def test_noalloc_requires_cufft_plan_set_up_and_checks_arguments():
    import pyfourier_b200 as pf
    from pyfourier_b200 import _lib

    L = _lib.load()
    plan = pf.plan_nufft(torch.as_tensor(_radial(40, 128, 64)), (64, 64), width=4, oversamp=2.0, device="cuda:0")
    h = plan.interpolator.handle
    o = _lib.ApplyT()
    o.batch, o.ncoeff, o.nseg, o.norm, o.flags = 7, 1, 1, _lib.PFB_NORM_NONE, 0  # no set-up for 7 planes
    y = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    out = torch.zeros((1,), dtype=torch.complex64, device="cuda:0")
    st_ptr = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 st_ptr)
    assert st == _lib.PFB_ERR_INVALID
    assert b"pfb_workspace_size" in L.pfb_last_error()
    # the same checks as pfb_nufft_adj (shared argument validation)
    o.norm = 7
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 st_ptr)
    assert st == _lib.PFB_ERR_INVALID and b"norm" in L.pfb_last_error()
    o.norm, o.batch = _lib.PFB_NORM_NONE, 1 << 31
    st = L.pfb_nufft_adj_noalloc(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 st_ptr)
    assert st == _lib.PFB_ERR_INVALID and b"too many channels" in L.pfb_last_error()
