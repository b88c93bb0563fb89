"""GPU parity of the libpfb200 stages against the reference's own Numba kernels
(golden vectors in tests/golden/kernels.npz), called through the C ABI."""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402


def _lib():
    from pyfourier_b200 import _lib

    return _lib


def _plan(coord, N, osf, w):
    import pyfourier_b200 as pf

    return pf.plan_nufft(torch.as_tensor(coord), tuple(int(n) for n in N), width=tuple(int(x) for x in w),
                         oversamp=tuple(float(o) for o in osf), device="cuda:0")


def _opts(batch, ncoeff, basis=None):
    L = _lib()
    o = L.ApplyT()
    o.batch, o.ncoeff, o.nseg, o.norm, o.flags = batch, ncoeff, 1, 0, 0
    o.basis = basis.data_ptr() if basis is not None else None
    return o


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def rel(a, b):
    return orc.rel_l2(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("w", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("osf", [1.25, 2.0])
def test_tables_edge_coords(golden, w, osf):
    c = golden["tab_coord"]
    N = int(golden["tab_N"])
    plan = _plan(c[None, None, :, None], (N,), (osf,), (w,))
    idx, val = plan.interpolator.tables(0)
    tag = f"tab_w{w}_os{osf}"
    np.testing.assert_array_equal(idx.cpu().numpy(), golden[tag + "_index"])
    np.testing.assert_allclose(val.cpu().numpy(), golden[tag + "_value"], rtol=3e-6, atol=1e-7)


@pytest.mark.parametrize("d", [1, 2, 3])
def test_tables_and_scale(golden, d):
    p = f"k{d}d_"
    coord = golden[p + "coord"]
    F = coord.shape[0]
    plan = _plan(coord[:, None], golden[p + "N"], golden[p + "osf"], golden[p + "width"])
    ip = plan.interpolator
    for a in range(d):
        idx, val = ip.tables(a)
        np.testing.assert_array_equal(idx.cpu().numpy().reshape(F, -1, idx.shape[-1]), golden[p + f"index{a}"])
        np.testing.assert_allclose(val.cpu().numpy().reshape(F, -1, val.shape[-1]), golden[p + f"value{a}"],
                                   rtol=3e-6, atol=1e-7)
    ref_scale = orc.kernel_scaling([float(b) for b in golden[p + "beta"]], golden[p + "width"])
    assert ip.scale == pytest.approx(ref_scale, rel=1e-12)


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("subspace", [False, True])
def test_spread_interp_vs_reference(golden, d, subspace):
    L = _lib()
    lib = L.load()
    p = f"k{d}d_"
    coord = golden[p + "coord"]
    F, M = coord.shape[:2]
    plan = _plan(coord[:, None], golden[p + "N"], golden[p + "osf"], golden[p + "width"])
    h = plan.interpolator.handle
    os_ = tuple(int(v) for v in golden[p + "os"])
    nc = golden[p + "noncart"]  # (F, B, M)
    B = nc.shape[1]
    y = torch.as_tensor(np.ascontiguousarray(nc.transpose(1, 0, 2).reshape(B, F * M))).cuda()
    basis = torch.as_tensor(golden[p + "basis"]).cuda() if subspace else None
    C = basis.shape[1] if subspace else F
    grid = torch.empty((B, C, *os_), dtype=torch.complex64, device="cuda")
    o = _opts(B, C, basis)
    L.check(lib.pfb_spread(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(grid.data_ptr()),
                           0, _stream()))
    ref = golden[p + ("spread_sub" if subspace else "spread")]  # (C, B, *os)
    assert rel(grid.cpu().numpy().swapaxes(0, 1), ref) < 1e-5

    gin = golden[p + ("grid_in_sub" if subspace else "grid_in")]  # (C, B, *os)
    g = torch.as_tensor(np.ascontiguousarray(gin.swapaxes(0, 1))).cuda()
    out = torch.empty((B, F * M), dtype=torch.complex64, device="cuda")
    L.check(lib.pfb_interp(h, ctypes.byref(o), ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                           0, _stream()))
    ref = golden[p + ("interp_sub" if subspace else "interp")]  # (F, B, M)
    got = out.cpu().numpy().reshape(B, F, M).transpose(1, 0, 2)
    assert rel(got, ref) < 1e-5


def test_spread_is_deterministic_in_layout_and_fft_shift(golden):
    """fft_layout=1 is the centred grid rolled by -(n_os // 2) on every axis."""
    L = _lib()
    lib = L.load()
    p = "k2d_"
    coord = golden[p + "coord"]
    F, M = coord.shape[:2]
    plan = _plan(coord[:, None], golden[p + "N"], golden[p + "osf"], golden[p + "width"])
    h = plan.interpolator.handle
    os_ = tuple(int(v) for v in golden[p + "os"])
    nc = golden[p + "noncart"]
    B = nc.shape[1]
    y = torch.as_tensor(np.ascontiguousarray(nc.transpose(1, 0, 2).reshape(B, F * M))).cuda()
    g0 = torch.empty((B, F, *os_), dtype=torch.complex64, device="cuda")
    g1 = torch.empty_like(g0)
    o = _opts(B, F)
    L.check(lib.pfb_spread(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(g0.data_ptr()), 0, _stream()))
    L.check(lib.pfb_spread(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(g1.data_ptr()), 1, _stream()))
    rolled = torch.fft.ifftshift(g0, dim=(-2, -1))
    assert rel(g1.cpu(), rolled.cpu()) < 1e-6


def _pipeline_both(plan, x, y, basis=None, zs=None, zt=None, L=1):
    """pfb_nufft_fwd / adj with a planar-size workspace (planar kernels) and with
    pfb_apply_workspace_size bytes (channel-interleaved kernels)."""
    Lb = _lib()
    lib = Lb.load()
    h = plan.interpolator.handle
    B, C = x.shape[0], x.shape[1]
    o = _opts(B, C, basis)
    if zs is not None:
        o.nseg, o.b0_time, o.b0_space = L, zt.data_ptr(), zs.data_ptr()
    nplanes = o.nseg * B * C
    small, big = ctypes.c_size_t(), ctypes.c_size_t()
    Lb.check(lib.pfb_workspace_size(h, nplanes, ctypes.byref(small)))
    Lb.check(lib.pfb_apply_workspace_size(h, ctypes.byref(o), ctypes.byref(big)))
    assert big.value > small.value
    res = {}
    for name, n in (("planar", small.value), ("fast", big.value)):
        ws = torch.empty(n, dtype=torch.uint8, device="cuda")
        k = torch.empty((B, plan.interpolator.total_samples), dtype=torch.complex64, device="cuda")
        im = torch.empty_like(x)
        Lb.check(lib.pfb_nufft_fwd(h, ctypes.byref(o), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(k.data_ptr()),
                                   ctypes.c_void_p(ws.data_ptr()), n, _stream()))
        Lb.check(lib.pfb_nufft_adj(h, ctypes.byref(o), ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(im.data_ptr()),
                                   ctypes.c_void_p(ws.data_ptr()), n, _stream()))
        res[name] = (k, im)
    assert rel(res["fast"][0].cpu(), res["planar"][0].cpu().numpy()) < 1e-5
    assert rel(res["fast"][1].cpu(), res["planar"][1].cpu().numpy()) < 1e-5


@pytest.mark.parametrize("case", ["2d_coils", "2d_frames", "3d", "basis", "b0", "3d_w6_odd", "2d_single_tile",
                                  "2d_single_tile_32ch", "3d_w6_32ch", "1d_32ch", "3d_12ch", "3d_single_tile",
                                  "3d_b0_basis"])
def test_interleaved_pipeline_matches_planar(case):
    rng = np.random.default_rng(21)
    crn = lambda *s: torch.as_tensor((rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)).cuda()  # noqa: E731
    if case == "2d_coils":
        N = (96, 96)
        coord = ((rng.random((1, 60, 192, 2)) - 0.5) * 96).astype(np.float32)
        plan = _plan(coord, N, (2.0, 2.0), (4, 4))
        _pipeline_both(plan, crn(12, 1, *N), crn(12, 60 * 192))
    elif case == "2d_frames":
        N = (40, 48)
        coord = ((rng.random((5, 7, 64, 2)) - 0.5) * np.array([48, 40])).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.5), (5, 4))
        _pipeline_both(plan, crn(3, 5, *N), crn(3, 5 * 7 * 64))
    elif case == "3d":
        N = (30, 28, 26)
        coord = ((rng.random((1, 50, 80, 3)) - 0.5) * np.array([26, 28, 30])).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.25, 1.25), (4, 4, 4))
        _pipeline_both(plan, crn(33, 1, *N), crn(33, 50 * 80))
    elif case == "2d_single_tile":
        # a 24 x 24 oversampled grid is one tile: taps wrap around inside the tile
        N = (12, 12)
        coord = np.concatenate([((rng.random((1, 1, 60, 2)) - 0.5) * 12),
                                np.full((1, 1, 4, 2), -6.0), np.full((1, 1, 4, 2), 5.9)], axis=2).astype(np.float32)
        plan = _plan(coord, N, (2.0, 2.0), (4, 4))
        _pipeline_both(plan, crn(3, 1, *N), crn(3, 68))
    elif case == "2d_single_tile_32ch":
        # 32 channels per warp with taps wrapping inside a single tile
        N = (12, 12)
        coord = np.concatenate([((rng.random((1, 1, 60, 2)) - 0.5) * 12),
                                np.full((1, 1, 4, 2), -6.0), np.full((1, 1, 4, 2), 5.9)], axis=2).astype(np.float32)
        plan = _plan(coord, N, (2.0, 2.0), (4, 4))
        _pipeline_both(plan, crn(40, 1, *N), crn(40, 68))
    elif case == "3d_w6_32ch":
        N = (17, 21, 19)
        coord = ((rng.random((1, 20, 50, 3)) - 0.5) * np.array([19, 21, 17])).astype(np.float32)
        plan = _plan(coord, N, (2.0, 1.5, 2.0), (6, 5, 7))
        _pipeline_both(plan, crn(32, 1, *N), crn(32, 20 * 50))
    elif case == "1d_32ch":
        N = (300,)
        coord = ((rng.random((1, 4, 100, 1)) - 0.5) * 300).astype(np.float32)
        plan = _plan(coord, N, (1.25,), (4,))
        _pipeline_both(plan, crn(32, 1, *N), crn(32, 400))
    elif case == "3d_w6_odd":
        N = (17, 21, 19)
        coord = ((rng.random((1, 20, 50, 3)) - 0.5) * np.array([19, 21, 17])).astype(np.float32)
        plan = _plan(coord, N, (2.0, 1.5, 2.0), (6, 5, 7))
        _pipeline_both(plan, crn(5, 1, *N), crn(5, 20 * 50))
    elif case == "3d_12ch":
        N = (24, 22, 20)
        coord = ((rng.random((1, 40, 60, 3)) - 0.5) * np.array([20, 22, 24])).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.25, 1.25), (4, 4, 4))
        _pipeline_both(plan, crn(12, 1, *N), crn(12, 40 * 60))
    elif case == "3d_single_tile":
        # a 6^3 image at osf 1.25 is an 8^3 grid, one tile: taps wrap around inside it on every axis
        N = (6, 6, 6)
        coord = np.concatenate([((rng.random((1, 1, 50, 3)) - 0.5) * 6),
                                np.full((1, 1, 3, 3), -3.0), np.full((1, 1, 3, 3), 2.95)], axis=2).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.25, 1.25), (4, 4, 4))
        _pipeline_both(plan, crn(3, 1, *N), crn(3, 56))
    elif case == "3d_b0_basis":
        # 3D subspace with B0 segments: channels = segments x batch x coefficients = 12
        N = (16, 18, 20)
        F, K, Lseg = 4, 2, 3
        coord = ((rng.random((F, 6, 40, 3)) - 0.5) * np.array([20, 18, 16])).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.25, 1.25), (4, 4, 4))
        zt = crn(Lseg, 40)
        zs = crn(Lseg, 16 * 18 * 20)
        _pipeline_both(plan, crn(2, K, *N), crn(2, F * 6 * 40), basis=crn(F, K), zs=zs, zt=zt, L=Lseg)
    elif case == "basis":
        N = (32, 32)
        F, K = 6, 3
        coord = ((rng.random((F, 9, 48, 2)) - 0.5) * 32).astype(np.float32)
        plan = _plan(coord, N, (2.0, 2.0), (4, 4))
        basis = crn(F, K)
        _pipeline_both(plan, crn(4, K, *N), crn(4, F * 9 * 48), basis=basis)
    else:
        N = (32, 32)
        Lseg = 5
        coord = ((rng.random((1, 12, 64, 2)) - 0.5) * 32).astype(np.float32)
        plan = _plan(coord, N, (1.25, 1.25), (4, 4))
        zt = crn(Lseg, 64)
        zs = crn(Lseg, 32 * 32)
        _pipeline_both(plan, crn(6, 1, *N), crn(6, 12 * 64), zs=zs, zt=zt, L=Lseg)


def _sorted_order(plan):
    M = plan.interpolator.total_samples
    order = torch.empty(M, dtype=torch.int32, device="cuda:0")
    _lib().check(_lib().load().pfb_plan_order(plan.interpolator.handle, ctypes.c_void_p(order.data_ptr()),
                                              _stream()))
    return order.cpu().numpy()


def _bin_keys(plan, op, frame, ndim, w=4):
    """Bin keys ((tile << d | edge code) * F + frame) from the oracle's first taps;
    tile t of an axis covers [t * tile - offset, (t + 1) * tile - offset) of the grid."""
    tile = plan.interpolator.tile[::-1]  # (x, y, z)
    off = plan.interpolator.tile_offset[::-1]
    nos = op.os_shape[::-1]
    M = frame.size
    key_bin = np.zeros(M, np.int64)
    code = np.zeros(M, np.int64)
    stride = 1
    for a in range(ndim):
        x0m = op.index[ndim - 1 - a].reshape(-1, op.index[ndim - 1 - a].shape[-1])[:, 0].astype(np.int64)
        nb = -(-(nos[a] + off[a]) // tile[a])
        tb = (x0m + off[a]) // tile[a]
        key_bin += tb * stride
        stride *= nb
        org = np.maximum(tb * tile[a] - off[a], 0)
        text = np.minimum((tb + 1) * tile[a] - off[a], nos[a]) - org
        if nb > 1:
            code |= ((x0m - org + w - 1 >= text).astype(np.int64) << a)
    return ((key_bin << ndim) | code) * plan.interpolator.nframes + frame


def test_counting_sort_large_3d_radial():
    """A 3D golden-means radial plan of 2 M samples (500 chunks of the sort, three
    8-bit passes for its 2^19 keys): sorted by key, stable, a permutation."""
    import bench
    import pyfourier_b200 as pf

    N = 160
    coord = bench.golden_means_radial_3d(8000, 256, N)
    plan = pf.plan_nufft(torch.as_tensor(coord), (N, N, N), width=4, oversamp=1.25, device="cuda:0")
    order = _sorted_order(plan)
    M = order.size
    assert np.array_equal(np.sort(order), np.arange(M))
    op = orc.plan_nufft(coord, (N, N, N), width=4, oversamp=1.25)
    key = _bin_keys(plan, op, np.zeros(M, np.int64), 3)
    ks = key[order]
    assert np.all(np.diff(ks) >= 0)
    assert np.all(np.diff(order)[np.diff(ks) == 0] > 0)


@pytest.mark.parametrize("ndim", [2, 3])
def test_counting_sort_is_stable_by_bin_key(ndim):
    """The plan's samples are ordered by the integer bin key
    ((tile << d | edge code) * F + frame) with the reference's grid-index
    arithmetic, and equal keys keep the caller's order (a stable sort): the
    exported order against keys recomputed here from the oracle's tables."""
    import pyfourier_b200 as pf

    rng = np.random.default_rng(70 + ndim)
    N = (40,) * ndim
    F = 3
    lens = [2500, 700, 4100]
    frames = [((rng.random((m, ndim)) - 0.5) * N[0]).astype(np.float32) for m in lens]
    frames[1][:300] *= 0.02  # a crowded bin
    plan = pf.plan_nufft([torch.as_tensor(c) for c in frames], N, width=4, oversamp=1.25, device="cuda:0")
    M = plan.interpolator.total_samples
    order = torch.empty(M, dtype=torch.int32, device="cuda:0")
    _lib().check(_lib().load().pfb_plan_order(plan.interpolator.handle, ctypes.c_void_p(order.data_ptr()),
                                              _stream()))
    order = order.cpu().numpy()
    assert np.array_equal(np.sort(order), np.arange(M))
    # keys from the first taps of the oracle's tables (x-first axes)
    coord = np.concatenate(frames)
    op = orc.plan_nufft(coord[None], N, width=4, oversamp=1.25)
    # a 50-point grid axis: tiles shifted by one point (first tile one narrower, last 3 wide)
    assert plan.interpolator.tile_offset == (1,) * ndim
    key = _bin_keys(plan, op, np.repeat(np.arange(F), lens), ndim)
    ks = key[order]
    assert np.all(np.diff(ks) >= 0)
    same = np.diff(ks) == 0
    assert np.all(np.diff(order)[same] > 0)
    # deterministic: a second plan gives the same order
    plan2 = pf.plan_nufft([torch.as_tensor(c) for c in frames], N, width=4, oversamp=1.25, device="cuda:0")
    order2 = torch.empty(M, dtype=torch.int32, device="cuda:0")
    _lib().check(_lib().load().pfb_plan_order(plan2.interpolator.handle, ctypes.c_void_p(order2.data_ptr()),
                                              _stream()))
    assert np.array_equal(order2.cpu().numpy(), order)
