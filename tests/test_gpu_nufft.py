"""GPU parity of the public operators (nufft, nufft_adj, B0, subspace, weights)
against the CPU oracle on identical seeded inputs; edge cases; error paths."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402

TOL = 1e-5  # rel-L2 vs the oracle (float32 atomics: order differs, so a tolerance)


def pf():
    import pyfourier_b200

    return pyfourier_b200


def crandn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def radial(nspokes, nread, N, seed=0, rot=0.0):
    ga = np.pi / ((1 + 5 ** 0.5) / 2)
    ang = np.arange(nspokes) * ga + rot
    kr = (np.arange(nread) - nread // 2) / nread * N
    return np.stack([np.cos(ang)[:, None] * kr, np.sin(ang)[:, None] * kr], -1).astype(np.float32)


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return orc.rel_l2(a, b)


def check_pair(coord, N, x, y, width=4, oversamp=2.0, norm=None, basis=None, weight=None, **plan_kw):
    """nufft and nufft_adj on GPU vs the oracle (same plan parameters)."""
    P = pf()
    oplan = orc.plan_nufft(coord, N, width=width, oversamp=oversamp, **plan_kw)
    gplan = P.plan_nufft(torch.as_tensor(coord), N, width=width, oversamp=oversamp, device="cuda:0", **plan_kw)
    xr = orc.nufft_fwd(x, oplan, basis=basis, weight=weight, norm=norm)
    xg = P.nufft(torch.as_tensor(x).cuda(), nufft_plan=gplan, basis=basis, weight=weight, norm=norm,
                 device="cuda:0")
    assert xg.shape == xr.shape
    e1 = rel(xg, xr)
    yr = orc.nufft_adj(y, oplan, basis=basis, weight=weight, norm=norm)
    yg = P.nufft_adj(torch.as_tensor(y).cuda(), nufft_plan=gplan, basis=basis, weight=weight, norm=norm,
                     device="cuda:0")
    assert yg.shape == yr.shape
    e2 = rel(yg, yr)
    assert e1 < TOL and e2 < TOL, (e1, e2)
    return gplan


def test_cfg1_radial_2d_full_size():
    rng = np.random.default_rng(0)
    N = 128
    coord = radial(201, 256, N)
    x = crandn(rng, 8, N, N)
    y = crandn(rng, 8, 201, 256)
    check_pair(coord, (N, N), x, y, width=4, oversamp=2.0)


@pytest.mark.parametrize("norm", [None, "ortho"])
def test_2d_small_norms(norm):
    rng = np.random.default_rng(1)
    N = 48
    coord = radial(37, 96, N)
    check_pair(coord, (N, N), crandn(rng, 3, N, N), crandn(rng, 3, 37, 96), norm=norm, oversamp=1.25)


@pytest.mark.parametrize("w", [2, 3, 5, 6, 7, 8])
def test_widths(w):
    rng = np.random.default_rng(2)
    N = 40
    coord = radial(21, 80, N)
    check_pair(coord, (N, N), crandn(rng, 2, N, N), crandn(rng, 2, 21, 80), width=w, oversamp=2.0)


def test_odd_sizes_and_anisotropic():
    rng = np.random.default_rng(3)
    N = (45, 37)
    coord = ((rng.random((30, 50, 2)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    check_pair(coord, N, crandn(rng, 2, *N), crandn(rng, 2, 30, 50), width=(5, 3), oversamp=(1.5, 2.0))


@pytest.mark.parametrize("N", [(128, 200), (200, 192), (96, 128, 200)])
def test_anisotropic_grids_with_fused_transform_lengths(N):
    """Grids whose axes have different lengths of the fused transform's compile-time
    plans (osf 1.25: 160 x 250, 250 x 240, 120 x 160 x 250): each axis reads its own
    twiddles, the two-stage 240 / 250 plans included."""
    rng = np.random.default_rng(11)
    d = len(N)
    coord = ((rng.random((20, 600, d)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    check_pair(coord, N, crandn(rng, 2, *N), crandn(rng, 2, 20, 600), width=4, oversamp=1.25)


def test_edges_and_out_of_range_wrap():
    """Samples at exactly -N/2 and +N/2 - eps, and beyond +-N/2 (reference wraps mod n_os)."""
    rng = np.random.default_rng(4)
    N = 32
    c = np.array([[-16, -16], [15.999, 15.999], [-16, 15.5], [16, 0], [20.25, -19.5], [0, 0], [0.5, -0.5],
                  [7.0, 7.0]], np.float32)
    coord = np.concatenate([c, ((rng.random((56, 2)) - 0.5) * N).astype(np.float32)])[None]
    check_pair(coord, (N, N), crandn(rng, 2, N, N), crandn(rng, 2, 1, 64), width=4, oversamp=1.25)


def test_all_samples_in_one_tile_and_chunking():
    """A crowded bin (k-space centre hot spot) split into several work items."""
    rng = np.random.default_rng(5)
    N = 64
    # every first tap x0 = ceil(2c + 62) in [56, 63]: one 32-wide tile on both axes
    coord = ((rng.random((1, 4000, 2)) - 1.0) * 3.0 + 0.49).astype(np.float32)
    gplan = check_pair(coord, (N, N), crandn(rng, 3, N, N), crandn(rng, 3, 1, 4000), oversamp=2.0)
    assert gplan.interpolator.max_bin >= 1000  # 4000 samples in one tile, split over <= 4 edge codes


def test_crowded_3d_tiles_with_many_channels():
    """3D, more than 16 channels (register-tile spread): a hot spot of 6000
    samples split into several work items combined with atomics, items of
    several staged batches, and tiles at the periodic edge."""
    rng = np.random.default_rng(15)
    N = 24
    hot = ((rng.random((6000, 3)) - 0.5) * 2.0).astype(np.float32)
    edge = ((rng.random((500, 3)) - 0.5) * N).astype(np.float32)
    edge[:100] = -N / 2  # first taps wrap across the periodic boundary
    coord = np.concatenate([hot, edge])[None]
    check_pair(coord, (N, N, N), crandn(rng, 20, N, N, N), crandn(rng, 20, 1, 6500), width=4, oversamp=1.25)
    check_pair(coord, (N, N, N), crandn(rng, 33, N, N, N), crandn(rng, 33, 1, 6500), width=6, oversamp=2.0)
    # exactly 32 and 64 channels (one and two full 32-channel groups) on split crowded tiles
    check_pair(coord, (N, N, N), crandn(rng, 32, N, N, N), crandn(rng, 32, 1, 6500), width=4, oversamp=1.25)
    check_pair(coord, (N, N, N), crandn(rng, 64, N, N, N), crandn(rng, 64, 1, 6500), width=4, oversamp=1.25)


@pytest.mark.parametrize("nch", [3, 8, 12, 16])
def test_3d_channel_groups(nch):
    """3D spreads take register tiles in channel groups of 8 (<= 8 channels), 16 (9-16)
    or 32 per lane group; every group size against the oracle, with crowded tiles."""
    rng = np.random.default_rng(40 + nch)
    N = 20
    coord = ((rng.random((1, 30, 90, 3)) - 0.5) * N).astype(np.float32)
    coord[0, :3] *= 0.05  # crowd the centre tiles
    check_pair(coord, (N, N, N), crandn(rng, nch, N, N, N), crandn(rng, nch, 30, 90), width=4, oversamp=1.25)


@pytest.mark.parametrize("N, nch", [(40, 36), (8, 33)])
def test_2d_register_tiles(N, nch):
    """2D spreads of more than 16 channels take 16 x 16 register tiles (32 channels per
    lane group, a second group for the rest); N = 8 at osf 2 is one tile whose taps wrap."""
    rng = np.random.default_rng(60 + N)
    coord = ((rng.random((1, 24, 64, 2)) - 0.5) * N).astype(np.float32)
    coord[0, :4] *= 0.05  # crowd the centre tiles
    check_pair(coord, (N, N), crandn(rng, nch, N, N), crandn(rng, nch, 24, 64), width=4, oversamp=2.0)


@pytest.mark.parametrize("N, width, oversamp", [((40, 40), 4, 2.0), ((36, 44), (3, 2), 2.0), ((20, 20, 20), 3, 2.0),
                                                ((16, 20, 24), (2, 4, 3), 1.25)])
def test_interp_x_rows_32_channels(N, width, oversamp):
    """Exactly 32 channels in 2D / 3D boxes up to 4 taps wide: the interp's x-row form with
    a compile-time channel count (fixed-offset taps; samples whose x taps straddle the
    fftshift seam take computed pointers), widths below 4 padding rows and columns."""
    rng = np.random.default_rng(70 + len(N))
    d = len(N)
    coord = ((rng.random((1, 40, 60, d)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    coord[0, :5] *= 0.05  # crowd the centre, where the x taps straddle the seam
    check_pair(coord, N, crandn(rng, 32, *N), crandn(rng, 32, 40, 60), width=width, oversamp=oversamp)


def test_multiframe_and_weights():
    rng = np.random.default_rng(6)
    N, F = 40, 3
    coord = np.stack([radial(10, 64, N, rot=0.3 * f) for f in range(F)])
    x = crandn(rng, 2, F, N, N)
    y = crandn(rng, 2, F, 10, 64)
    wps = rng.random((F, 10, 64)).astype(np.float32)
    check_pair(coord, (N, N), x, y, weight=wps)
    wfull = rng.random((2, F, 10, 64)).astype(np.float32)  # varies over the batch: torch multiply
    check_pair(coord, (N, N), x, y, weight=wfull)


def test_subspace_basis():
    rng = np.random.default_rng(7)
    N, F, K = 32, 6, 3
    coord = np.stack([radial(8, 48, N, rot=0.2 * f) for f in range(F)])
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    check_pair(coord, (N, N), crandn(rng, 2, K, N, N), crandn(rng, 2, F, 8, 48), basis=basis)


def test_3d():
    rng = np.random.default_rng(8)
    N = (20, 24, 22)
    coord = ((rng.random((40, 60, 3)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    check_pair(coord, N, crandn(rng, 2, *N), crandn(rng, 2, 40, 60), width=4, oversamp=1.25)


def test_1d():
    rng = np.random.default_rng(9)
    N = 100
    coord = ((rng.random((5, 70, 1)) - 0.5) * N).astype(np.float32)
    check_pair(coord, (N,), crandn(rng, 3, N), crandn(rng, 3, 5, 70), width=4, oversamp=2.0)


def test_stack_of_stars_cartesian_axis():
    """z Cartesian (integer positions, width 1, osf 1) as in _nufft/_plan.py:139-146."""
    rng = np.random.default_rng(10)
    N = (8, 32, 32)
    r = radial(12, 40, 32)
    kz = np.arange(-4, 4, dtype=np.float32)
    coord = np.concatenate([np.broadcast_to(r[None], (8, 12, 40, 2)),
                            np.broadcast_to(kz[:, None, None, None], (8, 12, 40, 1))], -1)
    coord = np.ascontiguousarray(coord.reshape(96, 40, 3))
    gplan = check_pair(coord, N, crandn(rng, 2, *N), crandn(rng, 2, 96, 40), width=4, oversamp=2.0)
    assert gplan.width[0] == 1 and gplan.os_shape[0] == 8


def test_b0_segments_and_chunks():
    rng = np.random.default_rng(11)
    N, nv, ns = 32, 10, 64
    coord = radial(nv, ns, N)
    yy, xx = np.mgrid[:N, :N] / N - 0.5
    b0 = 150 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 80
    dt = 5e-3 / ns
    for Lb in (None, 4):
        check_pair(coord, (N, N), crandn(rng, 3, N, N), crandn(rng, 3, nv, ns), zmap=b0, L=6, nbins=40,
                   dt=dt, L_batch_size=Lb)


def test_adjointness_ortho_gpu():
    P = pf()
    rng = np.random.default_rng(12)
    N = 64
    coord = radial(50, 128, N)
    plan = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    x = torch.as_tensor(crandn(rng, 4, N, N)).cuda()
    y = torch.as_tensor(crandn(rng, 4, 50, 128)).cuda()
    lhs = torch.vdot(y.flatten(), P.nufft(x, nufft_plan=plan, norm="ortho").flatten())
    rhs = torch.vdot(P.nufft_adj(y, nufft_plan=plan, norm="ortho").flatten(), x.flatten())
    assert abs((lhs - rhs) / lhs).item() < 1e-5


def test_ragged_frames_match_per_frame_calls():
    """A plan over frames of uneven length equals separate per-frame plans."""
    P = pf()
    rng = np.random.default_rng(13)
    N = 32
    frames = [radial(n, 64, N, rot=0.1 * i) for i, n in enumerate([5, 1, 17, 9])]
    frames.append(np.zeros((0, 64, 2), np.float32))  # an empty frame
    plan = P.plan_nufft([torch.as_tensor(f) for f in frames], (N, N), width=4, oversamp=2.0, device="cuda:0")
    F = len(frames)
    x = torch.as_tensor(crandn(rng, 2, F, N, N)).cuda()
    y = P.nufft(x, nufft_plan=plan)
    offs = plan.interpolator.frame_offsets
    tot = offs[-1]
    assert y.shape == (2, tot)
    yk = torch.as_tensor(crandn(rng, 2, tot)).cuda()
    xa = P.nufft_adj(yk, nufft_plan=plan)
    for f, c in enumerate(frames):
        if c.shape[0] == 0:
            assert torch.count_nonzero(xa[:, f]) == 0
            continue
        pl = P.plan_nufft(torch.as_tensor(c), (N, N), width=4, oversamp=2.0, device="cuda:0")
        yf = P.nufft(x[:, f], nufft_plan=pl)
        assert rel(y[:, offs[f]:offs[f + 1]], yf.reshape(2, -1).cpu().numpy()) < 1e-6
        xf = P.nufft_adj(yk[:, offs[f]:offs[f + 1]].reshape(2, *c.shape[:-1]), nufft_plan=pl)
        assert rel(xa[:, f], xf.cpu().numpy()) < 1e-6


def test_single_sample_and_real_input_dtype():
    P = pf()
    N = 16
    coord = np.array([[[1.25, -3.5]]], np.float32)
    x = np.random.default_rng(14).standard_normal((N, N)).astype(np.float32)
    plan = orc.plan_nufft(coord, (N, N), width=4, oversamp=2.0)
    ref = orc.nufft_fwd(x.astype(np.complex64), plan).real
    got = P.nufft(torch.as_tensor(x), torch.as_tensor(coord), (N, N), width=4, oversamp=2.0)
    assert got.dtype == torch.float32 and got.device.type == "cpu"
    assert rel(got, ref) < 1e-5
    got_np = P.nufft(x, coord, (N, N), width=4, oversamp=2.0)
    assert isinstance(got_np, np.ndarray)


def test_errors_raise_value_error():
    P = pf()
    coord = radial(4, 16, 16)
    plan = P.plan_nufft(torch.as_tensor(coord), (16, 16), device="cuda:0")
    with pytest.raises(ValueError):
        P.nufft(torch.zeros(2, 15, 16, dtype=torch.complex64), nufft_plan=plan)
    with pytest.raises(ValueError):
        P.nufft_adj(torch.zeros(2, 4, 15, dtype=torch.complex64), nufft_plan=plan)
    with pytest.raises(ValueError):
        P.plan_nufft(torch.full((1, 4, 2), float("nan")), (16, 16), device="cuda:0")
    with pytest.raises(ValueError):
        P.nufft(torch.zeros(16, 16, dtype=torch.complex64), nufft_plan=plan, norm="bogus")
    with pytest.raises(ValueError):
        P.plan_nufft(torch.as_tensor(coord), (16, 16), width=9, device="cuda:0")


def test_cuda_graph_capture():
    """An apply contains no host sync or allocation inside the library: capturable."""
    P = pf()
    rng = np.random.default_rng(15)
    N = 64
    coord = radial(40, 128, N)
    plan = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    x = torch.as_tensor(crandn(rng, 4, N, N)).cuda()
    ref = P.nufft_adj(P.nufft(x, nufft_plan=plan), nufft_plan=plan)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            P.nufft_adj(P.nufft(x, nufft_plan=plan), nufft_plan=plan)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = P.nufft_adj(P.nufft(x, nufft_plan=plan), nufft_plan=plan)
    g.replay()
    torch.cuda.synchronize()
    assert rel(out, ref.cpu().numpy()) < 1e-6


def test_autotune_keeps_results_and_caches(tmp_path, monkeypatch):
    """Tuning changes the tile / chunk, never the result; the choice is cached."""
    import json

    P = pf()
    monkeypatch.setenv("PYFOURIER_B200_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(16)
    N = 64
    coord = radial(40, 128, N)
    x = crandn(rng, 3, N, N)
    y = crandn(rng, 3, 40, 128)
    oplan = orc.plan_nufft(coord, (N, N), width=4, oversamp=2.0)
    plan = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    res = P.autotune(plan, batch=3, tiles=[(16, 16), (32, 32)], chunks=[256, 4096], iters=1)
    assert res["cached"] is False and tuple(res["tile"]) in {(16, 16), (32, 32)}
    assert rel(P.nufft(torch.as_tensor(x).cuda(), nufft_plan=plan), orc.nufft_fwd(x, oplan)) < TOL
    assert rel(P.nufft_adj(torch.as_tensor(y).cuda(), nufft_plan=plan), orc.nufft_adj(y, oplan)) < TOL
    cache = json.loads((tmp_path / "tune.json").read_text())
    assert len(cache) == 1
    plan2 = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    res2 = P.autotune(plan2, batch=3)
    assert res2["cached"] is True and list(res2["tile"]) == list(res["tile"])
    assert rel(P.nufft(torch.as_tensor(x).cuda(), nufft_plan=plan2), orc.nufft_fwd(x, oplan)) < TOL


def test_concurrent_applies_of_one_plan_from_two_threads():
    """Two host threads apply one plan (and one Gram) on their own streams at the
    same time: the shared cuFFT handle is used under the plan's lock from
    set-stream to exec, so each thread's transform runs with its own stream and
    work area and both results equal the sequential ones."""
    import threading

    P = pf()
    rng = np.random.default_rng(30)
    N = 96
    coord = ((rng.random((40, 90, 1)) - 0.5) * N).astype(np.float32)  # 1D: library FFT path
    plan = P.plan_nufft(torch.as_tensor(coord), (N,), width=4, oversamp=2.0, device="cuda:0")
    gcoord = radial(30, 64, 32)
    gm = P.plan_spgram(torch.as_tensor(gcoord), (32, 32), device="cuda:0")
    ys = [torch.as_tensor(crandn(rng, 6, 40, 90)).cuda() for _ in range(2)]
    xs = [torch.as_tensor(crandn(rng, 5, 32, 32)).cuda() for _ in range(2)]
    ref_a = [P.nufft_adj(y, nufft_plan=plan) for y in ys]
    ref_g = [P.sparse_gram(x, gm) for x in xs]
    torch.cuda.synchronize()
    out = [[None] * 2 for _ in range(2)]
    errs = []

    def work(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                for _ in range(20):
                    a = P.nufft_adj(ys[i], nufft_plan=plan)
                    g = P.sparse_gram(xs[i], gm)
                s.synchronize()
            out[i] = [a, g]
        except Exception as e:  # pragma: no cover
            errs.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for i in range(2):
        assert rel(out[i][0], ref_a[i].cpu().numpy()) < 1e-6
        assert rel(out[i][1], ref_g[i].cpu().numpy()) < 1e-6
