"""GPU parity at the benchmarked configurations, reduced in size so that the
oracle finishes in seconds, with the benchmark's own trajectory generators.

* 3D golden-means radial (osf 1.25, W 4, 32 coils): the 32-channel register-tile
  spread and the 32-channel interp, on 8^3 tiles of an 80^3 grid and on 8^3 tiles
  of a 90^3 grid shifted by one point (first tile 7, last tile 3 wide: the tile
  fit of the 250^3 benchmark grid, 7 + 30 x 8 + 3);
* Toeplitz Gram with a K = 4 exponential-recovery subspace over 48 rotated
  variable-density spiral frames, 16 coils;
* B0 time-segmented (L = 8) dynamic radial with 12 coils and frames of uneven
  length: one batched (ragged) plan against the oracle frame by frame, and the
  batched graph-captured form against the per-frame calls;
* the differentiable spiral NUFFT (8 coils, osf 2, W 4, "ortho").

Tolerance: rel-L2 <= 1e-5 against the oracle (float summation order differs)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import bench  # noqa: E402  (the benchmark's trajectory and phantom generators)
from oracle import nufft_oracle as orc  # noqa: E402

TOL = 1e-5


def pf():
    import pyfourier_b200

    return pyfourier_b200


def crandn(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return orc.rel_l2(a, b)


@pytest.mark.parametrize("N, nspokes, nread, offset", [(64, 2000, 128, 0), (72, 1500, 144, 1)])
def test_3d_golden_means_radial_32_coils(N, nspokes, nread, offset):
    P = pf()
    rng = np.random.default_rng(N)
    coord = bench.golden_means_radial_3d(nspokes, nread, N)
    B = 32
    oplan = orc.plan_nufft(coord, (N, N, N), width=4, oversamp=1.25)
    gplan = P.plan_nufft(torch.as_tensor(coord), (N, N, N), width=4, oversamp=1.25, device="cuda:0")
    assert gplan.interpolator.tile == (8, 8, 8)
    assert gplan.interpolator.tile_offset == (offset,) * 3
    ph = bench.phantom_3d(torch, N, 20, "cuda:0", seed=1)
    x = (bench.coil_maps_3d(torch, N, B, "cuda:0") * ph[None]).contiguous()
    yg = P.nufft(x, nufft_plan=gplan)
    yr = orc.nufft_fwd(x.cpu().numpy(), oplan)
    assert rel(yg, yr) < TOL
    # the adjoint of the structured (centre-heavy) k-space against the same algorithm
    # in float64: the reference's float32 serial sums drift from it (1e-4 here), the
    # GPU's per-block register sums stay close (about 1e-5) and always closer
    xa = P.nufft_adj(yg, nufft_plan=gplan)
    y0 = yg[:1].reshape(1, -1).cpu().numpy()
    x64 = orc.nufft_adj_f64(y0, oplan)
    x32 = orc.nufft_adj(y0.reshape(1, nspokes, nread), oplan)
    e_gpu, e_orc = rel(xa[:1], x64), rel(x32.reshape(x64.shape), x64)
    assert e_gpu < 2e-5 and e_gpu < e_orc, (e_gpu, e_orc)
    yk = crandn(rng, B, nspokes, nread)
    xg = P.nufft_adj(torch.as_tensor(yk).cuda(), nufft_plan=gplan)
    assert rel(xg, orc.nufft_adj(yk, oplan)) < TOL
    # no kernel of these applies gave up a bounded wait (the TMA column passes)
    gplan.interpolator.check()


def test_toeplitz_gram_subspace_spiral_48_frames_16_coils():
    P = pf()
    N, F, K, B = 64, 48, 4, 16
    coord = np.stack([bench.vd_spiral(4, 256, N, rot=f * np.pi * (3 - 5 ** 0.5)) for f in range(F)])
    basis = bench.exp_recovery_basis(K, nt=F)
    og = orc.plan_spgram(coord, (N, N), basis=basis)
    gg = P.plan_spgram(torch.as_tensor(coord), (N, N), basis=torch.as_tensor(basis), device="cuda:0")
    assert gg.islowrank and tuple(gg.value.shape) == tuple(og.value.shape)
    assert rel(gg.value, og.value) < TOL
    x = crandn(np.random.default_rng(3), B, K, N, N)
    assert rel(P.sparse_gram(torch.as_tensor(x).cuda(), gg), orc.sparse_gram(x, og)) < TOL


def test_b0_dynamic_radial_ragged_frames_batched_and_graph():
    P = pf()
    N, B, F, Lseg, nread = 48, 12, 12, 8, 64
    rng = np.random.default_rng(0)
    nsp = rng.integers(1, 9, F)
    starts = np.concatenate([[0], np.cumsum(nsp)[:-1]])
    frames = [bench.radial_2d(int(n), nread, N, start=int(s0)) for n, s0 in zip(nsp, starts)]
    b0 = bench.smooth_field(N)
    dt = 5e-3 / nread
    kw = dict(width=4, oversamp=1.25, zmap=b0, L=Lseg, nbins=40, dt=dt)
    bplan = P.plan_nufft([torch.as_tensor(c) for c in frames], (N, N), device="cuda:0",
                         **{**kw, "zmap": torch.as_tensor(b0)})
    x = crandn(rng, B, F, N, N)
    xt = torch.as_tensor(x).cuda()
    yb = P.nufft(xt, nufft_plan=bplan)
    offs = bplan.interpolator.frame_offsets
    yk = crandn(rng, B, int(offs[-1]))
    xb = P.nufft_adj(torch.as_tensor(yk).cuda(), nufft_plan=bplan)
    for f, c in enumerate(frames):
        op = orc.plan_nufft(c, (N, N), **kw)
        yr = orc.nufft_fwd(x[:, f], op).reshape(B, -1)
        assert rel(yb[:, offs[f]:offs[f + 1]], yr) < TOL, f
        xr = orc.nufft_adj(yk[:, offs[f]:offs[f + 1]].reshape(B, *c.shape[:-1]), op)
        assert rel(xb[:, f], xr) < TOL, f
    # the batched form captured in a CUDA graph gives the same result
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            P.nufft_adj(P.nufft(xt, nufft_plan=bplan), nufft_plan=bplan)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = P.nufft_adj(P.nufft(xt, nufft_plan=bplan), nufft_plan=bplan)
    g.replay()
    ref = P.nufft_adj(yb, nufft_plan=bplan)
    torch.cuda.synchronize()
    assert rel(out, ref.cpu().numpy()) < 1e-6


def test_differentiable_spiral_8_coils_ortho():
    P = pf()
    N, B, nimg = 64, 8, 4
    coord = bench.vd_spiral(16, 512, N)
    rng = np.random.default_rng(5)
    oplan = orc.plan_nufft(coord, (N, N), width=4, oversamp=2.0)
    gplan = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    x = crandn(rng, nimg, B, N, N)
    yg = P.nufft(torch.as_tensor(x).cuda(), nufft_plan=gplan, norm="ortho")
    yr = orc.nufft_fwd(x, oplan, norm="ortho")
    assert rel(yg, yr) < TOL
    xg = P.nufft_adj(yg, nufft_plan=gplan, norm="ortho")
    assert rel(xg, orc.nufft_adj(yr, oplan, norm="ortho")) < TOL


@pytest.mark.parametrize("B", [1, 8, 16])
def test_3d_w6_few_channel_spread_is_deterministic(B):
    """Width 6 (8-tap register blocks) with 8- and 16-channel groups on a crowded 3D
    radial plan: full batches whose last staging round is partial.  Two applies give
    the same image, and it matches the reference's adjoint in float64."""
    P = pf()
    N = 48
    coord = bench.golden_means_radial_3d(2000, 96, N)
    gplan = P.plan_nufft(torch.as_tensor(coord), (N, N, N), width=6, oversamp=1.5, device="cuda:0")
    oplan = orc.plan_nufft(coord, (N, N, N), width=6, oversamp=1.5)
    yk = crandn(np.random.default_rng(B), B, 2000, 96)
    yt = torch.as_tensor(yk).cuda()
    x1 = P.nufft_adj(yt, nufft_plan=gplan)
    x2 = P.nufft_adj(yt, nufft_plan=gplan)
    assert rel(x2, x1.cpu().numpy()) < 1e-6
    x64 = orc.nufft_adj_f64(yk[:1].reshape(1, -1), oplan)
    assert rel(x1[:1], x64) < 2e-5
