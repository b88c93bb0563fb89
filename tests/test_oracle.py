"""CPU tests of the oracle: pinned against the reference's golden vectors, then
checked against an FP64 direct NUDFT and for adjointness.  No GPU needed."""

import numpy as np
import pytest

from oracle import nufft_oracle as orc


def test_kaiser_bessel_matches_reference(golden):
    xs, betas, ref = golden["kb_x"], golden["kb_beta"], golden["kb_val"]
    got = np.array([[orc.kaiser_bessel(x, b) for x in xs] for b in betas])
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


def test_kernel_scaling_matches_reference(golden):
    for w, b, v in zip(golden["scal_width"], golden["scal_beta"], golden["scal_value"]):
        nd = int((w > 0).sum())
        got = orc.kernel_scaling(b[:nd], w[:nd])
        assert got == pytest.approx(v, rel=1e-13)


@pytest.mark.parametrize("w", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("osf", [1.25, 2.0])
def test_tables_match_reference(golden, w, osf):
    c = golden["tab_coord"]
    N = int(golden["tab_N"])
    beta = orc.beta_f32((w,), (osf,))
    c_os = orc.scale_coord(c[None, :, None], (N,), (osf,))
    n_os = orc.oversamp_shape((N,), (osf,))
    idx, val = orc.prepare_tables(c_os, n_os, (w,), beta)
    tag = f"tab_w{w}_os{osf}"
    np.testing.assert_array_equal(idx[0], golden[tag + "_index"])
    np.testing.assert_allclose(val[0], golden[tag + "_value"], rtol=2e-7, atol=0)


@pytest.mark.parametrize("d", [1, 2, 3])
def test_spread_interp_match_reference(golden, d):
    p = f"k{d}d_"
    N, osf, w, beta, os_ = (golden[p + k] for k in ("N", "osf", "width", "beta", "os"))
    coord = golden[p + "coord"]
    c_os = orc.scale_coord(coord, N[::-1], osf[::-1])
    idx, val = orc.prepare_tables(c_os, os_, w, beta)
    for a in range(d):
        np.testing.assert_array_equal(idx[a], golden[p + f"index{a}"])
        np.testing.assert_allclose(val[a], golden[p + f"value{a}"], rtol=2e-7)
    F = coord.shape[0]
    sp = orc.spread(golden[p + "noncart"], idx, val, tuple(os_))
    assert orc.rel_l2(sp, golden[p + "spread"]) < 1e-6
    it = orc.interp(golden[p + "grid_in"], idx, val, tuple(os_), F)
    assert orc.rel_l2(it, golden[p + "interp"]) < 1e-6
    basis = golden[p + "basis"]
    sps = orc.spread(golden[p + "noncart"], idx, val, tuple(os_), np.ascontiguousarray(basis.conj().T))
    assert orc.rel_l2(sps, golden[p + "spread_sub"]) < 1e-6
    its = orc.interp(golden[p + "grid_in_sub"], idx, val, tuple(os_), F, basis)
    assert orc.rel_l2(its, golden[p + "interp_sub"]) < 1e-6


def _radial(nspokes, nread, N, seed=0):
    ga = np.pi / ((1 + 5 ** 0.5) / 2)
    ang = np.arange(nspokes) * ga
    kr = (np.arange(nread) - nread // 2) / nread * N
    c = np.stack([np.cos(ang)[:, None] * kr, np.sin(ang)[:, None] * kr], -1)
    return c.astype(np.float32)


@pytest.mark.parametrize("osf,w,tol", [(2.0, 4, 2e-3), (1.25, 4, 2e-2), (2.0, 6, 1e-4)])
def test_oracle_nufft_vs_nudft(osf, w, tol):
    rng = np.random.default_rng(1)
    N = 32
    coord = _radial(24, 48, N)
    x = (rng.standard_normal((2, N, N)) + 1j * rng.standard_normal((2, N, N))).astype(np.complex64)
    plan = orc.plan_nufft(coord, (N, N), width=w, oversamp=osf)
    y = orc.nufft_fwd(x, plan)
    y_ref = orc.nudft_fwd(x, coord.reshape(-1, 2), (N, N)).reshape(y.shape)
    assert orc.rel_l2(y, y_ref) < tol
    G = float(np.prod(plan.os_shape))
    xa = orc.nufft_adj(y_ref.astype(np.complex64), plan) * G
    xa_ref = orc.nudft_adj(y_ref.reshape(2, -1), coord.reshape(-1, 2), (N, N))
    assert orc.rel_l2(xa, xa_ref) < tol


def test_oracle_adjointness_ortho():
    rng = np.random.default_rng(2)
    N = 24
    coord = _radial(16, 40, N)
    plan = orc.plan_nufft(coord, (N, N), width=4, oversamp=2.0)
    x = (rng.standard_normal((3, N, N)) + 1j * rng.standard_normal((3, N, N))).astype(np.complex64)
    y = (rng.standard_normal((3, 16, 40)) + 1j * rng.standard_normal((3, 16, 40))).astype(np.complex64)
    lhs = np.vdot(y, orc.nufft_fwd(x, plan, norm="ortho"))
    rhs = np.vdot(orc.nufft_adj(y, plan, norm="ortho"), x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_oracle_3d_vs_nudft():
    rng = np.random.default_rng(3)
    N = (10, 12, 14)
    M = 300
    coord = ((rng.random((M, 3)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    plan = orc.plan_nufft(coord, N, width=6, oversamp=2.0)
    y = orc.nufft_fwd(x, plan)
    y_ref = orc.nudft_fwd(x, coord, N)
    assert orc.rel_l2(y, y_ref) < 1e-4


def test_oracle_gram_exact_matches_ahwa():
    rng = np.random.default_rng(4)
    N = 20
    coord = _radial(12, 40, N)
    wgt = rng.random(coord.shape[:-1]).astype(np.float32)
    gm = orc.plan_spgram(coord, (N, N), weight=wgt, normalize=None)
    x = (rng.standard_normal((2, N, N)) + 1j * rng.standard_normal((2, N, N))).astype(np.complex64)
    g = orc.sparse_gram(x, gm)
    ref = orc.nudft_adj(wgt.ravel() * orc.nudft_fwd(x, coord.reshape(-1, 2), (N, N)),
                        coord.reshape(-1, 2), (N, N))
    assert orc.rel_l2(g, ref) < 1e-3


def test_oracle_gram_subspace_exact():
    rng = np.random.default_rng(5)
    N, F, K = 16, 6, 3
    coord = np.stack([_radial(6, 32, N) @ np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]],
                                                   np.float32) for a in np.linspace(0, 1, F)])
    basis = np.linalg.qr(rng.standard_normal((F, K)) + 1j * rng.standard_normal((F, K)))[0].astype(np.complex64)
    gm = orc.plan_spgram(coord, (N, N), basis=basis, normalize=None)
    x = (rng.standard_normal((2, K, N, N)) + 1j * rng.standard_normal((2, K, N, N))).astype(np.complex64)
    g = orc.sparse_gram(x, gm)
    # A: x_k -> y_f = sum_k basis[f,k] NUDFT_f(x_k); A^H: y -> sum_f conj(basis[f,k]) NUDFT_f^H y_f
    ref = np.zeros_like(g, dtype=np.complex128)
    for f in range(F):
        cf = coord[f].reshape(-1, 2)
        yf = sum(basis[f, k] * orc.nudft_fwd(x[:, k], cf, (N, N)) for k in range(K))
        af = orc.nudft_adj(yf, cf, (N, N))
        for k in range(K):
            ref[:, k] += np.conj(basis[f, k]) * af
    assert orc.rel_l2(g, ref) < 1e-3


def test_oracle_b0_segmentation_vs_exact():
    rng = np.random.default_rng(6)
    N, nv, ns = 24, 12, 64
    coord = _radial(nv, ns, N)
    yy, xx = np.mgrid[:N, :N] / N - 0.5
    b0 = (120 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 60 * np.exp(-((xx + 0.2) ** 2 + (yy - 0.2) ** 2) / 0.02))
    dt = 5e-3 / ns
    t = dt * np.arange(ns)
    plan = orc.plan_nufft(coord, (N, N), width=6, oversamp=2.0, zmap=b0, L=8, nbins=40, dt=dt)
    x = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    y = orc.nufft_fwd(x, plan)
    # exact: y(m) = sum_r x(r) exp(-2 pi i b0(r) t(m)) exp(-2 pi i k.r / N)
    r = orc.pixel_grid((N, N))
    cm = coord.reshape(-1, 2).astype(np.float64)
    tm = np.tile(t, nv)
    E = np.exp(-2j * np.pi * (cm / N) @ r.T) * np.exp(-2j * np.pi * tm[:, None] * b0.ravel()[None, :])
    y_ref = (E @ x.ravel().astype(np.complex128)).reshape(nv, ns)
    assert orc.rel_l2(y, y_ref) < 2e-3


def test_oracle_gram_with_field_map_vs_exact():
    """Toeplitz Gram with B0 segments approximates A^H W A of the exact
    off-resonance model (time segmentation error only)."""
    rng = np.random.default_rng(7)
    N, nv, ns = 24, 16, 64
    coord = _radial(nv, ns, N)
    yy, xx = np.mgrid[:N, :N] / N - 0.5
    b0 = 100 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 50
    dt = 5e-3 / ns
    t = dt * np.arange(ns)
    gm = orc.plan_spgram(coord, (N, N), normalize=None, zmap=b0, L=8, nbins=40, dt=dt)
    assert gm.value.shape[0] == 8 and gm.zmap_s_kernel.shape == (8, N, N)
    x = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    g = orc.sparse_gram(x, gm)
    r = orc.pixel_grid((N, N))
    cm = coord.reshape(-1, 2).astype(np.float64)
    tm = np.tile(t, nv)
    E = np.exp(-2j * np.pi * (cm / N) @ r.T) * np.exp(-2j * np.pi * tm[:, None] * b0.ravel()[None, :])
    ref = (E.conj().T @ (E @ x.ravel().astype(np.complex128))).reshape(N, N)
    assert orc.rel_l2(g, ref) < 2e-2


def test_oracle_pipe_menon_weights_grow_with_radius():
    """Pipe-Menon on a radial trajectory: the weights follow the 1/density of the
    spokes, growing with |k| (averaged over spokes, outer ring vs inner ring)."""
    N, ns = 32, 64
    coord = _radial(48, ns, N)
    w = orc.pipe_menon_dcf(coord, (N, N), niter=15)
    assert w.shape == coord.shape[:-1] and w.dtype == np.float32
    assert np.all(np.isfinite(w)) and np.all(w > 0)
    kr = np.abs(np.arange(ns) - ns // 2)
    inner = w[:, (kr >= 2) & (kr < 8)].mean()
    outer = w[:, (kr >= 20) & (kr < 28)].mean()
    assert outer > 2.0 * inner


def test_oracle_sparse_fft_is_the_width_one_nufft():
    """The sparse FFT restatement (centred FFT + gather / scatter-add + centred IFFT)
    equals the NUFFT restatement on integer coordinates (width 1, no oversampling),
    with frames, duplicates and a subspace basis."""
    rng = np.random.default_rng(11)
    N = (12, 16)
    F, K = 3, 2
    idx = np.stack([rng.integers(0, N[1], (F, 5, 7)), rng.integers(0, N[0], (F, 5, 7))], -1).astype(np.float32)
    idx[0, 0, :2] = idx[0, 0, 2]  # duplicates add in the adjoint
    basis = (rng.standard_normal((F, K)) + 1j * rng.standard_normal((F, K))).astype(np.complex64)
    coord = idx - np.array([N[1] // 2, N[0] // 2], np.float32)
    plan = orc.plan_nufft(coord, N, width=2, oversamp=1.0)
    assert plan.width == (1, 1) and plan.os_shape == N
    for b in (None, basis):
        C = K if b is not None else F
        x = (rng.standard_normal((2, C, *N)) + 1j * rng.standard_normal((2, C, *N))).astype(np.complex64)
        y = (rng.standard_normal((2, F, 5, 7)) + 1j * rng.standard_normal((2, F, 5, 7))).astype(np.complex64)
        for norm in (None, "ortho"):
            a = orc.sparse_fftn(x, idx, N, basis=b, norm=norm)
            r = orc.nufft_fwd(x, plan, basis=b, norm=norm).reshape(a.shape)
            assert orc.rel_l2(a, r) < 1e-6
            a = orc.sparse_ifftn(y, idx, N, basis=b, norm=norm)
            r = orc.nufft_adj(y, plan, basis=b, norm=norm).reshape(a.shape)
            assert orc.rel_l2(a, r) < 1e-6


def _line_masks(rng, F, N, nsel):
    """Cartesian phase-encode masks: per frame ``nsel`` random ky lines, fully
    sampled along x.  Returns the centred masks (F, ny, nx) and the sampled
    grid indexes (F, nsel, nx, 2), axes (x, y)."""
    ny, nx = N
    lines = np.stack([np.sort(rng.choice(ny, nsel, replace=False)) for _ in range(F)])
    mask = np.zeros((F, ny, nx), np.float32)
    for f in range(F):
        mask[f, lines[f]] = 1
    xx = np.broadcast_to(np.arange(nx), (F, nsel, nx))
    yy = np.broadcast_to(lines[:, :, None], (F, nsel, nx))
    return mask, np.stack([xx, yy], -1).astype(np.float32)


def test_oracle_cartesian_gram_is_the_sparse_fft_normal_operator():
    """Dense Gram restatement == sparse_ifftn(sparse_fftn(x)) on the mask's points,
    per frame and with a subspace basis, for both norms."""
    rng = np.random.default_rng(12)
    N, F, K = (16, 20), 4, 2
    mask, idx = _line_masks(rng, F, N, 6)
    basis = np.linalg.qr(rng.standard_normal((F, K)) + 1j * rng.standard_normal((F, K)))[0].astype(np.complex64)
    for b in (None, basis):
        C = K if b is not None else F
        gm = orc.plan_gram(mask, N, basis=b)
        x = (rng.standard_normal((2, C, *N)) + 1j * rng.standard_normal((2, C, *N))).astype(np.complex64)
        for norm in (None, "ortho"):
            ref = orc.sparse_ifftn(orc.sparse_fftn(x, idx, N, basis=b, norm=norm), idx, N, basis=b, norm=norm)
            assert orc.rel_l2(orc.gram(x, gm, norm=norm), ref.reshape(x.shape)) < 1e-5
    # one 2D mask (no frame axis) and a (ny,) line mask broadcast along x
    gm1 = orc.plan_gram(mask[0], N)
    x1 = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    ref1 = orc.sparse_ifftn(orc.sparse_fftn(x1, idx[0], N), idx[0], N).reshape(N)
    assert orc.rel_l2(orc.gram(x1, gm1), ref1) < 1e-5
    gml = orc.plan_gram(mask[0, :, 0], N, basis=basis[:1])
    assert gml.value.shape == (N[0] * N[1], K, K)


def test_oracle_cartesian_gram_with_field_map_vs_exact():
    """Dense Gram with B0 segments approximates E^H M E / (ny nx) of the exact
    off-resonance model (A^H A for the orthonormal sparse FFT), T the sampling
    time of every mask point (readout along x)."""
    rng = np.random.default_rng(13)
    N = (24, 24)
    mask, idx = _line_masks(rng, 1, N, 10)
    yy, xx = np.mgrid[:N[0], :N[1]] / N[0] - 0.5
    b0 = 100 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 50
    dt = 5e-3 / N[1]
    T = dt * np.broadcast_to(np.arange(N[1]), N)
    gm = orc.plan_gram(mask, N, zmap=b0, T=T, L=8, nbins=40)
    assert gm.value.shape == (8, 1, *N) and gm.zmap_s_kernel.shape == (8, *N)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    g = orc.gram(x, gm)
    r = orc.pixel_grid(N)
    pts = idx.reshape(-1, 2).astype(np.float64)
    cm = pts - np.array([N[1] // 2, N[0] // 2])
    tm = dt * pts[:, 0]
    E = np.exp(-2j * np.pi * (cm / np.array(N[::-1])) @ r.T) * np.exp(-2j * np.pi * tm[:, None] * b0.ravel()[None, :])
    ref = (E.conj().T @ (E @ x.ravel().astype(np.complex128))).reshape(N) / np.prod(N)
    assert orc.rel_l2(g, ref) < 2e-2


def shift_invariant_kspace(rng, nc, ndim, theta=0.8):
    """k(p) = u0 diag(exp(i p . th)) V^-1 for commuting shift operators
    G_a = V diag(exp(i th_a)) V^-1: a calibration on which GROG's least-squares
    operators are exact (lamda = 0).  Returns (k(p) for real positions p (..., ndim)
    in (x, y, z) order, calibration (nc, [nz,] ny, nx) on an 8^ndim grid)."""
    V = rng.standard_normal((nc, nc)) + 1j * rng.standard_normal((nc, nc))
    Vi = np.linalg.inv(V)
    th = rng.uniform(-theta, theta, (ndim, nc))
    u0 = (rng.standard_normal(nc) + 1j * rng.standard_normal(nc)) @ V

    def k_at(p):
        return (u0 * np.exp(1j * (np.asarray(p, np.float64) @ th))) @ Vi

    n = 8
    grid = np.stack(np.meshgrid(*([np.arange(n)] * ndim), indexing="ij"), -1)[..., ::-1]  # (z, y, x) -> (x, y, z)
    cal = np.moveaxis(k_at(grid.reshape(-1, ndim)).reshape(*([n] * ndim), nc), -1, 0)
    return k_at, cal


@pytest.mark.parametrize("ndim", [2, 3])
def test_oracle_grog_exact_on_shift_invariant_calibration(ndim):
    """Operator training, fractional powers, their composition order and the offset
    lookup: each sample at c = g - d (d = 0.05 + 0.1 q) must land on k(c + delta),
    delta = q / 10 the quantised offset, exactly up to rounding (the opposite shift
    direction or no shift at all misses by > 0.1)."""
    rng = np.random.default_rng(14)
    nc = 6
    k_at, cal = shift_invariant_kspace(rng, nc, ndim)
    g = rng.integers(-6, 6, (2, 30, ndim)).astype(np.float64)
    q = rng.integers(-5, 5, (2, 30, ndim))
    coord = (g - (0.05 + 0.1 * q)).astype(np.float32)
    x = np.moveaxis(k_at(coord.astype(np.float64)), -1, 0).astype(np.complex64)  # (nc, 2, 30)
    out, ind, w = orc.grog_interp(x, cal, coord, 16, lamda=0.0)
    delta = (np.floor(10 * (np.round(coord) - coord)).astype(np.float64)) / 10
    ref = np.moveaxis(k_at(coord.astype(np.float64) + delta), -1, 0)
    assert orc.rel_l2(out, ref) < 1e-5
    assert orc.rel_l2(out, np.moveaxis(k_at(coord.astype(np.float64) - delta), -1, 0)) > 0.1
    assert orc.rel_l2(x, ref) > 0.05
    np.testing.assert_array_equal(ind, np.round(coord).astype(np.int64) + 8)
    flat = (ind * np.array([1, 16, 256])[:ndim]).sum(-1).ravel()
    cnt = np.array([np.sum(flat == f) for f in flat])
    np.testing.assert_allclose(w.ravel(), 1.0 / cnt)


@pytest.mark.parametrize("d", [2, 3])
def test_masking_kernels_match_reference(golden, d):
    """The oracle's gather / scatter-add (the sparse FFT's masking step) against outputs
    of the reference's own _dense2sparse / _sparse2dense Numba kernels: gathers exact,
    sums within float32 rounding (the reference compiles with fastmath)."""
    p = f"m{d}d_"
    idx, shape, basis = golden[p + "index"], tuple(golden[p + "shape"]), golden[p + "basis"]
    np.testing.assert_array_equal(orc.dense_to_sparse(golden[p + "dense"], idx), golden[p + "sparse"])
    assert orc.rel_l2(orc.sparse_to_dense(golden[p + "ksp"], idx, shape), golden[p + "fill"]) < 1e-6
    assert orc.rel_l2(orc.dense_to_sparse(golden[p + "dense_sub"], idx, basis), golden[p + "sparse_sub"]) < 1e-6
    fill_s = orc.sparse_to_dense(golden[p + "ksp"], idx, shape, np.ascontiguousarray(basis.conj().T))
    assert orc.rel_l2(fill_s, golden[p + "fill_sub"]) < 1e-6


def test_threaded_glue_is_identical_to_per_item_glue():
    """The oracle's apodize / resize / centred FFT split large batches over host
    threads; every item sees the same operations, so the result is bit-identical."""
    rng = np.random.default_rng(30)
    x = (rng.standard_normal((5, 96, 96, 96)) + 1j * rng.standard_normal((5, 96, 96, 96))).astype(np.complex64)
    args = (3, (1.25,) * 3, (4,) * 3, (6.9966590477,) * 3)
    a = orc.apodize(x, *args)
    assert all(np.array_equal(a[i], orc.apodize(x[i:i + 1], *args)[0]) for i in range(5))
    r = orc.resize(x, (120, 120, 120))
    assert all(np.array_equal(r[i], orc.resize(x[i:i + 1], (120, 120, 120))[0]) for i in range(5))
    f = orc.fft_c(x, 3)
    assert all(np.array_equal(f[i], orc.fft_c(x[i:i + 1], 3)[0]) for i in range(5))


@pytest.mark.parametrize("ndim", [2, 3])
def test_float64_adjoint_restatement(ndim):
    """nufft_adj_f64 (the reference's adjoint algorithm in float64) agrees with the
    float32 restatement to float32 rounding and with the direct NUDFT adjoint to the
    kernel accuracy."""
    rng = np.random.default_rng(31 + ndim)
    N = (20,) * ndim
    coord = ((rng.random((300, ndim)) - 0.5) * N[0]).astype(np.float32)
    plan = orc.plan_nufft(coord, N, width=6, oversamp=2.0)
    y = (rng.standard_normal((2, 300)) + 1j * rng.standard_normal((2, 300))).astype(np.complex64)
    x64 = orc.nufft_adj_f64(y, plan)
    x32 = orc.nufft_adj(y, plan)
    assert orc.rel_l2(x32, x64) < 1e-6
    G = float(np.prod(plan.os_shape))
    ref = orc.nudft_adj(y, coord, N) / G
    assert orc.rel_l2(x64, ref) < 1e-4
