"""GPU: Toeplitz Gram vs the oracle and vs A^H W A; autograd image and trajectory
gradients vs float64 references (central finite differences with h = 1e-4 and
a float64 direct-NUDFT autograd gradient)."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402
from tests.test_gpu_nufft import crandn, radial, rel  # noqa: E402


def pf():
    import pyfourier_b200

    return pyfourier_b200


def spiral_frames(F, ninter, nsamp, N, seed=0):
    t = np.linspace(0, 1, nsamp, dtype=np.float64)
    r = t * (N / 2 - 1)
    th = 2 * np.pi * 6 * np.sqrt(t)
    ga = np.pi * (3 - np.sqrt(5))
    out = []
    for f in range(F):
        arms = []
        for i in range(ninter):
            a = th + 2 * np.pi * i / ninter + f * ga
            arms.append(np.stack([r * np.cos(a), r * np.sin(a)], -1))
        out.append(np.stack(arms))
    return np.stack(out).astype(np.float32)


@pytest.mark.parametrize("normalize", ["reference", None])
def test_gram_subspace_vs_oracle(normalize):
    P = pf()
    rng = np.random.default_rng(0)
    N, F, K = 24, 8, 4
    coord = spiral_frames(F, 4, 128, N)
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    og = orc.plan_spgram(coord, (N, N), basis=basis, normalize=normalize)
    gg = P.plan_spgram(torch.as_tensor(coord), (N, N), basis=torch.as_tensor(basis), device="cuda:0",
                       normalize=normalize)
    assert gg.islowrank and gg.value.shape == og.value.shape
    assert rel(gg.value, og.value) < 1e-5
    x = crandn(rng, 3, K, N, N)
    assert rel(P.sparse_gram(torch.as_tensor(x).cuda(), gg), orc.sparse_gram(x, og)) < 1e-5


@pytest.mark.parametrize("zmap", [False, True])
def test_psf_float64_matches_oracle(zmap):
    """The Toeplitz kernel is built in float64 at plan time on the GPU (float64
    spread kernel, complex128 transforms) and by the oracle (float64 C spread,
    NumPy complex128): both stored as complex64, they agree to 1e-6."""
    P = pf()
    rng = np.random.default_rng(20)
    N, F, K = 24, 8, 4
    coord = spiral_frames(F, 4, 128, N)
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    kw = dict(zmap=_b0_map(N), L=4, nbins=40, dt=5e-3 / 128) if zmap else {}
    og = orc.plan_spgram(coord, (N, N), basis=basis, normalize=None, **kw)
    gg = P.plan_spgram(torch.as_tensor(coord), (N, N), basis=torch.as_tensor(basis), device="cuda:0",
                       normalize=None, **{k: (torch.as_tensor(v) if k == "zmap" else v) for k, v in kw.items()})
    assert tuple(gg.value.shape) == tuple(og.value.shape)
    assert rel(gg.value, og.value) < 1e-6


def test_gram_exact_equals_ahwa_gpu():
    """normalize=None: sparse_gram(x) == A^H W A x (A = nufft norm None, A^H exact adjoint)."""
    P = pf()
    rng = np.random.default_rng(1)
    N = 32
    coord = radial(40, 64, N)
    w = rng.random((40, 64)).astype(np.float32)
    gm = P.plan_spgram(torch.as_tensor(coord), (N, N), weight=torch.as_tensor(w), device="cuda:0",
                       normalize=None)
    x = torch.as_tensor(crandn(rng, 2, N, N)).cuda()
    g = P.sparse_gram(x, gm)
    ref = orc.nudft_adj(w.ravel() * orc.nudft_fwd(x.cpu().numpy(), coord.reshape(-1, 2), (N, N)),
                        coord.reshape(-1, 2), (N, N))
    assert rel(g, ref) < 2e-3


def test_gram_elementwise_multiframe():
    P = pf()
    rng = np.random.default_rng(2)
    N, F = 20, 3
    coord = spiral_frames(F, 3, 96, N)
    og = orc.plan_spgram(coord, (N, N))
    gg = P.plan_spgram(torch.as_tensor(coord), (N, N), device="cuda:0")
    x = crandn(rng, 2, F, N, N)
    assert rel(P.sparse_gram(torch.as_tensor(x).cuda(), gg), orc.sparse_gram(x, og)) < 1e-5


def test_gram_autograd_self_adjoint():
    P = pf()
    rng = np.random.default_rng(3)
    N = 16
    coord = radial(12, 32, N)
    gm = P.plan_spgram(torch.as_tensor(coord), (N, N), device="cuda:0")
    x = torch.as_tensor(crandn(rng, N, N)).cuda().requires_grad_(True)
    v = torch.as_tensor(crandn(rng, N, N)).cuda()
    loss = torch.real(torch.vdot(v.flatten(), P.sparse_gram(x, gm).flatten()))
    loss.backward()
    ref = P.sparse_gram(v, gm)  # G Hermitian => d Re<v, Gx>/dx* ~ G v
    assert rel(x.grad, ref.detach().cpu().numpy()) < 1e-5


def _b0_map(N):
    yy, xx = np.mgrid[:N, :N] / N - 0.5
    return 100 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 50


@pytest.mark.parametrize("subspace", [False, True])
def test_gram_field_map_vs_oracle(subspace):
    """Time-segmented Gram: L kernels, sum_l conj(C_l) G_l(C_l x), same as the oracle."""
    P = pf()
    rng = np.random.default_rng(4)
    N, ns = 24, 64
    dt = 5e-3 / ns
    b0 = _b0_map(N)
    if subspace:
        F, K = 6, 3
        coord = spiral_frames(F, 3, ns, N)
        basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
        x = crandn(rng, 2, K, N, N)
    else:
        coord, basis = radial(16, ns, N), None
        x = crandn(rng, 2, N, N)
    og = orc.plan_spgram(coord, (N, N), basis=basis, zmap=b0, L=6, nbins=40, dt=dt)
    gg = P.plan_spgram(torch.as_tensor(coord), (N, N), basis=None if basis is None else torch.as_tensor(basis),
                       zmap=torch.as_tensor(b0), L=6, nbins=40, dt=dt, device="cuda:0")
    assert gg.nseg == 6 and gg.value.shape == og.value.shape
    assert rel(gg.value, og.value) < 1e-5
    assert rel(gg.zmap_s_kernel, og.zmap_s_kernel) < 1e-6
    assert rel(P.sparse_gram(torch.as_tensor(x).cuda(), gg), orc.sparse_gram(x, og)) < 1e-5


def test_gram_field_map_vs_exact_model():
    """normalize=None: the segmented Gram approximates E^H E of the exact
    off-resonance model E = exp(-i 2 pi (k r + t b0(r))) (segmentation error only)."""
    P = pf()
    rng = np.random.default_rng(7)
    N, nv, ns = 24, 16, 64
    coord = radial(nv, ns, N)
    b0 = _b0_map(N)
    dt = 5e-3 / ns
    gm = P.plan_spgram(torch.as_tensor(coord), (N, N), zmap=torch.as_tensor(b0), L=8, nbins=40, dt=dt,
                       device="cuda:0", normalize=None)
    x = crandn(rng, N, N)
    g = P.sparse_gram(torch.as_tensor(x).cuda(), gm)
    r = orc.pixel_grid((N, N))
    cm = coord.reshape(-1, 2).astype(np.float64)
    tm = np.tile(dt * np.arange(ns), nv)
    E = np.exp(-2j * np.pi * (cm / N) @ r.T) * np.exp(-2j * np.pi * tm[:, None] * b0.ravel()[None, :])
    ref = (E.conj().T @ (E @ x.ravel().astype(np.complex128))).reshape(N, N)
    assert rel(g, ref) < 2e-2


# ---------------------------------------------------------------------------------
# autograd
# ---------------------------------------------------------------------------------
def _kb64(u, beta):
    u = np.asarray(u, np.float64)
    out = np.zeros_like(u)
    m = np.abs(u) <= 1
    a = beta * np.sqrt(1 - u[m] ** 2)
    t = a / 3.75
    small = a < 3.75
    v = np.empty_like(a)
    ts = t[small]
    v[small] = (1 + 3.5156229 * ts ** 2 + 3.0899424 * ts ** 4 + 1.2067492 * ts ** 6 + 0.2659732 * ts ** 8
                + 0.0360768 * ts ** 10 + 0.0045813 * ts ** 12)
    al, tl = a[~small], t[~small]
    v[~small] = al ** -0.5 * np.exp(al) * (0.39894228 + 0.01328592 / tl + 0.00225319 / tl ** 2 - 0.00157565 / tl ** 3
                                          + 0.00916281 / tl ** 4 - 0.02057706 / tl ** 5 + 0.02635537 / tl ** 6
                                          - 0.01647633 / tl ** 7 + 0.00392377 / tl ** 8)
    out[m] = v
    return out


def _fwd64(x, coord, N, W, osf, beta, x0_fixed=None):
    """Float64 restatement of the discretised forward NUFFT (2D), for finite differences.
    x (N, N) ; coord (M, 2) float64 (x, y).  Returns (y (M,), x0 (M, 2))."""
    nos = int(np.ceil(np.float32(osf) * np.float32(N)))
    a = orc.apod_vector(N, osf, W, beta).astype(np.float64)
    img = x * a[:, None] * a[None, :]
    pad = orc.resize(img.astype(np.complex128), (nos, nos))
    H = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(pad)))
    scale = orc.kernel_scaling([beta, beta], [W, W])
    c = coord * (nos / N) + nos // 2
    x0 = np.ceil(c - W / 2) if x0_fixed is None else x0_fixed
    taps = np.arange(W)
    wx = _kb64(((x0[:, 0:1] + taps) - c[:, 0:1]) / (W / 2), beta)
    wy = _kb64(((x0[:, 1:2] + taps) - c[:, 1:2]) / (W / 2), beta)
    ix = np.mod(x0[:, 0:1] + taps, nos).astype(int)
    iy = np.mod(x0[:, 1:2] + taps, nos).astype(int)
    vals = H[iy[:, :, None], ix[:, None, :]]  # (M, W, W) [y, x]
    y = np.einsum("my,mx,myx->m", wy, wx, vals) / scale
    return y, x0


def test_image_gradient_is_exact_adjoint():
    P = pf()
    rng = np.random.default_rng(4)
    N = 32
    coord = radial(20, 64, N)
    plan = P.plan_nufft(torch.as_tensor(coord), (N, N), width=4, oversamp=2.0, device="cuda:0")
    for norm in (None, "ortho"):
        x = torch.as_tensor(crandn(rng, 2, N, N)).cuda().requires_grad_(True)
        v = torch.as_tensor(crandn(rng, 2, 20, 64)).cuda()
        loss = torch.real(torch.vdot(v.flatten(), P.nufft(x, nufft_plan=plan, norm=norm).flatten()))
        loss.backward()
        G = 1.0 if norm == "ortho" else float(np.prod(plan.os_shape))
        ref = P.nufft_adj(v, nufft_plan=plan, norm=norm) * G
        assert rel(x.grad, ref.detach().cpu().numpy()) < 1e-5
        # and for the adjoint operator
        yk = torch.as_tensor(crandn(rng, 2, 20, 64)).cuda().requires_grad_(True)
        u = torch.as_tensor(crandn(rng, 2, N, N)).cuda()
        loss = torch.real(torch.vdot(u.flatten(), P.nufft_adj(yk, nufft_plan=plan, norm=norm).flatten()))
        loss.backward()
        ref = P.nufft(u, nufft_plan=plan, norm=norm) / G
        assert rel(yk.grad, ref.detach().cpu().numpy()) < 1e-5


def test_traj_grad_vs_fp64_finite_differences():
    """d/dk Re<v, A(k) x> on the GPU vs float64 central differences (h = 1e-4)
    of the same discretised operator, per sample and axis, away from the
    kernel-support switch points (where x0 jumps)."""
    P = pf()
    rng = np.random.default_rng(5)
    N, W, osf = 32, 4, 2.0
    M = 300
    coord = ((rng.random((M, 2)) - 0.5) * (N - 2)).astype(np.float32)
    beta = float(orc.beta_f32((W,), (osf,))[0])
    x = crandn(rng, N, N)
    v = crandn(rng, M)
    ct = torch.as_tensor(coord).cuda().requires_grad_(True)
    y = P.nufft(torch.as_tensor(x).cuda(), ct, (N, N), width=W, oversamp=osf, device="cuda:0")
    loss = torch.real(torch.vdot(torch.as_tensor(v).cuda(), y.flatten()))
    loss.backward()
    g_gpu = ct.grad.cpu().numpy().astype(np.float64)
    c64 = coord.astype(np.float64)
    _, x0 = _fwd64(x, c64, N, W, osf, beta)
    nos = 2 * N
    cos_ = c64 * (nos / N) + nos // 2
    frac = cos_ - W / 2 - np.floor(cos_ - W / 2)
    safe = np.all((frac > 1e-2) & (frac < 1 - 1e-2), axis=1)
    h = 1e-4
    g_fd = np.zeros_like(c64)
    for ax in range(2):
        cp = c64.copy()
        cm = c64.copy()
        cp[:, ax] += h
        cm[:, ax] -= h
        yp, _ = _fwd64(x, cp, N, W, osf, beta, x0_fixed=x0)
        ym, _ = _fwd64(x, cm, N, W, osf, beta, x0_fixed=x0)
        # loss is separable over samples: per-sample central difference
        g_fd[:, ax] = np.real(np.conj(v) * (yp - ym)) / (2 * h)
    err = np.linalg.norm((g_gpu - g_fd)[safe]) / np.linalg.norm(g_fd[safe])
    assert safe.sum() > 250
    assert err < 1e-3, err


def test_traj_and_image_grad_vs_fp64_nudft_autograd():
    """Loss ||A^H A x - x||^2 at 64x64: GPU gradients vs torch float64 autograd of
    the direct NUDFT (differences are the NUFFT approximation error)."""
    P = pf()
    rng = np.random.default_rng(6)
    N, W, osf = 64, 6, 2.0
    coord = spiral_frames(1, 4, 256, N)[0]  # (4, 256, 2)
    x = crandn(rng, N, N)
    # GPU (norm="ortho" so that A^H is the true adjoint)
    ct = torch.as_tensor(coord).cuda().requires_grad_(True)
    xt = torch.as_tensor(x).cuda().requires_grad_(True)
    plan = P.plan_nufft(ct.detach(), (N, N), width=W, oversamp=osf, device="cuda:0")
    y = P.nufft(xt, ct, nufft_plan=plan, norm="ortho")
    z = P.nufft_adj(y, ct, nufft_plan=plan, norm="ortho")
    loss = torch.sum(torch.abs(z - xt) ** 2)
    loss.backward()
    # float64 NUDFT with the same normalisation: A = E / sqrt(G_os) ... ortho NUFFT ~ E / sqrt(G)
    G = float(np.prod(plan.os_shape))
    c64 = torch.as_tensor(coord.reshape(-1, 2), dtype=torch.float64).requires_grad_(True)
    x64 = torch.as_tensor(x, dtype=torch.complex128).requires_grad_(True)
    r = torch.as_tensor(orc.pixel_grid((N, N)))
    E = torch.exp(-2j * math.pi * ((c64 / N) @ r.T)) / math.sqrt(G)
    y64 = E @ x64.flatten()
    z64 = (E.conj().T @ y64).reshape(N, N)
    loss64 = torch.sum(torch.abs(z64 - x64) ** 2)
    loss64.backward()
    gx_err = rel(xt.grad, x64.grad.numpy())
    gc_err = rel(ct.grad.reshape(-1, 2), c64.grad.numpy())
    assert gx_err < 1e-3, gx_err
    assert gc_err < 1e-2, gc_err
