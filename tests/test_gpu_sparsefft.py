"""GPU: sparse (Cartesian-subsampled) FFT, plan_spfft / sparse_fftn / sparse_ifftn,
against the oracle's restatement of src/pyfourier/_sparsefft and its masking
kernels (centred FFT + gather, scatter-add + centred inverse FFT)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402
from tests.test_gpu_nufft import crandn, rel  # noqa: E402

TOL = 1e-5  # rel-L2 vs the oracle (float32 FFT and scatter order differ)


def pf():
    import pyfourier_b200

    return pyfourier_b200


def _indexes(rng, shape, lead):
    """Random grid indexes in [0, N), axes (x, y[, z]) for a (z, y, x) shape."""
    return np.stack([rng.integers(0, n, lead) for n in shape[::-1]], -1).astype(np.float32)


@pytest.mark.parametrize("norm", [None, "ortho"])
def test_sparse_fft_2d_frames_and_duplicates(norm):
    rng = np.random.default_rng(0)
    N, F = (40, 48), 3
    idx = _indexes(rng, N, (F, 20, 30))
    idx[1, 3, :5] = idx[1, 3, 5]  # repeated points add in the adjoint
    x = crandn(rng, 2, F, *N)
    y = crandn(rng, 2, F, 20, 30)
    k = pf().sparse_fftn(torch.as_tensor(x).cuda(), torch.as_tensor(idx), N, norm=norm)
    assert k.shape == (2, F, 20, 30)
    assert rel(k, orc.sparse_fftn(x, idx, N, norm=norm).reshape(k.shape)) < TOL
    im = pf().sparse_ifftn(torch.as_tensor(y).cuda(), torch.as_tensor(idx), N, norm=norm)
    assert im.shape == (2, F, *N)
    assert rel(im, orc.sparse_ifftn(y, idx, N, norm=norm)) < TOL


def test_sparse_fft_3d_plan_reuse_and_centred_input():
    rng = np.random.default_rng(1)
    N = (16, 20, 24)
    idx = _indexes(rng, N, (30, 50))
    plan = pf().plan_spfft(torch.as_tensor(idx).cuda(), N)
    assert plan.ishape == N and plan.dshape == (30, 50) and len(plan.index) == 3
    x = crandn(rng, 3, *N)
    k = pf().sparse_fftn(torch.as_tensor(x).cuda(), plan=plan)
    assert rel(k, orc.sparse_fftn(x, idx, N).reshape(k.shape)) < TOL
    # the same points given as centred coordinates (negative entries present)
    centred = idx - np.array([s // 2 for s in N[::-1]], np.float32)
    k2 = pf().sparse_fftn(torch.as_tensor(x).cuda(), torch.as_tensor(centred), N)
    assert rel(k2, k.cpu().numpy()) < TOL
    y = crandn(rng, 3, 30, 50)
    im = pf().sparse_ifftn(torch.as_tensor(y).cuda(), plan=plan)
    assert rel(im, orc.sparse_ifftn(y, idx, N).reshape(im.shape)) < TOL


def test_sparse_fft_subspace_basis_and_numpy():
    rng = np.random.default_rng(2)
    N, F, K = (32, 32), 6, 3
    idx = _indexes(rng, N, (F, 8, 40))
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    x = crandn(rng, 2, K, *N)
    y = crandn(rng, 2, F, 8, 40)
    k = pf().sparse_fftn(x, idx, N, basis=basis)
    assert isinstance(k, np.ndarray)
    assert rel(k, orc.sparse_fftn(x, idx, N, basis=basis).reshape(k.shape)) < TOL
    im = pf().sparse_ifftn(y, idx, N, basis=basis)
    assert rel(im, orc.sparse_ifftn(y, idx, N, basis=basis).reshape(im.shape)) < TOL


def test_sparse_fft_b0_segments_vs_width_one_nufft():
    """With a field map the sparse FFT is the width-1 NUFFT with B0 segments; the
    oracle's NUFFT restatement gives the reference's B0 model."""
    rng = np.random.default_rng(3)
    N, nv, ns = (32, 32), 10, 64
    idx = _indexes(rng, N, (nv, ns))
    yy, xx = np.mgrid[:32, :32] / 32 - 0.5
    b0 = 120 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 60
    dt = 5e-3 / ns
    coord = idx - np.array([16, 16], np.float32)
    oplan = orc.plan_nufft(coord, N, width=2, oversamp=1.0, zmap=b0, L=6, nbins=40, dt=dt)
    x = crandn(rng, 2, *N)
    y = crandn(rng, 2, nv, ns)
    k = pf().sparse_fftn(torch.as_tensor(x).cuda(), torch.as_tensor(idx), N, zmap=torch.as_tensor(b0), L=6,
                         nbins=40, dt=dt)
    assert rel(k, orc.nufft_fwd(x, oplan)) < TOL
    im = pf().sparse_ifftn(torch.as_tensor(y).cuda(), torch.as_tensor(idx), N, zmap=torch.as_tensor(b0), L=6,
                           nbins=40, dt=dt)
    assert rel(im, orc.nufft_adj(y, oplan)) < TOL


def test_sparse_fft_rejects_off_grid_points():
    with pytest.raises(ValueError):
        pf().plan_spfft(torch.tensor([[0.5, 1.0]]), (8, 8))
