"""GPU: Cartesian (dense) Gram, plan_gram / gram, against the oracle's restatement
of src/pyfourier/_gram and against the normal operator of this package's own
sparse FFT on the mask's points."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402
from tests.test_gpu_nufft import crandn, rel  # noqa: E402
from tests.test_oracle import _line_masks  # noqa: E402

TOL = 1e-5  # rel-L2 vs the oracle (float32 FFTs in a different order)


def pf():
    import pyfourier_b200

    return pyfourier_b200


@pytest.mark.parametrize("norm", [None, "ortho"])
def test_dense_gram_frames_vs_oracle_and_sparse_fft(norm):
    rng = np.random.default_rng(0)
    N, F = (40, 48), 3
    mask, idx = _line_masks(rng, F, N, 12)
    gm = pf().plan_gram(torch.as_tensor(mask).cuda(), N)
    assert not gm.islowrank and gm.ncoeff == F
    x = crandn(rng, 2, F, *N)
    y = pf().gram(torch.as_tensor(x).cuda(), gm, norm=norm)
    assert y.shape == x.shape and y.is_cuda
    assert rel(y, orc.gram(x, orc.plan_gram(mask, N), norm=norm)) < TOL
    xs = torch.as_tensor(x).cuda()
    ahax = pf().sparse_ifftn(pf().sparse_fftn(xs, torch.as_tensor(idx), N, norm=norm), torch.as_tensor(idx), N,
                             norm=norm)
    assert rel(y, ahax.cpu().numpy().reshape(x.shape)) < TOL


def test_dense_gram_subspace_vs_oracle_and_sparse_fft():
    rng = np.random.default_rng(1)
    N, F, K = (32, 36), 10, 4
    mask, idx = _line_masks(rng, F, N, 6)
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    gm = pf().plan_gram(mask, N, basis=basis, device="cuda:0")
    assert gm.islowrank and tuple(gm.value.shape) == (N[0] * N[1], K, K)
    og = orc.plan_gram(mask, N, basis=basis)
    assert rel(gm.value, og.value) < TOL
    x = crandn(rng, 2, 3, K, *N)
    y = pf().gram(torch.as_tensor(x).cuda(), gm)
    assert rel(y, orc.gram(x, og)) < TOL
    ahax = pf().sparse_ifftn(pf().sparse_fftn(x, idx, N, basis=basis), idx, N, basis=basis)
    assert rel(y, ahax.reshape(x.shape)) < TOL


def test_dense_gram_line_mask_numpy_and_weights():
    """A (ny,) line mask broadcast along x, non-binary mask values (weights),
    NumPy in and out."""
    rng = np.random.default_rng(2)
    N = (24, 30)
    line = (rng.random(N[0]) < 0.4) * rng.random(N[0]).astype(np.float32)
    basis = crandn(rng, 1, 2)
    gm = pf().plan_gram(line, N, basis=basis)
    x = crandn(rng, 5, 2, *N)
    y = pf().gram(x, gm)
    assert isinstance(y, np.ndarray) and y.shape == x.shape
    assert rel(y, orc.gram(x, orc.plan_gram(line, N, basis=basis))) < TOL
    m2 = rng.random(N).astype(np.float32)  # one 2D weight plane, no frame axis
    y2 = pf().gram(x[:, 0], pf().plan_gram(m2, N))
    assert rel(y2, orc.gram(x[:, 0], orc.plan_gram(m2, N))) < TOL


def test_dense_gram_field_map_vs_oracle():
    rng = np.random.default_rng(3)
    N, F = (32, 32), 2
    mask, _ = _line_masks(rng, F, N, 10)
    yy, xx = np.mgrid[:N[0], :N[1]] / N[0] - 0.5
    b0 = 120 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 60
    T = 5e-3 / N[1] * np.broadcast_to(np.arange(N[1]), N)
    gm = pf().plan_gram(mask, N, zmap=torch.as_tensor(b0), T=T, L=6, device="cuda:0")
    og = orc.plan_gram(mask, N, zmap=b0, T=T, L=6)
    assert gm.nseg == 6 and tuple(gm.value.shape) == og.value.shape
    x = crandn(rng, 2, F, *N)
    assert rel(pf().gram(torch.as_tensor(x).cuda(), gm), orc.gram(x, og)) < TOL


def test_dense_gram_autograd_is_self_adjoint():
    rng = np.random.default_rng(4)
    N, F, K = (16, 24), 5, 3
    mask, _ = _line_masks(rng, F, N, 5)
    basis = np.linalg.qr(crandn(rng, F, K))[0].astype(np.complex64)
    gm = pf().plan_gram(mask, N, basis=basis, device="cuda:0")
    x = torch.as_tensor(crandn(rng, 2, K, *N)).cuda().requires_grad_(True)
    v = torch.as_tensor(crandn(rng, 2, K, *N)).cuda()
    (pf().gram(x, gm) * v.conj()).real.sum().backward()
    assert rel(x.grad, pf().gram(v, gm).cpu().numpy()) < TOL


def test_dense_gram_rejects_bad_shapes():
    with pytest.raises(ValueError):
        pf().plan_gram(np.ones((4, 4, 4), np.float32), (4, 4, 4))
    with pytest.raises(ValueError):
        pf().plan_gram(np.ones((2, 6, 5), np.float32), (6, 6))
    gm = pf().plan_gram(np.ones((6, 6), np.float32), (6, 6))
    with pytest.raises(ValueError):
        pf().gram(torch.zeros(6, 5, dtype=torch.complex64).cuda(), gm)
