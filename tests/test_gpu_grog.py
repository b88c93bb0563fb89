"""GPU: GROG pre-interpolation (grog_interp through pfb_grog_apply) against the
oracle's restatement of src/pyfourier/_preinterp/_grog.py, and against the exact
shifts of a shift-invariant calibration."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402
from tests.test_gpu_nufft import crandn, rel  # noqa: E402
from tests.test_oracle import shift_invariant_kspace  # noqa: E402

TOL = 1e-5  # rel-L2 vs the oracle (complex64 operators and float32 sums)


def pf():
    import pyfourier_b200

    return pyfourier_b200


def _coords(rng, lead, ndim, half):
    return ((rng.random((*lead, ndim)) - 0.5) * 2 * half).astype(np.float32)


def _check(out, ind, w, ref):
    o, i, ww = ref
    assert rel(out, o) < TOL
    np.testing.assert_array_equal(ind.cpu().numpy() if isinstance(ind, torch.Tensor) else ind, i)
    np.testing.assert_array_equal(w.cpu().numpy() if isinstance(w, torch.Tensor) else w, ww)


@pytest.mark.parametrize("nc", [8, 7, 40])
def test_grog_2d_vs_oracle(nc):
    """Single calibration slice, extra batch axes, coil counts in both apply variants
    (operator column in registers for nc <= 32, in shared memory above), odd nc."""
    rng = np.random.default_rng(nc)
    N = 48
    coord = _coords(rng, (3, 20, 64), 2, N / 2)  # reaches the grid edge: some samples fall outside
    cal = crandn(rng, nc, 16, 16)
    x = crandn(rng, 2, nc, 3, 20, 64)
    out, ind, w = pf().grog_interp(torch.as_tensor(x).cuda(), torch.as_tensor(cal), torch.as_tensor(coord), N)
    assert out.shape == x.shape and out.is_cuda and ind.shape == (3, 20, 64, 2) and ind.dtype == torch.int64
    _check(out, ind, w, orc.grog_interp(x, cal, coord, N))
    outside = ((np.round(coord) + N // 2 < 0) | (np.round(coord) + N // 2 >= N)).any(-1)
    assert outside.any() and np.all(out.cpu().numpy()[..., outside] == 0)


def test_grog_2d_per_slice_operators_and_numpy():
    rng = np.random.default_rng(1)
    N, nz, nc = 40, 3, 12
    coord = _coords(rng, (30, 50), 2, 15)
    cal = crandn(rng, nc, nz, 12, 12)
    x = crandn(rng, nz, nc, 30, 50)
    out, ind, w = pf().grog_interp(x, cal, coord, (N, N), lamda=0.05, nsteps=9)
    assert isinstance(out, np.ndarray) and isinstance(ind, np.ndarray)
    _check(out, ind, w, orc.grog_interp(x, cal, coord, (N, N), lamda=0.05, nsteps=9))
    with pytest.raises(ValueError):
        pf().grog_interp(x[:2], cal, coord, N)


def test_grog_3d_vs_oracle_with_crowded_operators():
    """3D; half of the samples share one offset, so that operator spans many chunks."""
    rng = np.random.default_rng(2)
    N, nc = 32, 16
    coord = _coords(rng, (40, 100), 3, 14)
    coord[:20] = np.round(coord[:20]) - np.float32(0.25)
    cal = crandn(rng, nc, 8, 8, 8)
    x = crandn(rng, 2, nc, 40, 100)
    out, ind, w = pf().grog_interp(torch.as_tensor(x).cuda(), torch.as_tensor(cal).cuda(),
                                   torch.as_tensor(coord).cuda(), (N, N, N))
    _check(out, ind, w, orc.grog_interp(x, cal, coord, (N, N, N)))


@pytest.mark.parametrize("ndim", [2, 3])
def test_grog_exact_shifts_on_shift_invariant_calibration(ndim):
    rng = np.random.default_rng(3 + ndim)
    nc = 10
    k_at, cal = shift_invariant_kspace(rng, nc, ndim)
    g = rng.integers(-6, 6, (4, 256, ndim)).astype(np.float64)
    d = 0.05 + 0.1 * rng.integers(-5, 5, (4, 256, ndim))
    coord = (g - d).astype(np.float32)
    x = np.moveaxis(k_at(coord.astype(np.float64)), -1, 0).astype(np.complex64)
    out, _, _ = pf().grog_interp(torch.as_tensor(x).cuda(), torch.as_tensor(cal), torch.as_tensor(coord), 16,
                                 lamda=0.0)
    delta = np.floor(10 * (np.round(coord) - coord)).astype(np.float64) / 10
    assert rel(out, np.moveaxis(k_at(coord.astype(np.float64) + delta), -1, 0)) < 1e-4


def test_grog_plan_reuse_and_all_outside():
    rng = np.random.default_rng(4)
    N, nc = 16, 4
    cal = crandn(rng, nc, 8, 8)
    plan = pf().GrogPlan(cal, _coords(rng, (10, 30), 2, 7), N, device="cuda:0")
    x = torch.as_tensor(crandn(rng, 5, nc, 300)).cuda()
    assert rel(plan.apply(x), plan.apply(x.clone()).cpu().numpy()) == 0
    far = np.full((2, 5, 2), 40.0, np.float32)  # every sample outside the grid
    out, ind, w = pf().grog_interp(torch.as_tensor(crandn(rng, nc, 2, 5)).cuda(), cal, far, N)
    assert torch.count_nonzero(out) == 0 and int(ind.max()) == N - 1
