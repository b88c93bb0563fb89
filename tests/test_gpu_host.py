"""GPU: operators called with host (CPU) data.  Large host batches take the chunked
path whose copies overlap the computation; the results must match the same call
on device-resident data."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from tests.test_gpu_nufft import crandn, radial, rel  # noqa: E402

TOL = 1e-5  # rel-L2: chunks with fewer channels may take another spread kernel (other summation order)


@pytest.fixture
def chunked(monkeypatch):
    from pyfourier_b200 import _nufft

    monkeypatch.setattr(_nufft, "_HOST_PIPELINE_MIN_BYTES", 0)
    return _nufft


@pytest.mark.parametrize("pinned", [True, False])
def test_host_batches_match_device_results(chunked, pinned):
    import pyfourier_b200 as pf

    rng = np.random.default_rng(0)
    N = 24
    coord = ((rng.random((40, 60, 3)) - 0.5) * N).astype(np.float32)
    plan = pf.plan_nufft(torch.as_tensor(coord).cuda(), (N, N, N), width=4, oversamp=1.25, device="cuda:0")
    x = torch.as_tensor(crandn(rng, 5, N, N, N))  # 5 coils: uneven chunks
    xh = x.pin_memory() if pinned else x
    y_dev = pf.nufft(x.cuda(), nufft_plan=plan)
    y_host = pf.nufft(xh, nufft_plan=plan)
    assert y_host.device.type == "cpu" and y_host.is_pinned() and y_host.shape == (5, 40, 60)
    assert rel(y_host, y_dev.cpu().numpy()) < TOL
    k = torch.as_tensor(crandn(rng, 5, 40, 60))
    kh = k.pin_memory() if pinned else k
    a_dev = pf.nufft_adj(k.cuda(), nufft_plan=plan)
    a_host = pf.nufft_adj(kh, nufft_plan=plan)
    assert a_host.device.type == "cpu" and a_host.shape == (5, N, N, N)
    assert rel(a_host, a_dev.cpu().numpy()) < TOL


def test_host_numpy_round_trip_2d(chunked):
    import pyfourier_b200 as pf

    rng = np.random.default_rng(1)
    N = 32
    coord = radial(20, 64, N)
    plan = pf.plan_nufft(torch.as_tensor(coord).cuda(), (N, N), width=4, oversamp=2.0, device="cuda:0")
    x = crandn(rng, 3, 2, N, N)  # two leading batch axes
    y = pf.nufft(x, nufft_plan=plan)
    assert isinstance(y, np.ndarray) and y.shape == (3, 2, 20, 64)
    assert rel(y, pf.nufft(torch.as_tensor(x).cuda(), nufft_plan=plan).cpu().numpy()) < TOL
    a = pf.nufft_adj(y, nufft_plan=plan, norm="ortho")
    assert rel(a, pf.nufft_adj(torch.as_tensor(y).cuda(), nufft_plan=plan, norm="ortho").cpu().numpy()) < TOL
