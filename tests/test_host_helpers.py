"""Host-side helpers of the operators (no GPU): norm codes, sample shapes, the split of
`weight` between the kernels (real per-sample weights) and torch (everything else),
dtype promotion of the input and the choice of the chunked host path."""

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from pyfourier_b200 import _lib, _nufft

CPU = torch.device("cpu")


def test_norm_code():
    assert _nufft.norm_code(None) == _lib.PFB_NORM_NONE
    assert _nufft.norm_code("ortho") == _lib.PFB_NORM_ORTHO
    with pytest.raises(ValueError):
        _nufft.norm_code("forward")


def test_sample_shape():
    flat = SimpleNamespace(dshape=None, total_samples=123, nframes=4)
    assert _nufft._sample_shape(flat) == (123,)
    one = SimpleNamespace(dshape=(16, 40), total_samples=640, nframes=1)
    assert _nufft._sample_shape(one) == (16, 40)
    many = SimpleNamespace(dshape=(16, 40), total_samples=1920, nframes=3)
    assert _nufft._sample_shape(many) == (3, 16, 40)


def test_split_weight_kernel_and_torch_parts():
    ss = (3, 16, 40)
    assert _nufft._split_weight(None, ss, CPU) == (None, None)
    # a real per-sample weight goes to the kernels, flattened in sample order, float32
    w = np.random.default_rng(0).random(ss)
    ws, wt = _nufft._split_weight(w, ss, CPU)
    assert wt is None and ws.dtype == torch.float32 and ws.shape == (3 * 16 * 40,)
    assert torch.equal(ws, torch.as_tensor(w, dtype=torch.float32).reshape(-1))
    # leading singleton axes and broadcasting over views are still per-sample
    ws, wt = _nufft._split_weight(w[None, None], ss, CPU)
    assert wt is None and ws.shape == (1920,)
    ws, wt = _nufft._split_weight(np.ones((1, 1, 40)), ss, CPU)
    assert wt is None and torch.equal(ws, torch.ones(1920))
    # a weight with a real batch axis (one per coil) is applied with torch
    ws, wt = _nufft._split_weight(np.ones((8,) + ss), ss, CPU)
    assert ws is None and wt.shape == (8,) + ss and wt.dtype == torch.float32
    # complex weights are applied with torch, in complex64
    ws, wt = _nufft._split_weight(np.ones(ss, np.complex128), ss, CPU)
    assert ws is None and wt.dtype == torch.complex64
    # a shape that does not broadcast to the samples is left to torch (which will raise there)
    ws, wt = _nufft._split_weight(np.ones((7,)), ss, CPU)
    assert ws is None and wt is not None


@pytest.mark.parametrize("dtype", [np.float16, np.float32, np.float64, np.complex64, np.complex128])
def test_to_compute_promotes_to_complex64(dtype):
    x = np.arange(6).reshape(2, 3).astype(dtype)
    orig, xc = _nufft._to_compute(x, CPU)
    assert xc.dtype == torch.complex64 and xc.shape == (2, 3)
    assert np.allclose(xc.numpy(), x.astype(np.complex128))
    assert orig.dtype == torch.as_tensor(x).dtype


def test_host_pipeline_choice(monkeypatch):
    monkeypatch.setattr(_nufft, "_HOST_PIPELINE_MIN_BYTES", 1024)
    big = torch.zeros(200, dtype=torch.complex64)  # 1600 bytes
    assert _nufft._host_pipelined(big, None)
    assert not _nufft._host_pipelined(torch.zeros(100, dtype=torch.complex64), None)  # 800 bytes
    assert not _nufft._host_pipelined(big.to(torch.complex128), None)
    assert not _nufft._host_pipelined(big.clone().requires_grad_(True), None)
    assert not _nufft._host_pipelined(big, torch.zeros(3, requires_grad=True))
    assert _nufft._HOST_PIPELINE_CHUNKS_FWD >= _nufft._HOST_PIPELINE_CHUNKS_ADJ >= 1


def test_resolve_device_maps_the_reference_arguments(monkeypatch):
    from pyfourier_b200 import _plan

    monkeypatch.setattr(torch.cuda, "is_available", lambda: True)
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 1)
    rd = _plan.resolve_device
    assert rd("cpu") == torch.device("cuda:1")          # the reference's default: the current GPU
    assert rd(-1) == torch.device("cuda:1")
    assert rd(None) == torch.device("cuda:1")
    assert rd(3) == torch.device("cuda:3")
    assert rd("cuda") == torch.device("cuda:1")
    assert rd("cuda:2") == torch.device("cuda:2")
    assert rd(torch.device("cuda:0")) == torch.device("cuda:0")
    assert rd("cpu", fallback=torch.device("cuda:2")) == torch.device("cuda:2")  # the input's GPU
    assert rd("cpu", fallback=torch.device("cpu")) == torch.device("cuda:1")
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        rd("cuda:0")


@pytest.mark.parametrize("B", [1, 2, 3, 5, 8, 16, 31, 32, 33, 64, 100])
@pytest.mark.parametrize("chunks", [1, 4, 7])
def test_host_pipeline_chunks_partition_the_batch(B, chunks):
    """The host pipeline's chunks cover 0..B once, in order, none empty; with enough items
    the first and the last are the small B / 16 end chunks."""
    bounds = _nufft._chunk_bounds(B, chunks)
    assert bounds[0][0] == 0 and bounds[-1][1] == B
    assert all(b > a for a, b in bounds)
    assert all(bounds[i][1] == bounds[i + 1][0] for i in range(len(bounds) - 1))
    if B == 32 and chunks == 4:
        assert [b - a for a, b in bounds] == [2, 7, 7, 7, 7, 2]
    if B == 32 and chunks == 7:
        assert [b - a for a, b in bounds] == [2, 4, 4, 4, 4, 4, 4, 4, 2]
