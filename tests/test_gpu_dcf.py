"""GPU: Pipe-Menon density compensation (pfb_pipe_menon_dcf, through
pyfourier_b200.pipe_menon_dcf and the C ABI) against the oracle's restatement of
src/pyfourier/_dcomp/pipemenon.py on the same trajectories.

The reference's iteration w <- w / |A A^H w| is chaotic on oversampled radial
trajectories: started from ones + 1e-6 noise, the oracle itself drifts from its
unperturbed run by O(1) (rel-L2) within about 15 iterations, as the smallest
weights fall towards zero.  So full runs are compared only over iterations where
that drift stays far below the tolerance, and the 30-iteration loop is checked
step by step: for GPU iterates w_k, w_{k+1}, the magnitude w_k / w_{k+1} the GPU
divided by must be the oracle's |A A^H w_k|.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from oracle import nufft_oracle as orc  # noqa: E402
from tests.test_gpu_nufft import radial, rel  # noqa: E402

TOL = 1e-5  # rel-L2 of one iteration (float32 sums in a different order)
TOL_RUN = 1e-4  # rel-L2 of a few iterations run end to end (the per-step differences add up)


def pf():
    import pyfourier_b200

    return pyfourier_b200


def _gpu_iterate(plan, w, niter):
    """niter GPU iterations starting from w (device float32), in place."""
    from pyfourier_b200 import _lib

    L = _lib.load()
    h = plan.interpolator.handle
    n = ctypes.c_size_t()
    _lib.check(L.pfb_dcf_workspace_size(h, ctypes.byref(n)))
    ws = torch.empty(int(n.value), dtype=torch.uint8, device=w.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.pfb_pipe_menon_dcf(h, ctypes.c_void_p(w.data_ptr()), int(niter), ctypes.c_void_p(ws.data_ptr()),
                                    ws.numel(), st))
    torch.cuda.synchronize()
    return w


def _oracle_ghg(plan, w):
    """|A A^H w| of the reference's map (the well-conditioned, linear part of a step)."""
    ghg = orc.nufft_fwd(orc.nufft_adj(w.astype(np.complex64), plan, norm="ortho"), plan, norm="ortho")
    return np.abs(ghg).astype(np.float64)


def _step_error(oplan, wk, wnext):
    """One GPU step w_k -> w_{k+1} against the reference's map: the GPU's implied
    |A A^H w_k| = w_k / w_{k+1} vs the oracle's (comparing the weights themselves
    would divide by near-zero |A A^H w| at late, chaotic iterates)."""
    return rel(wk.astype(np.float64) / wnext.astype(np.float64), _oracle_ghg(oplan, wk))


def test_dcf_2d_radial_default_kernel_first_iterations():
    N = 48
    coord = radial(40, 96, N)
    w = pf().pipe_menon_dcf(torch.as_tensor(coord).cuda(), (N, N), niter=5)
    ref = orc.pipe_menon_dcf(coord, (N, N), niter=5)
    assert w.shape == ref.shape and w.dtype == torch.float32 and w.is_cuda
    assert rel(w, ref) < TOL_RUN


def test_dcf_30_iterations_step_by_step():
    """Each of the 30 GPU iterations applies the reference's map to the GPU's own
    previous iterate."""
    N = 48
    coord = radial(40, 96, N)
    gplan = pf().plan_nufft(torch.as_tensor(coord), (N, N), width=6, oversamp=1.5, device="cuda:0")
    oplan = orc.plan_nufft(coord, (N, N), width=6, oversamp=1.5)
    w = torch.ones(coord.shape[:-1], dtype=torch.float32, device="cuda:0").reshape(-1)
    done = 0
    for k in (10, 20, 29):
        _gpu_iterate(gplan, w, k - done)
        wk = w.cpu().numpy().reshape(coord.shape[:-1])
        nxt = _gpu_iterate(gplan, w.clone(), 1).cpu().numpy().reshape(coord.shape[:-1])
        assert _step_error(oplan, wk, nxt) < TOL, k
        done = k


def test_dcf_3d_and_numpy_roundtrip():
    rng = np.random.default_rng(3)
    N = (20, 22, 24)
    coord = ((rng.random((30, 40, 3)) - 0.5) * np.array(N[::-1])).astype(np.float32)
    w = pf().pipemenon.pipe_menon_dcf(coord, N, niter=8, width=4, oversamp=1.25)
    ref = orc.pipe_menon_dcf(coord, N, niter=8, width=4, oversamp=1.25)
    assert isinstance(w, np.ndarray) and w.shape == ref.shape
    assert rel(w, ref) < TOL_RUN


def test_dcf_multiframe_and_zero_iterations():
    """3 frames of 12 spokes: sparse enough that a 1e-6 perturbation of the start
    grows 200-fold in the first iteration of the reference's loop, so the full
    run is compared after one iteration and a later iterate step by step."""
    N, F = 32, 3
    coord = np.stack([radial(12, 64, N, rot=0.4 * f) for f in range(F)])
    w = pf().pipe_menon_dcf(torch.as_tensor(coord), N, niter=1)
    ref = orc.pipe_menon_dcf(coord, (N, N), niter=1)
    assert w.shape == (F, 12, 64) and w.device.type == "cpu"
    assert rel(w, ref) < TOL
    gplan = pf().plan_nufft(torch.as_tensor(coord), (N, N), width=6, oversamp=1.5, device="cuda:0")
    oplan = orc.plan_nufft(coord, (N, N), width=6, oversamp=1.5)
    w3 = _gpu_iterate(gplan, torch.ones(coord.shape[:-1], dtype=torch.float32, device="cuda:0").reshape(-1), 3)
    w4 = _gpu_iterate(gplan, w3.clone(), 1)
    assert _step_error(oplan, w3.cpu().numpy().reshape(coord.shape[:-1]),
                       w4.cpu().numpy().reshape(coord.shape[:-1])) < TOL
    w0 = pf().pipe_menon_dcf(torch.as_tensor(coord), N, niter=0)
    assert torch.equal(w0, torch.ones_like(w0))


def test_repeated_calls_reuse_pooled_plan_memory():
    """Each call builds and destroys a plan; its device memory comes back from the
    library's pool, so back-to-back calls do not grow the device's footprint, give
    the same weights, and the kept blocks can be handed back.  One iteration: the
    chaotic iteration amplifies the float-atomic ordering of the crowded tiles
    (about 1e-3 after three iterations on this trajectory)."""
    P = pf()
    bench = pytest.importorskip("bench")
    coord = bench.golden_means_radial_3d(3000, 128, 64)
    w0 = P.pipe_menon_dcf(coord, 64, niter=1, device="cuda:0")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        w = P.pipe_menon_dcf(coord, 64, niter=1, device="cuda:0")
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert abs(free1 - free0) < (32 << 20), (free0, free1)
    assert rel(w, w0) < TOL
    P.release_cached_memory("cuda:0")
    assert torch.cuda.mem_get_info(0)[0] >= free1
