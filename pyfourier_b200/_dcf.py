"""Pipe-Menon density compensation: ``pipe_menon_dcf``.

Mirrors src/pyfourier/_dcomp/pipemenon.py:9-96 (same arguments, defaults and
return shape): starting from ones, ``niter`` times ``w <- w / |A A^H w|`` with
``A`` the NUFFT of a plan built with ``width`` / ``oversamp`` and norm
"ortho" (``_GHG``, :99-115).  The whole loop is one call into libpfb200
(``pfb_pipe_menon_dcf``): every iteration runs on the current CUDA stream with
no host synchronisation in between.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._plan import _as_tensor, plan_nufft, resolve_device


def pipe_menon_dcf(coord, shape, niter=30, threadsperblock=128, device=None, width=6, oversamp=1.5):
    """Pipe-Menon density compensation factors.

    coord: (ncontrasts, nviews, nsamples, ndim) (or fewer leading axes) in
    cycles/FOV, axes (x, y, z); shape: (z, y, x) or a scalar.  Returns float32
    weights of shape ``coord.shape[:-1]`` on coord's device (NumPy in, NumPy out).
    ``threadsperblock`` is accepted for compatibility and not used.
    """
    as_numpy = not isinstance(coord, torch.Tensor)
    coord_t = _as_tensor(coord, torch.float32)
    idevice = coord_t.device
    dev = resolve_device(device, idevice)
    plan = plan_nufft(coord_t.to(dev), shape, width=width, oversamp=oversamp, device=dev)
    L = _lib.load()
    h = plan.interpolator.handle
    w = torch.ones(plan.interpolator.total_samples, dtype=torch.float32, device=dev)
    n = ctypes.c_size_t()
    _lib.check(L.pfb_dcf_workspace_size(h, ctypes.byref(n)))
    ws = torch.empty(int(n.value), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(L.pfb_pipe_menon_dcf(h, ctypes.c_void_p(w.data_ptr()), int(niter), ctypes.c_void_p(ws.data_ptr()),
                                        ws.numel(), st))
    w = w.reshape(coord_t.shape[:-1]).to(idevice)
    return w.cpu().numpy() if as_numpy else w
