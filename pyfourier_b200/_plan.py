"""NUFFT planning: ``plan_nufft``, ``NUFFTPlan`` and the device ``Interpolator``.

Mirrors src/pyfourier/_nufft/_plan.py:20-225 and the Interpolator of
src/pyfourier/_subroutines/_grid/_plan.py:14-114.  The reference precomputes
per-sample index/value tables on the CPU; here the plan is a device object of
libpfb200 (bin-sorted oversampled-grid coordinates and tile offsets), and the
Kaiser-Bessel weights are recomputed in every apply.  ``Interpolator.index`` /
``.value`` materialise the reference's tables on request.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._b0 import mri_exp_approx


def _as_tensor(x, dtype=None):
    if isinstance(x, torch.Tensor):
        return x if dtype is None else x.to(dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype)


def release_cached_memory(device=None):
    """Hand the device memory kept from destroyed plans back to the driver (plans
    allocate from a pool that keeps it for the next plan); synchronises the device."""
    dev = resolve_device(device)
    _lib.check(_lib.load().pfb_release_cached_memory(int(dev.index)))


def resolve_device(device, fallback=None):
    """Map the reference's device argument ("cpu", "cuda:n", -1, n, None) to a CUDA device.

    The library computes on CUDA only.  ``"cpu"`` / ``-1`` (the reference's
    default) and ``None`` select ``fallback`` when it is a CUDA device, else the
    current CUDA device; results are returned on the caller's device.
    """
    if not torch.cuda.is_available():
        raise RuntimeError("pyfourier_b200 needs a CUDA device (no CPU fallback)")
    if isinstance(device, torch.device):
        device = str(device)
    if isinstance(device, str) and device.startswith("cuda"):
        return torch.device(device if ":" in device else f"cuda:{torch.cuda.current_device()}")
    if isinstance(device, int) and device >= 0:
        return torch.device(f"cuda:{device}")
    if fallback is not None and torch.device(fallback).type == "cuda":
        return torch.device(fallback)
    return torch.device(f"cuda:{torch.cuda.current_device()}")


def to_caller(t, idevice, dtype=None):
    """Move a result computed on the GPU to the caller's device, in ``dtype``.

    A result for a CPU caller is copied into page-locked host memory taken from
    torch's caching host allocator (reused from the second call on, so no fresh
    pages are faulted in per call) with an asynchronous copy, then the stream is
    synchronised: the transfer runs at the link's pinned-memory bandwidth instead
    of through the driver's pageable staging.  Results that carry autograd history
    take the ordinary differentiable ``.to`` path.
    """
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    idevice = torch.device(idevice)
    if idevice.type != "cpu" or t.device.type != "cuda" or (t.requires_grad and torch.is_grad_enabled()):
        return t.to(idevice)
    t = t.contiguous()
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    with torch.cuda.device(t.device):
        out.copy_(t, non_blocking=True)
        torch.cuda.current_stream(t.device).synchronize()
    return out


def beta_f32(width, oversamp):
    """Kaiser-Bessel beta of src/pyfourier/_nufft/_plan.py:128 (int16 width, float32 osf)."""
    w = np.asarray(width, dtype=np.int16)
    o = np.asarray(oversamp, dtype=np.float32)
    return (np.pi * (((w / o) * (o - 0.5)) ** 2 - 0.8) ** 0.5).astype(np.float32)


def oversamp_shape(shape, oversamp):
    """ceil(osf * N) in float32 (the intent of _subroutines/_utils/_common.py:16-18)."""
    return [int(np.ceil(np.float32(o) * np.float32(n))) for n, o in zip(shape, oversamp)]


class Interpolator:
    """Device plan of one trajectory (owner of a ``pfb_plan`` handle).

    Attributes follow the reference's Interpolator: ``dshape`` (sample shape
    per frame), ``ishape`` (oversampled grid shape, (z, y, x)), ``scale``,
    ``ndim``, ``device``; plus ``nframes``, ``frame_offsets`` and
    ``readout_len``.
    """

    def __init__(self, coord, frame_offsets, readout_len, dshape, shape, os_shape, width, beta,
                 is_cart, device, tile=None):
        self._handle = None
        self.ndim = int(coord.shape[-1])
        self.dshape = tuple(dshape) if dshape is not None else None
        self.ishape = tuple(int(s) for s in os_shape)
        self.shape = tuple(int(s) for s in shape)
        self.width = tuple(int(w) for w in width)
        self.beta = tuple(float(b) for b in beta)
        self.is_cart = tuple(bool(c) for c in is_cart)
        self.nframes = len(frame_offsets) - 1
        self.frame_offsets = tuple(int(o) for o in frame_offsets)
        self.readout_len = int(readout_len)
        self.total_samples = self.frame_offsets[-1]
        self.device = torch.device(device)
        self._coord = coord  # float32 (total, ndim) on device, kept for rebuilds
        self._tile = tile
        self._build()

    def _build(self):
        L = _lib.load()
        nd = self.ndim
        offs = (ctypes.c_int64 * (self.nframes + 1))(*self.frame_offsets)
        tile = _lib.int_array(self._tile) if self._tile is not None else None
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device)
            c = self._coord.to(self.device, torch.float32).contiguous()
            _lib.check(L.pfb_plan_create(
                ctypes.c_void_p(c.data_ptr()), nd, self.nframes, offs, self.readout_len,
                _lib.int_array(self.shape), _lib.int_array(self.ishape), _lib.int_array(self.width),
                _lib.float_array(self.beta), _lib.int_array([int(v) for v in self.is_cart]), tile,
                self.device.index, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        self._handle = h
        info = _lib.PlanInfoT()
        _lib.check(L.pfb_plan_info(h, ctypes.byref(info)))
        self.scale = float(info.scale)
        self.n_items = int(info.n_items)
        self.max_bin = int(info.max_bin)
        self.tile = tuple(int(info.tile[i]) for i in range(nd))
        # tile t of an axis covers [t * tile - offset, (t + 1) * tile - offset) of the grid
        self.tile_offset = tuple(int(info.tile_offset[i]) for i in range(nd))

    @property
    def handle(self):
        return self._handle

    def to(self, device):
        device = torch.device(device)
        if device.type != "cuda":
            return self
        if device != self.device:
            self._destroy()
            self.device = device
            self._build()
        return self

    def check(self):
        """Raise RuntimeError if a kernel of this plan's applies gave up a bounded
        wait since the last check (those results are invalid).  Synchronises the
        device's current stream."""
        s = torch.cuda.current_stream(self.device)
        _lib.check(_lib.load().pfb_plan_check(self._handle, ctypes.c_void_p(s.cuda_stream)))

    def retile(self, tile):
        """Rebuild the device plan with another tile extent ((z, y, x) order)."""
        tile = tuple(int(t) for t in tile)
        if len(tile) != self.ndim:
            raise ValueError("tile needs one extent per axis")
        if self._handle is not None and tuple(self._tile or ()) == tile:
            return self
        old = self._tile
        self._destroy()
        self._tile = tile
        try:
            self._build()
        except Exception:
            self._tile = old
            self._build()
            raise
        return self

    def set_tuning(self, spread_threads=0, interp_threads=0, spread_channels=0, chunk=None):
        L = _lib.load()
        _lib.check(L.pfb_plan_set_tuning(self._handle, int(spread_threads), int(interp_threads),
                                         int(spread_channels)))
        if chunk is not None:
            with torch.cuda.device(self.device):
                _lib.check(L.pfb_plan_set_chunk(self._handle, int(chunk)))

    def tables(self, axis):
        """Reference tables of one axis ((z, y, x) order): (index int32, value float32)
        shaped (nframes, samples per frame, width) for equal-length frames, else (total, width)."""
        L = _lib.load()
        w = self.width[axis] if not self.is_cart[axis] else 1
        idx = torch.empty((self.total_samples, w), dtype=torch.int32, device=self.device)
        val = torch.empty((self.total_samples, w), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream(self.device)
            _lib.check(L.pfb_plan_tables(self._handle, axis, ctypes.c_void_p(idx.data_ptr()),
                                         ctypes.c_void_p(val.data_ptr()), ctypes.c_void_p(s.cuda_stream)))
        lens = np.diff(self.frame_offsets)
        if len(set(lens.tolist())) == 1:
            idx = idx.reshape(self.nframes, -1, w)
            val = val.reshape(self.nframes, -1, w)
        return idx, val

    @property
    def index(self):
        return tuple(self.tables(a)[0] for a in range(self.ndim))

    @property
    def value(self):
        return tuple(self.tables(a)[1] for a in range(self.ndim))

    def _destroy(self):
        if self._handle is not None and _lib._lib is not None:
            try:
                with torch.cuda.device(self.device):
                    _lib.load().pfb_plan_destroy(self._handle)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
        self._handle = None

    def __del__(self):
        self._destroy()


@dataclass
class NUFFTPlan:
    """Fields as src/pyfourier/_nufft/_plan.py:203-215."""

    ndim: int
    oversamp: tuple
    width: tuple
    beta: tuple
    os_shape: tuple
    shape: tuple
    interpolator: Interpolator
    zmap_t_kernel: object
    zmap_s_kernel: object
    zmap_batch_size: int
    device: object

    def to(self, device):
        device = resolve_device(device, self.device)
        if self.device is None or device != self.device:
            self.interpolator = self.interpolator.to(device)
            if self.zmap_s_kernel is not None:
                self.zmap_t_kernel = self.zmap_t_kernel.to(device)
                self.zmap_s_kernel = self.zmap_s_kernel.to(device)
            self.device = device
        return self


def _frames_from_coord(coord):
    """(coord_flat (total, ndim), frame_offsets, readout_len, dshape) for one coord array
    or a list of per-frame arrays (frames of uneven length)."""
    if isinstance(coord, (list, tuple)):
        parts = [_as_tensor(c, torch.float32) for c in coord]
        nd = parts[0].shape[-1]
        flat = [p.reshape(-1, nd) for p in parts]
        offs = np.concatenate([[0], np.cumsum([f.shape[0] for f in flat])]).astype(np.int64)
        readout = int(parts[0].shape[-2]) if parts[0].ndim >= 2 else int(flat[0].shape[0])
        return torch.cat(flat, 0), offs, readout, None
    coord = _as_tensor(coord, torch.float32)
    nd = coord.shape[-1]
    cs = list(coord.shape[:-1])
    while len(cs) < 3:
        cs = [1] + cs
    nframes = cs[0]
    per = int(np.prod(cs[1:]))
    offs = (np.arange(nframes + 1) * per).astype(np.int64)
    dshape = tuple(coord.shape[-3:-1]) if coord.ndim >= 3 else tuple(coord.shape[-2:-1])
    readout = int(coord.shape[-2])
    return coord.reshape(-1, nd), offs, readout, dshape


def plan_nufft(coord, shape, width=4, oversamp=1.25, zmap=None, L=6, nbins=(40, 40), dt=None,
               T=None, L_batch_size=None, device=None, tile=None, autotune_batch=None):
    """Precompute a NUFFT plan (src/pyfourier/_nufft/_plan.py:20-199).

    ``coord``: (ncontrasts, nviews, nsamples, ndim), (nviews, nsamples, ndim)
    or (nsamples, ndim) in cycles/FOV, axes (x, y, z); or a list of per-frame
    arrays with different numbers of samples.  ``shape``/``width``/``oversamp``
    are (z, y, x).  Coordinates in [-N/2, N/2) are used as given (the
    reference's ``normalize_coordinates`` is the identity for them by its
    documented contract).  ``device`` selects the CUDA device of the plan
    (default: coord's device if CUDA, else the current device).  ``tile``
    overrides the tile extent ((z, y, x)); ``autotune_batch=B`` times the tile /
    chunk candidates for B coils and keeps the fastest (cached on disk).
    """
    flat, offs, readout, dshape = _frames_from_coord(coord)
    ndim = int(flat.shape[-1])
    width = np.asarray([width] * ndim if np.isscalar(width) else list(width), np.int16)
    oversamp = np.asarray([oversamp] * ndim if np.isscalar(oversamp) else list(oversamp), np.float32)
    beta = beta_f32(width, oversamp)
    shape = np.asarray([shape] * ndim if np.isscalar(shape) else list(shape)[-ndim:], np.int64)
    dev = resolve_device(device, flat.device)
    flat = flat.to(dev)
    # Cartesian axes (_plan.py:139-146): integer-valued coordinates
    is_cart = [bool(torch.allclose(flat[:, ax], torch.round(flat[:, ax]))) if flat.numel() else False
               for ax in range(ndim)][::-1]
    is_cart = np.asarray(is_cart)
    oversamp[is_cart] = 1.0
    width[is_cart] = 1
    os_shape = oversamp_shape(shape, oversamp)
    interp = Interpolator(flat, offs, readout, dshape, shape, os_shape, width, beta, is_cart, dev,
                          tile=tile)
    zt = zs = None
    if zmap is not None:
        if T is None:
            if dt is None:
                raise ValueError("Please provide raster time dt if T is not known")
            T = dt * np.arange(readout, dtype=np.float32)
        b, c = mri_exp_approx(_as_tensor(zmap).to(dev), T, L, nbins)
        zt = torch.as_tensor(b, dtype=torch.complex64, device=dev).contiguous()
        zs = c.to(torch.complex64).contiguous()
        if L_batch_size is None:
            L_batch_size = L
    plan = NUFFTPlan(ndim, tuple(float(o) for o in oversamp), tuple(int(w) for w in width),
                     tuple(float(b) for b in beta), tuple(os_shape), tuple(int(s) for s in shape),
                     interp, zt, zs, L_batch_size, dev)
    if autotune_batch:
        from ._autotune import autotune

        autotune(plan, batch=int(autotune_batch))
    return plan
