"""Forward / adjoint NUFFT operators and their autograd forms.

Public functions mirror src/pyfourier/_nufft/_fwd.py:18-230 (``nufft``) and
src/pyfourier/_nufft/_adj.py:18-216 (``nufft_adj``): same arguments,
defaults and shape conventions.  The work runs in libpfb200 (sm_100a CUDA +
cuFFT); nothing here computes on the CPU.

Layouts handed to the library: images (B, C, *shape) and k-space (B, total
samples), complex64, contiguous on the plan's device.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._plan import NUFFTPlan, _as_tensor, plan_nufft, resolve_device, to_caller


def norm_code(norm):
    if norm is None:
        return _lib.PFB_NORM_NONE
    if norm == "ortho":
        return _lib.PFB_NORM_ORTHO
    raise ValueError(f"norm must be None or 'ortho', got {norm!r}")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class _Ctx:
    """Everything an apply needs besides the data: plan, basis, B0 chunk, weight."""

    def __init__(self, plan: NUFFTPlan, basis, weight_ps, norm):
        self.plan = plan
        self.interp = plan.interpolator
        self.dev = plan.device
        self.basis = basis
        self.weight = weight_ps
        self.norm = norm
        self.nframes = self.interp.nframes
        self.C = basis.shape[1] if basis is not None else self.nframes
        self.G = float(np.prod(plan.os_shape))
        s = self.interp.scale
        self.fac_fwd = (1.0 / s) / (math.sqrt(self.G) if norm == _lib.PFB_NORM_ORTHO else 1.0)
        self.fac_adj = (1.0 / s) / (math.sqrt(self.G) if norm == _lib.PFB_NORM_ORTHO else self.G)

    def segments(self):
        """Yield (start, stop) chunks of B0 segments ((0, 1) without a field map)."""
        p = self.plan
        if p.zmap_s_kernel is None:
            yield 0, 1
            return
        Lseg = p.zmap_s_kernel.shape[0]
        step = p.zmap_batch_size or Lseg
        for start in range(0, Lseg, step):
            yield start, min(Lseg, start + step)

    def opts(self, batch, seg, flags=0):
        o = _lib.ApplyT()
        o.batch = int(batch)
        o.ncoeff = int(self.C)
        o.basis = self.basis.data_ptr() if self.basis is not None else None
        o.weight = self.weight.data_ptr() if self.weight is not None else None
        p = self.plan
        if p.zmap_s_kernel is not None:
            start, stop = seg
            o.nseg = stop - start
            o.b0_time = p.zmap_t_kernel[start:stop].data_ptr()
            o.b0_space = p.zmap_s_kernel[start:stop].data_ptr()
        else:
            o.nseg = 1
        o.norm = self.norm
        o.flags = flags
        return o

    def workspace(self, opts):
        """Workspace of the fastest path for these apply options (caching allocator)."""
        n = ctypes.c_size_t()
        _lib.check(_lib.load().pfb_apply_workspace_size(self.interp.handle, ctypes.byref(opts), ctypes.byref(n)))
        return torch.empty(max(int(n.value), 1), dtype=torch.uint8, device=self.dev)


def fwd_core(ctx: _Ctx, image):
    """image (B, C, *shape) complex64 -> kspace (B, total) complex64."""
    L = _lib.load()
    B = image.shape[0]
    out = torch.empty((B, ctx.interp.total_samples), dtype=torch.complex64, device=ctx.dev)
    if B == 0 or out.numel() == 0:
        return out.zero_()
    st = _stream(ctx.dev)
    for i, seg in enumerate(ctx.segments()):
        o = ctx.opts(B, seg, 0 if i == 0 else _lib.PFB_FLAG_ACCUMULATE)
        ws = ctx.workspace(o)
        _lib.check(L.pfb_nufft_fwd(ctx.interp.handle, ctypes.byref(o), _ptr(image), _ptr(out),
                                   _ptr(ws), ws.numel(), st))
    return out


def adj_core(ctx: _Ctx, kspace):
    """kspace (B, total) complex64 -> image (B, C, *shape) complex64."""
    L = _lib.load()
    B = kspace.shape[0]
    out = torch.empty((B, ctx.C, *ctx.plan.shape), dtype=torch.complex64, device=ctx.dev)
    if B == 0:
        return out
    if ctx.interp.total_samples == 0:
        return out.zero_()
    st = _stream(ctx.dev)
    for i, seg in enumerate(ctx.segments()):
        o = ctx.opts(B, seg, 0 if i == 0 else _lib.PFB_FLAG_ACCUMULATE)
        ws = ctx.workspace(o)
        _lib.check(L.pfb_nufft_adj(ctx.interp.handle, ctypes.byref(o), _ptr(kspace), _ptr(out),
                                   _ptr(ws), ws.numel(), st))
    return out


def traj_grad_core(ctx: _Ctx, image_side, values, factor):
    """d/dk of sum_b Re(<values_b, Interp(H_b)>), H = FFT(pad(apod * factor * image_side)).

    image_side (B, C, *shape); values (B, total).  Returns (total, ndim) float32
    in coordinate units.  Weights are recomputed from the plan coordinates.
    """
    L = _lib.load()
    B = image_side.shape[0]
    grad = torch.zeros((ctx.interp.total_samples, ctx.interp.ndim), dtype=torch.float32, device=ctx.dev)
    if B == 0 or grad.numel() == 0:
        return grad
    st = _stream(ctx.dev)
    for seg in ctx.segments():
        o = ctx.opts(B, seg, _lib.PFB_FLAG_ACCUMULATE)
        ws = ctx.workspace(o)
        _lib.check(L.pfb_nufft_traj_grad(ctx.interp.handle, ctypes.byref(o), _ptr(image_side), _ptr(values),
                                         ctypes.c_void_p(grad.data_ptr()), ctypes.c_float(factor), _ptr(ws),
                                         ws.numel(), st))
    return grad


class NUFFTFunction(torch.autograd.Function):
    """y = A(k) x.  Backward: image gradient by the hand-written adjoint (scaled to be
    the exact adjoint for either norm), trajectory gradient by the analytic
    Kaiser-Bessel derivative kernel (weights recomputed, nothing stored)."""

    @staticmethod
    def forward(fctx, image, coord, ctx):
        fctx.ctx = ctx
        fctx.coord_shape = coord.shape if coord is not None else None
        if coord is not None and coord.requires_grad:
            fctx.save_for_backward(image)
        return fwd_core(ctx, image.contiguous())

    @staticmethod
    def backward(fctx, gy):
        ctx = fctx.ctx
        gy = gy.contiguous().to(torch.complex64)
        gimg = gcoord = None
        if fctx.needs_input_grad[0]:
            gimg = adj_core(ctx, gy)
            if ctx.norm == _lib.PFB_NORM_NONE:
                gimg = gimg * ctx.G  # exact adjoint of the unnormalised forward
        if fctx.needs_input_grad[1]:
            (image,) = fctx.saved_tensors
            g = traj_grad_core(ctx, image.contiguous(), gy, ctx.fac_fwd)
            gcoord = g.reshape(fctx.coord_shape)
        return gimg, gcoord, None


class NUFFTAdjointFunction(torch.autograd.Function):
    """x = A(k)^H y (with nufft_adj's normalisation)."""

    @staticmethod
    def forward(fctx, kspace, coord, ctx):
        fctx.ctx = ctx
        fctx.coord_shape = coord.shape if coord is not None else None
        if coord is not None and coord.requires_grad:
            fctx.save_for_backward(kspace)
        return adj_core(ctx, kspace.contiguous())

    @staticmethod
    def backward(fctx, gx):
        ctx = fctx.ctx
        gx = gx.contiguous().to(torch.complex64)
        gk = gcoord = None
        if fctx.needs_input_grad[0]:
            gk = fwd_core(ctx, gx)
            if ctx.norm == _lib.PFB_NORM_NONE:
                gk = gk / ctx.G
        if fctx.needs_input_grad[1]:
            (kspace,) = fctx.saved_tensors
            g = traj_grad_core(ctx, gx, kspace.contiguous(), ctx.fac_adj)
            gcoord = g.reshape(fctx.coord_shape)
        return gk, gcoord, None


# --------------------------------------------------------------------------------------
# argument handling shared by nufft / nufft_adj
# --------------------------------------------------------------------------------------
def _prep_basis(basis, dev):
    if basis is None:
        return None
    b = _as_tensor(basis)
    return b.to(dev, torch.complex64).contiguous()


def _sample_shape(interp):
    if interp.dshape is None:
        return (interp.total_samples,)
    return ((interp.nframes,) if interp.nframes > 1 else ()) + interp.dshape


def _split_weight(weight, sample_shape, dev):
    """Per-sample real weights go to the kernels; anything else is applied with torch."""
    if weight is None:
        return None, None
    w = _as_tensor(weight)
    w = w.to(dev)
    if not torch.is_complex(w):
        w = w.to(torch.float32)
        lead = w.ndim - len(sample_shape)
        ws = w.reshape(w.shape[max(lead, 0):]) if lead <= 0 or all(s == 1 for s in w.shape[:lead]) else None
        if ws is not None:
            try:
                ws = torch.broadcast_to(ws, sample_shape).reshape(-1).contiguous()
                return ws, None
            except RuntimeError:
                pass
    else:
        w = w.to(torch.complex64)
    return None, w


def _to_compute(x, dev):
    x = _as_tensor(x)
    if x.dtype in (torch.float16, torch.float32, torch.float64, torch.bfloat16):
        xc = x.to(dev, torch.float32).to(torch.complex64)
    else:
        xc = x.to(dev, torch.complex64)
    return x, xc


def _finish(out, dtype, idevice, as_numpy):
    if not torch.is_complex(torch.empty((), dtype=dtype)):
        out = out.real
    out = to_caller(out, idevice, dtype)
    return out.detach().numpy() if as_numpy else out


# Host inputs of at least this many bytes are processed in batch chunks whose
# host->device copy, compute and device->host copy overlap (three streams).  The
# forward is copy-bound and takes more, smaller chunks (a shorter first copy and last
# read-back); the adjoint is compute-bound and keeps chunks large enough for its
# spread to stay efficient (3D radial, 32 coils of 8 M samples: forward 55.6 ms with
# 8 chunks against 58.6 ms with 4; adjoint 68.8 ms with 4 against 99.2 ms with 8).
# The first and the last chunk run alone (their host->device copy, their compute and
# read-back), so they are small: B / 16 items each, the rest in CHUNKS even chunks (an
# adjoint chunk computes in about the same time for 1 to 8 coils; 32 coils: chunks 2,
# 7, 7, 7, 7, 2 ran 53.9 ms against 58.0 ms for 4, 8, 8, 8, 4).
_HOST_PIPELINE_MIN_BYTES = 64 << 20
_HOST_PIPELINE_CHUNKS_FWD = 7
_HOST_PIPELINE_CHUNKS_ADJ = 4
_HOST_PIPELINE_END = 1.0 / 16
_HOST_PIPELINE_SHIFT = True


def _host_pipelined(t, grad_coord):
    """A CPU complex64 input without autograd history takes the chunked host path."""
    return (t.device.type == "cpu" and t.dtype == torch.complex64 and not t.requires_grad and grad_coord is None
            and t.numel() * 8 >= _HOST_PIPELINE_MIN_BYTES)


def _chunk_bounds(B, chunks):
    """Batch ranges of the host pipeline: with _HOST_PIPELINE_SHIFT set, a first and a
    last chunk of B x _HOST_PIPELINE_END items (at least one; their host->device copy
    and read-back are the ones that run alone) and the rest in ``chunks`` even chunks:
    32 in 7 gives 2, 4, 4, 4, 4, 4, 4, 4, 2 and 32 in 4 gives 2, 7, 7, 7, 7, 2.
    Otherwise ``chunks`` even chunks."""
    n = max(1, min(B, chunks))
    e = max(1, int(round(_HOST_PIPELINE_END * B)))
    if _HOST_PIPELINE_SHIFT and n >= 2 and B - 2 * e >= n:
        mid = B - 2 * e
        edges = [0] + [e + mid * j // n for j in range(n + 1)] + [B]
    else:
        edges = [B * j // n for j in range(n + 1)]
    return [(a, b) for a, b in zip(edges[:-1], edges[1:]) if b > a]


def _pipeline(xh, run, out_tail, dev, chunks):
    """Apply ``run`` (device (b, ...) complex64 -> device (b, *out_tail) complex64, on the
    current stream) to a CPU batch ``xh`` (B, ...) in up to ``chunks`` chunks:
    chunk j + 1 is copied to the device on one stream and chunk j - 1's result copied back
    on another while chunk j computes.  Pageable inputs are staged chunk by chunk through
    page-locked buffers.  Returns a page-locked CPU tensor (B, *out_tail)."""
    B = xh.shape[0]
    out = torch.empty((B, *out_tail), dtype=torch.complex64, pin_memory=True)
    bounds = _chunk_bounds(B, chunks)
    pinned = xh.is_pinned()
    with torch.cuda.device(dev):
        comp = torch.cuda.current_stream(dev)
        h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        h2d.wait_stream(comp)
        for b0, b1 in bounds:
            src = xh[b0:b1]
            if not pinned:
                stage = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
                stage.copy_(src)
                src = stage
            with torch.cuda.stream(h2d):
                xd = torch.empty(src.shape, dtype=torch.complex64, device=dev)
                xd.copy_(src, non_blocking=True)
            comp.wait_stream(h2d)
            xd.record_stream(comp)
            yd = run(xd)
            d2h.wait_stream(comp)
            with torch.cuda.stream(d2h):
                out[b0:b1].copy_(yd, non_blocking=True)
            yd.record_stream(d2h)
        d2h.synchronize()
    return out


def nufft(image, coord=None, shape=None, nufft_plan=None, basis=None, zmap=None, L=6, nbins=(40, 40),
          dt=None, T=None, L_batch_size=None, weight=None, norm=None, device="cpu", threadsperblock=128,
          width=4, oversamp=1.25):
    """N-dimensional non-uniform FFT (src/pyfourier/_nufft/_fwd.py:18-230).

    image: (..., ncontrasts, ny, nx) or (..., ncontrasts, nz, ny, nx)
    (the contrast axis is present when the trajectory has several frames or a
    subspace ``basis`` (ncontrasts, ncoeff) is given; it then holds ncoeff).
    Returns k-space (..., [ncontrasts], nviews, nsamples) in image's dtype and
    on image's device.  Computation runs on a CUDA device (``device="cpu"``,
    the reference's default, selects the current CUDA device).
    ``threadsperblock`` is accepted for compatibility; launch shapes come from
    the plan's tuning.  Differentiable w.r.t. ``image`` and, when ``coord``
    requires grad, w.r.t. ``coord``.
    """
    as_numpy = isinstance(image, np.ndarray)
    image_t = _as_tensor(image)
    idevice = image_t.device
    dev = resolve_device(device, idevice)
    coord_t = None if coord is None else (coord if isinstance(coord, torch.Tensor) else _as_tensor(coord))
    if nufft_plan is None:
        if coord is None:
            raise ValueError("either coord or nufft_plan is required")
        if shape is None:
            shape = image_t.shape[-coord_t.shape[-1]:]
        nufft_plan = plan_nufft(coord_t.detach(), shape, width, oversamp, zmap, L, nbins, dt, T,
                                L_batch_size, device=dev)
    nufft_plan.to(dev)
    plan = nufft_plan
    ip = plan.interpolator
    nd = plan.ndim
    dtype = image_t.dtype
    c_in = coord_t if (coord_t is not None and coord_t.requires_grad) else None
    host = _host_pipelined(image_t, c_in)
    x = image_t if host else _to_compute(image_t, dev)[1]
    basis_t = _prep_basis(basis, dev)
    has_c = ip.nframes > 1 or basis_t is not None
    C = basis_t.shape[1] if basis_t is not None else ip.nframes
    if tuple(x.shape[x.ndim - nd:]) != tuple(plan.shape):
        raise ValueError(f"image spatial shape {tuple(x.shape[x.ndim - nd:])} != plan shape {plan.shape}")
    if has_c and (x.ndim < nd + 1 or x.shape[-nd - 1] != C):
        raise ValueError(f"image needs a contrast/coefficient axis of size {C} before the spatial axes")
    batch_shape = x.shape[: x.ndim - nd - (1 if has_c else 0)]
    B = int(np.prod(batch_shape)) if len(batch_shape) else 1
    sshape = _sample_shape(ip)
    wps, wfull = _split_weight(weight, sshape, dev)
    ctx = _Ctx(plan, basis_t, wps, norm_code(norm))
    if host and B >= 2 and wfull is None:
        y = _pipeline(x.reshape(B, C, *plan.shape), lambda xd: fwd_core(ctx, xd), (ip.total_samples,), dev,
                      _HOST_PIPELINE_CHUNKS_FWD)
        return _finish(y.reshape(*batch_shape, *sshape), dtype, idevice, as_numpy)
    if host:
        x = _to_compute(x, dev)[1]
    xb = x.reshape(B, C, *plan.shape)
    y = NUFFTFunction.apply(xb, c_in, ctx)
    y = y.reshape(*batch_shape, *sshape)
    if wfull is not None:
        y = wfull * y
    return _finish(y, dtype, idevice, as_numpy)


def nufft_adj(kspace, coord=None, shape=None, nufft_plan=None, basis=None, zmap=None, L=6, nbins=(40, 40),
              dt=None, T=None, L_batch_size=None, weight=None, norm=None, device="cpu", threadsperblock=128,
              width=4, oversamp=1.25):
    """Adjoint non-uniform FFT (src/pyfourier/_nufft/_adj.py:18-216).

    kspace: (..., [ncontrasts], nviews, nsamples) -> image (..., [ncontrasts or
    ncoeff], *shape).  With ``norm=None`` the result is the adjoint scaled by
    1/prod(os_shape), as in the reference.
    """
    as_numpy = isinstance(kspace, np.ndarray)
    k_t = _as_tensor(kspace)
    idevice = k_t.device
    dev = resolve_device(device, idevice)
    coord_t = None if coord is None else (coord if isinstance(coord, torch.Tensor) else _as_tensor(coord))
    if nufft_plan is None:
        if coord is None or shape is None:
            raise ValueError("coord and shape (or nufft_plan) are required")
        nufft_plan = plan_nufft(coord_t.detach(), shape, width, oversamp, zmap, L, nbins, dt, T,
                                L_batch_size, device=dev)
    nufft_plan.to(dev)
    plan = nufft_plan
    ip = plan.interpolator
    dtype = k_t.dtype
    c_in = coord_t if (coord_t is not None and coord_t.requires_grad) else None
    host = _host_pipelined(k_t, c_in)
    k = k_t if host else _to_compute(k_t, dev)[1]
    basis_t = _prep_basis(basis, dev)
    has_c = ip.nframes > 1 or basis_t is not None
    C = basis_t.shape[1] if basis_t is not None else ip.nframes
    sshape = _sample_shape(ip)
    if tuple(k.shape[k.ndim - len(sshape):]) != tuple(sshape):
        raise ValueError(f"k-space trailing shape {tuple(k.shape[k.ndim - len(sshape):])} != {sshape}")
    batch_shape = k.shape[: k.ndim - len(sshape)]
    B = int(np.prod(batch_shape)) if len(batch_shape) else 1
    wps, wfull = _split_weight(weight, sshape, dev)
    ctx = _Ctx(plan, basis_t, wps, norm_code(norm))
    if host and B >= 2 and wfull is None:
        x = _pipeline(k.reshape(B, ip.total_samples), lambda kd: adj_core(ctx, kd), (C, *plan.shape), dev,
                      _HOST_PIPELINE_CHUNKS_ADJ)
        x = x.reshape(*batch_shape, *((C,) if has_c else ()), *plan.shape)
        return _finish(x, dtype, idevice, as_numpy)
    if host:
        k = _to_compute(k, dev)[1]
    if wfull is not None:
        k = wfull * k
    kb = k.reshape(B, ip.total_samples)
    x = NUFFTAdjointFunction.apply(kb, c_in, ctx)
    x = x.reshape(*batch_shape, *((C,) if has_c else ()), *plan.shape)
    return _finish(x, dtype, idevice, as_numpy)
