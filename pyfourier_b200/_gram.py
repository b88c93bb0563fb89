"""Toeplitz Gram operator of the NUFFT: ``plan_spgram``, ``GramMatrix``, ``sparse_gram``.

Mirrors src/pyfourier/_sparsegram/_plan.py:20-270 and
src/pyfourier/_sparsegram/_fwd.py:17-119.  The point-spread function is built
at plan time in float64 -- the adjoint NUFFT of the sample weights at twice the
coordinates on the 2N grid (the reference's construction, _plan.py:201-208,
which runs its complex64 NUFFT) with a float64 spread kernel (pfb_spread_f64)
and complex128 transforms -- then Fourier transformed and stored as complex64
per-voxel K x K matrices (subspace) or per-frame planes.  The apply
(pad -> FFT -> mix -> inverse FFT -> crop) runs in libpfb200.

Intent fixes relative to the shipped reference (whose plan cannot run,
_plan.py:141-147, :201-208, :229-239):
* the per-voxel product is ``out[v] = T[v] @ in[v]`` with
  ``T[v][k2][k1] = FFT(PSF)[k1, k2](v)``; the shipped ``_dot_nb``
  (_bmatvec/_bdot.py:119-127) computes ``in * colsum(T)``;
* ``normalize="reference"`` (default) divides the kernel by the mean of its
  non-zero magnitudes (_plan.py:242) like the reference; ``normalize=None``
  keeps the exact scale, for which ``sparse_gram(x) == A^H W A x`` with
  ``A = nufft(norm=None)`` and ``A^H`` its exact adjoint.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._b0 import mri_exp_approx
from ._plan import _as_tensor, plan_nufft, resolve_device, to_caller


class _GramHandle:
    def __init__(self, ndim, shape, os_shape, ncoeff, lowrank, nseg, kernel, device):
        L = _lib.load()
        self.device = torch.device(device)
        h = ctypes.c_void_p()
        k = kernel.to(self.device, torch.complex64).contiguous()
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream(self.device)
            _lib.check(L.pfb_gram_create(ndim, _lib.int_array(shape), _lib.int_array(os_shape), int(ncoeff),
                                         int(lowrank), int(nseg), ctypes.c_void_p(k.data_ptr()),
                                         self.device.index, ctypes.c_void_p(s.cuda_stream), ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            try:
                with torch.cuda.device(self.device):
                    _lib.load().pfb_gram_destroy(self.handle)
            except Exception:  # pragma: no cover
                pass
            self.handle = None


@dataclass
class GramMatrix:
    """Fields as src/pyfourier/_sparsegram/_plan.py:253-262.

    ``value``: (nvox, K, K) complex64 per-voxel matrices (``islowrank``) or
    (nframes, *os_shape) / (*os_shape) planes, uncentred layout.
    """

    value: object
    shape: tuple
    ndim: int
    islowrank: bool
    zmap_s_kernel: object
    zmap_batch_size: int
    device: object
    image_shape: tuple = None
    _handle: object = None

    def to(self, device):
        device = resolve_device(device, self.device)
        if self.device is None or device != self.device or self._handle is None:
            self.value = self.value.to(device)
            if self.zmap_s_kernel is not None:
                self.zmap_s_kernel = self.zmap_s_kernel.to(device)
            self.device = device
            self._handle = None
        return self

    @property
    def nseg(self):
        return 1 if self.zmap_s_kernel is None else int(self.zmap_s_kernel.shape[0])

    @property
    def ncoeff(self):
        """Image planes per batch item: K (low rank) or frames (elementwise, 1 if none)."""
        if self.islowrank:
            return int(self.value.shape[-1])
        lead = 1 if self.zmap_s_kernel is not None else 0
        return 1 if self.value.ndim == self.ndim + lead else int(self.value.shape[lead])

    def handle(self):
        if self._handle is None:
            self._handle = _GramHandle(self.ndim, self.image_shape, self.shape, self.ncoeff, self.islowrank,
                                       self.nseg, self.value, self.device)
        return self._handle


def _apod64(n, oversamp, width, beta, dev):
    """Deapodisation vector of one axis in float64 (_subroutines/_apod.py:27-41)."""
    os_i = float(np.ceil(np.float32(oversamp) * np.float32(n)))
    i = torch.arange(n, dtype=torch.float64, device=dev)
    a = torch.sqrt(float(beta) ** 2 - (math.pi * int(width) * (i - n // 2) / os_i) ** 2)  # NaN where < 0
    a = a / torch.sinh(a)
    a = a / a[n // 2]
    return torch.nan_to_num(a, nan=1.0)


def _centred(x, nd, inverse, norm):
    axes = tuple(range(-nd, 0))
    f = torch.fft.ifftn if inverse else torch.fft.fftn
    return torch.fft.fftshift(f(torch.fft.ifftshift(x, dim=axes), dim=axes, norm=norm), dim=axes)


def _psf_f64(vals, pplan, os_shape, basis):
    """The Toeplitz PSF in float64: adjoint NUFFT of the per-sample values on the
    PSF plan, cropped to ``os_shape`` (the 2N grid).

    vals (L, total samples) complex128 in the plan's sample order.  The spread
    runs in libpfb200 in float64 (pfb_spread_f64) into per-frame grids; with a
    basis (F, K) the subspace projection of the reference (delta[k1, f] =
    basis[f, k1] spread with conj(basis[f, k2]), _noncart2cart/_2D_subspace.py:49-53)
    follows by linearity: P[l, k1, k2] = sum_f basis[f, k1] conj(basis[f, k2]) G[l, f].
    Division by the kernel scale, the centred inverse FFT (norm None), the crop
    and the deapodisation follow _nufft/_nufft.py:254-287, in complex128.
    Returns (L, K, K, *os_shape) or (L, F, *os_shape)."""
    dev = pplan.device
    nd = pplan.ndim
    it = pplan.interpolator
    Ls = vals.shape[0]
    grid = torch.zeros((Ls, it.nframes, *pplan.os_shape), dtype=torch.complex128, device=dev)
    v = vals.to(dev, torch.complex128).contiguous()
    with torch.cuda.device(dev):
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(_lib.load().pfb_spread_f64(it.handle, ctypes.c_void_p(v.data_ptr()), int(Ls),
                                              ctypes.c_void_p(grid.data_ptr()), st))
    grid = grid / it.scale
    if basis is not None:
        b = basis.to(dev, torch.complex128)
        grid = torch.einsum("fa,fb,lf...->lab...", b, b.conj(), grid)
    x = _centred(grid, nd, True, "backward")
    # centred crop to os_shape (_subroutines/_resize.py:23-42)
    sl = [slice(None)] * (x.ndim - nd)
    for i, o in zip(x.shape[-nd:], os_shape):
        s0 = max(i // 2 - o // 2, 0)
        sl.append(slice(s0, s0 + min(i, o)))
    x = x[tuple(sl)]
    for n in range(1, nd + 1):
        ax = -n
        if int(pplan.width[ax]) != 1:
            a = _apod64(x.shape[ax], pplan.oversamp[ax], pplan.width[ax], pplan.beta[ax], dev)
            x = x * a.reshape([x.shape[ax]] + [1] * (n - 1))
    return x


def plan_spgram(coord, shape, basis=None, zmap=None, L=6, nbins=(40, 40), dt=None, T=None,
                L_batch_size=None, weight=None, oversamp=None, width=6, device="cpu",
                normalize="reference"):
    """Toeplitz kernel of A^H W A (src/pyfourier/_sparsegram/_plan.py:20-249).

    With a field map (:162-182) there is one kernel per time segment l, built
    from the sample weights B_l(t), and the apply is sum_l conj(C_l) G_l(C_l x)
    (_sparsegram/_sparsegram.py:26-53); B and C are fitted over the pair
    histogram of the field map (``mri_exp_approx(..., acorr=True)``), which is
    what the Gram's pairwise phase exp(-(z(r') + conj(z(r))) t) needs.
    """
    coord_t = _as_tensor(coord, torch.float32)
    dev = resolve_device(device, coord_t.device)
    coord_t = coord_t.to(dev)
    ndim = coord_t.shape[-1]
    shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in list(shape)[-ndim:]]
    # Cartesian axes stay at osf 1 (_plan.py:185-192)
    n_xyz = shape[::-1]
    is_cart = [bool(torch.allclose(n_xyz[ax] * coord_t[..., ax], torch.round(n_xyz[ax] * coord_t[..., ax])))
               for ax in range(ndim)][::-1]
    osf = np.asarray([1.0 if c else 2.0 for c in is_cart], np.float32)
    os_shape = [int(np.ceil(np.float32(o) * np.float32(n))) for n, o in zip(shape, osf)]
    if weight is None:
        wgt = torch.ones(coord_t.shape[:-1], dtype=torch.float32, device=dev)
    else:
        wgt = _as_tensor(weight).to(dev, torch.float32)
    basis_t = _as_tensor(basis).to(dev, torch.complex64) if basis is not None else None
    vals = wgt.to(torch.complex128)[None]  # (L = 1, ...)
    zs = None
    if zmap is not None:
        if T is None:
            if dt is None:
                raise ValueError("Please provide raster time dt if T is not known")
            T = dt * np.arange(coord_t.shape[-2], dtype=np.float32)
        bt, zs = mri_exp_approx(_as_tensor(zmap).to(dev), T, L, nbins, acorr=True)
        # segment l weights each sample by B_l(t) of its readout position (last axis)
        bl = torch.as_tensor(bt, dtype=torch.complex128, device=dev)
        vals = vals * bl.reshape(L, *([1] * (vals.ndim - 2)), bl.shape[-1])
        zs = zs.to(torch.complex64).contiguous()
    scale_xyz = torch.as_tensor(osf[::-1].copy(), device=dev)
    pplan = plan_nufft(coord_t * scale_xyz, os_shape, width=width, oversamp=1.25, device=dev)
    psf = _psf_f64(vals.reshape(vals.shape[0], -1), pplan, os_shape, basis_t)
    if normalize is None:
        G_os = float(np.prod(pplan.os_shape))
        Tk = _centred(psf * G_os, ndim, False, "backward")
    else:
        Tk = _centred(psf, ndim, False, "ortho")
    axes = tuple(range(-ndim, 0))
    nlead = 1 if zs is not None else 0
    if not nlead:
        Tk = Tk[0]
    if basis_t is None and Tk.ndim > ndim + nlead and Tk.shape[nlead] == 1:
        Tk = Tk[:, 0] if nlead else Tk[0]
    Tk = torch.fft.ifftshift(Tk, dim=axes)
    if basis_t is not None:
        K = basis_t.shape[1]
        Tk = Tk.reshape(-1, K, K, int(np.prod(os_shape))).permute(0, 3, 2, 1)  # (L, nvox, k2, k1)
        Tk = Tk if nlead else Tk[0]
    if normalize == "reference":
        Tk = Tk / torch.mean(torch.abs(Tk[Tk != 0]))
    elif normalize is not None:
        raise ValueError("normalize must be 'reference' or None")
    Tk = torch.nan_to_num(Tk).to(torch.complex64).contiguous()
    return GramMatrix(Tk, tuple(os_shape), ndim, basis_t is not None, zs, L_batch_size, dev,
                      image_shape=tuple(shape))


def _gram_core(gm: GramMatrix, x):
    """x (B, C, *shape) complex64 on gm.device -> same."""
    L = _lib.load()
    h = gm.handle()
    B = x.shape[0]
    out = torch.empty_like(x)
    if B == 0:
        return out
    n = ctypes.c_size_t()
    _lib.check(L.pfb_gram_workspace_size(h.handle, B, ctypes.byref(n)))
    ws = torch.empty(int(n.value), dtype=torch.uint8, device=gm.device)
    st = ctypes.c_void_p(torch.cuda.current_stream(gm.device).cuda_stream)
    zs = gm.zmap_s_kernel
    zp = ctypes.c_void_p(zs.data_ptr()) if zs is not None else None
    _lib.check(L.pfb_gram_apply(h.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), B,
                                zp, ctypes.c_void_p(ws.data_ptr()), ws.numel(), st))
    return out


class SparseGramFunction(torch.autograd.Function):
    """Self-adjoint: backward applies the same operator (_sparsegram/_fwd.py:104-119)."""

    @staticmethod
    def forward(fctx, x, gm):
        fctx.gm = gm
        return _gram_core(gm, x.contiguous())

    @staticmethod
    def backward(fctx, g):
        return _gram_core(fctx.gm, g.contiguous().to(torch.complex64)), None


def sparse_gram(image, gram_matrix, norm=None, device="cpu", threadsperblock=128):
    """Apply the Toeplitz Gram (src/pyfourier/_sparsegram/_fwd.py:17-84).

    image: (..., [ncoeff or ncontrasts], *shape); returned in its dtype and on its device.
    ``norm`` does not change the result (the forward and inverse FFT scalings
    always multiply to 1/prod(os_shape)).
    """
    if norm not in (None, "ortho", "backward", "forward"):
        raise ValueError(f"unknown norm {norm!r}")
    as_numpy = isinstance(image, np.ndarray)
    x_t = _as_tensor(image)
    idevice = x_t.device
    dtype = x_t.dtype
    dev = resolve_device(device, idevice)
    gm = gram_matrix.to(dev)
    if gm.image_shape is None:
        raise ValueError("GramMatrix has no image shape")
    nd = gm.ndim
    C = gm.ncoeff
    xc = x_t.to(dev)
    xc = xc.to(torch.complex64) if torch.is_complex(xc) else xc.to(torch.float32).to(torch.complex64)
    if tuple(xc.shape[xc.ndim - nd:]) != tuple(gm.image_shape):
        raise ValueError(f"image spatial shape {tuple(xc.shape[xc.ndim - nd:])} != {gm.image_shape}")
    has_c = gm.islowrank or C > 1
    batch_shape = xc.shape[: xc.ndim - nd - (1 if has_c else 0)]
    if has_c and xc.shape[-nd - 1] != C:
        raise ValueError(f"image needs an axis of size {C} before the spatial axes")
    B = int(np.prod(batch_shape)) if len(batch_shape) else 1
    y = SparseGramFunction.apply(xc.reshape(B, C, *gm.image_shape), gm)
    y = y.reshape(xc.shape)
    if not torch.is_complex(torch.empty((), dtype=dtype)):
        y = y.real
    y = to_caller(y, idevice, dtype)
    return y.detach().numpy() if as_numpy else y
