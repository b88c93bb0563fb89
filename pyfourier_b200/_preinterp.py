"""GROG (GRAPPA operator gridding) pre-interpolation: ``grog_interp``.

Mirrors src/pyfourier/_preinterp/_grog.py:22-250 (same arguments and returns):
per axis a GRAPPA operator that shifts the coil vectors of a sample by one grid
step is trained on the calibration region (Tikhonov-regularised least squares,
:253-356); fractional powers G^d of the operators for the quantised offsets
d = (i - (n - 1) / 2) / (n - 1) are multiplied into one table of n^ndim operators
(:131-170); every sample is moved to its nearest grid point,
out = in @ G[offset(sample)], and the caller gets the gridded samples, their
grid indexes and 1 / (number of samples on the same grid point).

The operator training and the table (a few thousand nc x nc matrices) are built
in complex128 with torch on the plan's device; the per-sample apply runs in
libpfb200 (``pfb_grog_apply``): samples sorted by operator at plan time, coil
vectors transposed into sorted rows, persistent CTAs walking chunks of rows that
share an operator, transposed back.

Intent fixes relative to the shipped reference:
* the operator helpers take the array backend of the calibration data (the
  shipped ones pass the builtin ``input``, :288, :326, :359);
* the per-sample product is ``in @ G`` (the shipped ``_dot_product``, :406-412,
  computes ``in * colsum(G)``), and in 3D every (batch, sample) row gets its own
  sample's operator (the shipped 3D path treats the sample axis as the batch,
  :205-207);
* the offset quantisation scales by n - 1 (the literal 10 of :175, n = 11 by
  default); 2D operators trained on one calibration slice apply to every
  leading batch item.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._plan import _as_tensor, resolve_device, to_caller


def _operators(calib, ndim, lamda):
    """Per-axis GRAPPA operators in (x, y[, z]) order, complex128 on calib's device
    (_grog.py:253-356): (nz, nc, nc) per calibration slice in 2D, (nc, nc) in 3D."""
    c = calib.to(torch.complex128)
    if c.ndim == 3:
        c = c[:, None]
    c = torch.movedim(c, 0, -1)  # (nz, ny, nx, nc)
    nc = c.shape[-1]
    eye = torch.eye(nc, dtype=c.dtype, device=c.device)

    def train(S, T):
        Sh = S.conj().transpose(-1, -2)
        l0 = lamda * torch.linalg.norm(Sh, dim=(-2, -1)) / nc
        return torch.linalg.solve(Sh @ S + l0[..., None, None] * eye, Sh @ T)

    nz = c.shape[0]
    if ndim == 2:
        gy = train(c[:, :-1].reshape(nz, -1, nc), c[:, 1:].reshape(nz, -1, nc))
        gx = train(c[:, :, :-1].reshape(nz, -1, nc), c[:, :, 1:].reshape(nz, -1, nc))
        return [gx, gy]
    gz = train(c[:-1].reshape(-1, nc), c[1:].reshape(-1, nc))
    gy = train(c[:, :-1].reshape(-1, nc), c[:, 1:].reshape(-1, nc))
    gx = train(c[:, :, :-1].reshape(-1, nc), c[:, :, 1:].reshape(-1, nc))
    return [gx, gy, gz]


def _table(ops, nsteps):
    """G[(iz n + iy) n + ix] = Gx^dx @ Gy^dy (@ Gz^dz) (_grog.py:131-170, :369-396),
    fractional powers through the eigendecomposition (principal branch)."""
    n = 2 * (nsteps // 2) + 1
    d = (torch.arange(n, dtype=torch.float64, device=ops[0].device) - (n - 1) // 2) / (n - 1)

    def powers(A):
        L, V = torch.linalg.eig(A)
        Vi = torch.linalg.inv(V)
        Lp = L[None] ** d.reshape(-1, *([1] * L.ndim)).to(L.dtype)  # (n, ..., nc)
        return (V[None] * Lp[..., None, :]) @ Vi[None]

    P = [powers(o) for o in ops]
    if len(ops) == 2:
        G = P[0][None, :] @ P[1][:, None]  # [iy, ix] = Gx[ix] @ Gy[iy]
        return G.reshape(n * n, *G.shape[2:])
    G = (P[0][None, None, :] @ P[1][None, :, None]) @ P[2][:, None, None]
    return G.reshape(n ** 3, *G.shape[3:])


def _lut(coord, nsteps):
    """indexes = round(coord) (half to even); per axis the step floor((n - 1)(index -
    coord)) + n // 2, combined as sum_a step_a n^a over (x, y, z) (_grog.py:172-182).
    float32 arithmetic throughout."""
    n = 2 * (nsteps // 2) + 1
    c = coord.to(torch.float32)
    idx = torch.round(c)
    st = torch.floor((idx - c) * float(n - 1)).to(torch.int64) + n // 2
    w = torch.tensor([1, n, n * n], dtype=torch.int64, device=c.device)[: c.shape[-1]]
    return idx, (st.reshape(-1, c.shape[-1]) * w).sum(-1)


class GrogPlan:
    """Device state of one GROG interpolation: the operator table and the samples
    sorted by operator (C handle), the grid indexes (clipped) and the weights.
    ``apply`` can be called repeatedly (e.g. per coil batch of a dynamic series)."""

    def __init__(self, calib, coord, shape, lamda=0.01, nsteps=11, device=None):
        coord_t = _as_tensor(coord, torch.float32)
        self.device = dev = resolve_device(device, coord_t.device)
        coord_t = coord_t.to(dev)
        self.ndim = ndim = int(coord_t.shape[-1])
        if ndim not in (2, 3):
            raise ValueError("GROG needs 2D or 3D coordinates")
        self.cshape = tuple(coord_t.shape[:-1])
        self.M = int(np.prod(self.cshape))
        shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in list(shape)[-ndim:]]
        self.shape = tuple(shape)
        cal = _as_tensor(calib).to(dev)
        if cal.ndim not in (3, 4):
            raise ValueError("calib must be (nc, ny, nx) or (nc, nz, ny, nx)")
        if ndim == 3 and cal.ndim != 4:
            raise ValueError("3D GROG needs a (nc, nz, ny, nx) calibration region")
        cal = cal.to(torch.complex128)
        cal = cal / torch.linalg.norm(cal)
        self.nc = nc = int(cal.shape[0])
        G = _table(_operators(cal, ndim, lamda), nsteps)
        if ndim == 3:
            G = G[:, None]
        self.nslices = int(G.shape[1])
        self.ntable = int(G.shape[0])
        self.table = G.to(torch.complex64).contiguous()
        idx, lut = _lut(coord_t, nsteps)
        n_xyz = torch.tensor(shape[::-1], dtype=torch.int64, device=dev)
        ind = (idx + (n_xyz // 2).to(torch.float32)).to(torch.int64)
        # weights: 1 / occurrences of each flattened index over all samples (before clipping)
        unfold = torch.tensor([1, shape[-1], shape[-1] * (shape[-2] if ndim > 1 else 1)], dtype=torch.int64,
                              device=dev)[:ndim]
        flat = (ind * unfold).sum(-1).reshape(-1)
        _, inv, counts = torch.unique(flat, return_inverse=True, return_counts=True)
        self.weights = (1.0 / counts[inv].to(torch.float32)).reshape(self.cshape)
        outside = ((ind < 0) | (ind >= n_xyz)).any(-1)
        self.indexes = torch.minimum(torch.clamp(ind, min=0), n_xyz - 1)
        self.outside = outside
        lut = torch.where(outside.reshape(-1), torch.full_like(lut, -1), lut).to(torch.int32).contiguous()
        L = _lib.load()
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(L.pfb_grog_create(ctypes.c_void_p(lut.data_ptr()), self.M, self.ntable, nc, self.nslices,
                                         ctypes.c_void_p(self.table.data_ptr()), dev.index, st, ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            try:
                with torch.cuda.device(self.device):
                    _lib.load().pfb_grog_destroy(self.handle)
            except Exception:  # pragma: no cover
                pass
            self.handle = None

    def apply(self, x):
        """x (B, nc, M) complex64 on the plan's device -> same."""
        L = _lib.load()
        B = int(x.shape[0])
        if tuple(x.shape[1:]) != (self.nc, self.M) or x.dtype != torch.complex64:
            raise ValueError(f"GROG apply needs complex64 (B, {self.nc}, {self.M}), got {tuple(x.shape)} {x.dtype}")
        if self.nslices > 1 and B != self.nslices:
            raise ValueError(f"2D GROG with {self.nslices} calibration slices needs {self.nslices} leading input "
                             f"slices, got {B}")
        x = x.contiguous()
        out = torch.empty_like(x)
        n = ctypes.c_size_t()
        _lib.check(L.pfb_grog_workspace_size(self.handle, B, ctypes.byref(n)))
        ws = torch.empty(int(n.value), dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
            _lib.check(L.pfb_grog_apply(self.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                        B, ctypes.c_void_p(ws.data_ptr()), ws.numel(), st))
        return out


def grog_interp(input, calib, coord, shape, lamda=0.01, nsteps=11, device=None, threadsperblock=128):
    """GRAPPA Operator Gridding of non-Cartesian k-space (src/pyfourier/_preinterp/_grog.py:22-250).

    input: (..., nc, ncontrasts, nviews, nsamples) (the axes of ``coord[..., 0]``
    preceded by the coil axis); calib: (nc, ny, nx) / (nc, nz, ny, nx) centre of
    k-space (2D: one operator set per calibration slice, applied to the matching
    leading slice of ``input``); coord: (..., ndim) in [-N/2, N/2), axes (x, y[, z]).
    Returns (output like input, indexes (..., ndim) int64 in [0, N), weights float32).
    ``threadsperblock`` is accepted for compatibility and not used.
    """
    as_numpy = isinstance(input, np.ndarray)
    x_t = _as_tensor(input)
    idevice = x_t.device
    dev = resolve_device(device, idevice)
    plan = GrogPlan(calib, coord, shape, lamda=lamda, nsteps=nsteps, device=dev)
    nk = len(plan.cshape)
    ishape = tuple(x_t.shape)
    if len(ishape) < nk + 1 or tuple(ishape[len(ishape) - nk:]) != plan.cshape or ishape[-nk - 1] != plan.nc:
        raise ValueError(f"input {ishape} must end with (nc={plan.nc}, *{plan.cshape})")
    x = x_t.to(dev)
    x = (x if torch.is_complex(x) else x.to(torch.float32)).to(torch.complex64).reshape(-1, plan.nc, plan.M)
    out = plan.apply(x).reshape(ishape)
    ind, w = plan.indexes, plan.weights
    out, ind, w = to_caller(out, idevice), to_caller(ind, idevice), to_caller(w, idevice)
    if as_numpy:
        return out.numpy(), ind.numpy(), w.numpy()
    return out, ind, w
