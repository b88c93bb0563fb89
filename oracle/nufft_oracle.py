"""CPU oracle for the pyfourier NUFFT hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the cpu-baseline leg of
``bench.py`` may import this module, and only as the checker (or as the timed
CPU baseline).  The product path (``pyfourier_b200``) never imports it.

It restates the reference's NUFFT path on the CPU:

* the numerical kernels (Kaiser-Bessel tables, spread, interp, subspace
  variants) come from ``oracle_kernels.c`` (``liboracle.so``), a C
  restatement of the reference's Numba kernels pinned bit-for-bit (indices)
  and to float32 rounding (values, sums) against golden vectors produced by
  the reference itself (``tests/golden/kernels.npz``);
* the glue is restated in NumPy, line by line from the cited reference lines.

Where a reference glue line is defective the evident intent is implemented;
each such place says so.  References are paths inside the pyfourier project.
"""

from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np

try:  # multithreaded pocketfft with complex64 support
    import scipy.fft as _fft

    def _fftn(x, axes, norm):
        return _fft.fftn(x, axes=axes, norm=norm, workers=-1)

    def _ifftn(x, axes, norm):
        return _fft.ifftn(x, axes=axes, norm=norm, workers=-1)

except ImportError:  # pragma: no cover
    def _fftn(x, axes, norm):
        return np.fft.fftn(x, axes=axes, norm=norm)

    def _ifftn(x, axes, norm):
        return np.fft.ifftn(x, axes=axes, norm=norm)


_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    """Load (building on demand) the C restatement of the reference kernels."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        f32p = ctypes.POINTER(ctypes.c_float)
        i32p = ctypes.POINTER(ctypes.c_int32)
        vp = ctypes.c_void_p
        i64 = ctypes.c_int64
        ci = ctypes.c_int
        L.orc_kaiser_bessel.restype = ctypes.c_double
        L.orc_kaiser_bessel.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_kernel_scaling.restype = ctypes.c_double
        L.orc_kernel_scaling.argtypes = [ci, i32p, ctypes.POINTER(ctypes.c_double)]
        L.orc_prepare_interpolator.restype = None
        L.orc_prepare_interpolator.argtypes = [f32p, i32p, f32p, i64, ci, ctypes.c_double, ci]
        tab = [vp] * 6
        L.orc_grid.argtypes = [vp, vp] + tab + [i64, i64, i64] + [ci] * 6
        L.orc_degrid.argtypes = [vp, vp] + tab + [i64, i64, i64] + [ci] * 6
        L.orc_grid_subspace.argtypes = [vp, vp] + tab + [vp, i64, i64, i64, i64] + [ci] * 6
        L.orc_degrid_subspace.argtypes = [vp, vp] + tab + [vp, i64, i64, i64, i64] + [ci] * 6
        for f in (L.orc_grid, L.orc_degrid, L.orc_grid_subspace, L.orc_degrid_subspace):
            f.restype = None
        L.orc_grid_f64.restype = None
        L.orc_grid_f64.argtypes = [vp, vp, vp, ci, i64, i64, i64, vp, vp, vp, vp]
        L.orc_num_threads.restype = ci
        _LIB = L
    return _LIB


def build():
    """Compile liboracle.so with the committed Makefile."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------------------
# Kernel math
# --------------------------------------------------------------------------------------
def kaiser_bessel(x, beta):
    """_subroutines/_grid/_plan.py:157-189 (scalar)."""
    return lib().orc_kaiser_bessel(float(x), float(beta))


def kernel_scaling(beta_zyx, width_zyx):
    """_subroutines/_grid/_plan.py:118-141 (order of axes does not change the sum)."""
    nd = len(width_zyx)
    w = (ctypes.c_int32 * nd)(*[int(v) for v in width_zyx])
    b = (ctypes.c_double * nd)(*[float(v) for v in beta_zyx])
    return lib().orc_kernel_scaling(nd, w, b)


def beta_f32(width, oversamp):
    """_nufft/_plan.py:128 with width int16 and oversamp float32 (float32 result)."""
    w = np.asarray(width, dtype=np.int16)
    o = np.asarray(oversamp, dtype=np.float32)
    return (np.pi * (((w / o) * (o - 0.5)) ** 2 - 0.8) ** 0.5).astype(np.float32)


def oversamp_shape(shape, oversamp):
    """_utils/_common.py:16-18 intent (the shipped loop iterates an int): ceil(osf*N) in float32."""
    return [int(np.ceil(np.float32(o) * np.float32(n))) for n, o in zip(shape, oversamp)]


def scale_coord(coord, shape_xyz, oversamp_xyz):
    """_subroutines/_traj.py:57-65: c * (n_os / N) + n_os // 2, in float32 on each axis."""
    out = np.array(coord, dtype=np.float32, copy=True)
    for i in range(coord.shape[-1]):
        n_os = np.ceil(np.float32(oversamp_xyz[i]) * np.float32(shape_xyz[i]))
        s = np.float32(n_os / np.float32(shape_xyz[i]))
        shift = np.float32(n_os // 2)
        out[..., i] = out[..., i] * s
        out[..., i] = out[..., i] + shift
    return out


def prepare_tables(c_os, os_zyx, width_zyx, beta_zyx, is_cart_zyx=None):
    """Interpolator tables, _subroutines/_grid/_plan.py:14-91.

    c_os: (F, M, ndim) oversampled-grid coordinates in (x, y, z) order.
    Returns (index, value) tuples ordered (z, y, x), each (F, M, W_axis).
    Cartesian axes (width 1): the shipped line ``coord[i][..., None].to(np.int32)``
    (:71) is not valid NumPy; the intent, the integer grid position, is
    implemented as round-to-nearest and wrapped into the grid.
    """
    F, M, nd = c_os.shape
    flat = c_os.reshape(F * M, nd)
    idx, val = [], []
    for ax in range(nd):  # (x, y, z)
        az = nd - 1 - ax
        w = int(width_zyx[az])
        c = np.ascontiguousarray(flat[:, ax], dtype=np.float32)
        if is_cart_zyx is not None and is_cart_zyx[az]:
            i = np.mod(np.rint(c).astype(np.int64), int(os_zyx[az])).astype(np.int32)[:, None]
            v = np.ones((F * M, 1), np.float32)
        else:
            v = np.zeros((F * M, w), np.float32)
            i = np.zeros((F * M, w), np.int32)
            lib().orc_prepare_interpolator(
                v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                F * M, w, float(beta_zyx[az]), int(os_zyx[az]),
            )
        idx.append(i.reshape(F, M, -1))
        val.append(v.reshape(F, M, -1))
    return tuple(idx[::-1]), tuple(val[::-1])


def _as3(index, value, os_zyx):
    """Pad (z, y, x) tables to 3 axes with unit-width tables (index 0, value 1)."""
    nd = len(index)
    F, M = index[0].shape[:2]
    ones_i = np.zeros((F, M, 1), np.int32)
    ones_v = np.ones((F, M, 1), np.float32)
    I = [ones_i] * (3 - nd) + [np.ascontiguousarray(a) for a in index]
    V = [ones_v] * (3 - nd) + [np.ascontiguousarray(a) for a in value]
    G = [1] * (3 - nd) + [int(v) for v in os_zyx]
    return I, V, G


def spread(noncart, index, value, os_zyx, basis_kf=None):
    """_grid_nb / subspace _grid_nb.  noncart (F, B, M) complex64 -> (C, B, *os) (not scaled)."""
    I, V, G = _as3(index, value, os_zyx)
    F, B, M = noncart.shape
    noncart = np.ascontiguousarray(noncart, np.complex64)
    W = [a.shape[-1] for a in I]
    if basis_kf is None:
        out = np.zeros((F, B, *os_zyx), np.complex64)
        lib().orc_grid(_p(out), _p(noncart), *[_p(v) for v in V], *[_p(i) for i in I],
                       F, B, M, *W, *G)
    else:
        basis_kf = np.ascontiguousarray(basis_kf, np.complex64)
        K = basis_kf.shape[0]
        out = np.zeros((K, B, *os_zyx), np.complex64)
        lib().orc_grid_subspace(_p(out), _p(noncart), *[_p(v) for v in V], *[_p(i) for i in I],
                                _p(basis_kf), K, F, B, M, *W, *G)
    return out


def interp(grid, index, value, os_zyx, nframes, basis_fk=None):
    """_degrid_nb / subspace _degrid_nb.  grid (C, B, *os) -> (F, B, M) (not scaled)."""
    I, V, G = _as3(index, value, os_zyx)
    grid = np.ascontiguousarray(grid, np.complex64)
    B = grid.shape[1]
    F, M = I[0].shape[:2]
    W = [a.shape[-1] for a in I]
    out = np.zeros((F, B, M), np.complex64)
    if basis_fk is None:
        lib().orc_degrid(_p(out), _p(grid), *[_p(v) for v in V], *[_p(i) for i in I],
                         F, B, M, *W, *G)
    else:
        basis_fk = np.ascontiguousarray(basis_fk, np.complex64)
        K = basis_fk.shape[1]
        lib().orc_degrid_subspace(_p(out), _p(grid), *[_p(v) for v in V], *[_p(i) for i in I],
                                  _p(basis_fk), K, F, B, M, *W, *G)
    return out


# --------------------------------------------------------------------------------------
# Array-level glue
# --------------------------------------------------------------------------------------
def apod_vector(n, oversamp, width, beta):
    """_subroutines/_apod.py:27-41 for one axis of length n (float64 math, float32 result)."""
    os_i = float(np.ceil(np.float32(oversamp) * np.float32(n)))
    idx = np.arange(n, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        a = np.sqrt(float(beta) ** 2 - (math.pi * int(width) * (idx - n // 2) / os_i) ** 2)
        a = a / np.sinh(a)
        a = a / a[n // 2]
    a = np.nan_to_num(a, nan=1.0)
    return a.astype(np.float32)


_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        from concurrent.futures import ThreadPoolExecutor

        _POOL = ThreadPoolExecutor(max_workers=os.cpu_count() or 1)
    return _POOL


def _map_batch(fn, x, ndim, tail=None, dtype=None):
    """fn over the leading (batch) items of x, in host threads for large arrays.

    NumPy releases the GIL in copies and elementwise arithmetic, so the items run
    in parallel; every item goes through exactly the operations fn(x) would apply
    to it, so the result is identical to fn on the whole array (the reference's
    glue runs its array library's threaded kernels; a single-threaded NumPy pass
    would understate it in the timed CPU baseline)."""
    lead = x.shape[: x.ndim - ndim]
    n = int(np.prod(lead)) if lead else 1
    if n < 2 or x.size < (1 << 22):
        return fn(x)
    xs = x.reshape(n, *x.shape[x.ndim - ndim:])
    first = fn(xs[0])
    out = np.empty((n, *first.shape), first.dtype)
    out[0] = first

    def work(i):
        out[i] = fn(xs[i])

    list(_pool().map(work, range(1, n)))
    return out.reshape(*lead, *first.shape)


def _apodize1(x, ndim, oversamp_zyx, width_zyx, beta_zyx):
    out = np.array(x, copy=True)
    for n in range(1, ndim + 1):
        ax = -n
        if int(width_zyx[ax]) != 1:
            i = out.shape[ax]
            a = apod_vector(i, oversamp_zyx[ax], width_zyx[ax], beta_zyx[ax])
            out = out * a.reshape([i] + [1] * (n - 1))
    return out.astype(x.dtype)


def apodize(x, ndim, oversamp_zyx, width_zyx, beta_zyx):
    """_subroutines/_apod.py:16-46, returning a new array (the shipped code mutates its input)."""
    return _map_batch(lambda xi: _apodize1(xi, ndim, oversamp_zyx, width_zyx, beta_zyx), x, ndim)


def _resize1(x, oshape):
    oshape = list(x.shape[: x.ndim - len(oshape)]) + list(oshape)
    if list(x.shape) == oshape:
        return x
    ishift = [max(i // 2 - o // 2, 0) for i, o in zip(x.shape, oshape)]
    oshift = [max(o // 2 - i // 2, 0) for i, o in zip(x.shape, oshape)]
    copy = [min(i - si, o - so) for i, si, o, so in zip(x.shape, ishift, oshape, oshift)]
    out = np.zeros(oshape, x.dtype)
    out[tuple(slice(s, s + c) for s, c in zip(oshift, copy))] = x[
        tuple(slice(s, s + c) for s, c in zip(ishift, copy))]
    return out


def resize(x, oshape):
    """_subroutines/_resize.py:16-42: centred zero-pad / crop over the trailing axes."""
    oshape = list(oshape)
    if list(x.shape[x.ndim - len(oshape):]) == oshape:
        return x
    return _map_batch(lambda xi: _resize1(xi, oshape), x, len(oshape))


def fft_c(x, ndim, norm=None, centered=True):
    """_subroutines/_fft.py:72-79: fftshift(fftn(ifftshift(x)))."""
    ax = tuple(range(-ndim, 0))
    if centered:
        xi = _map_batch(lambda v: np.fft.ifftshift(v, axes=ax), x, ndim)
        y = _fftn(xi, ax, norm)
        return _map_batch(lambda v: np.fft.fftshift(v, axes=ax), y, ndim).astype(x.dtype, copy=False)
    return _fftn(x, ax, norm).astype(x.dtype, copy=False)


def ifft_c(x, ndim, norm=None, centered=True):
    """_subroutines/_fft.py:165-172: fftshift(ifftn(ifftshift(x)))."""
    ax = tuple(range(-ndim, 0))
    if centered:
        xi = _map_batch(lambda v: np.fft.ifftshift(v, axes=ax), x, ndim)
        y = _ifftn(xi, ax, norm)
        return _map_batch(lambda v: np.fft.fftshift(v, axes=ax), y, ndim).astype(x.dtype, copy=False)
    return _ifftn(x, ax, norm).astype(x.dtype, copy=False)


# --------------------------------------------------------------------------------------
# B0 time segmentation
# --------------------------------------------------------------------------------------
def _acorr_hist(hk, c0, c1=None):
    """Histogram of z(r') + conj(z(r)) over pixel pairs, from the histogram of z.

    Real (B0) axis: differences c0[i] - c0[j] (an autocorrelation).  R2* axis:
    sums c1[i] + c1[j] (a self-convolution).  This is the Toeplitz form of the
    histogram (the commented ``acorr`` branch of _subroutines/_b0.py:86-106).
    """
    if c1 is None:
        h = np.correlate(hk, hk, mode="full")  # index i - j + n - 1
        d0 = c0[1] - c0[0]
        zk = 1j * d0 * np.arange(-(len(c0) - 1), len(c0))
        return h, zk
    n0, n1 = hk.shape
    h = np.zeros((2 * n0 - 1, 2 * n1 - 1))
    i0, i1 = np.nonzero(hk)
    for a0, a1 in zip(i0, i1):
        # pixel pairs (a, b): B0 index a0 - b0 + n0 - 1, R2* index a1 + b1
        h[a0 - np.arange(n0)[:, None] + n0 - 1, a1 + np.arange(n1)[None, :]] += hk[a0, a1] * hk
    d0, d1 = c0[1] - c0[0], (c1[1] - c1[0]) if n1 > 1 else 0.0
    zk = 1j * d0 * np.arange(-(n0 - 1), n0)[:, None] + (2 * c1[0] + d1 * np.arange(2 * n1 - 1))[None, :]
    return h, zk


def mri_exp_approx(zmap, t, L=6, bins=(40, 40), acorr=False):
    """_subroutines/_b0.py:10-135 in float64, with three intent fixes.

    * bin centres are the midpoints of the histogram edges (the shipped
      ``ze[1:] - ze[1] / 2`` subtracts half an edge value, not half a bin);
    * the temporal basis fits exp(-z t), the same sign as the spatial
      coefficients C_l = exp(-z t_l) (the shipped code fits exp(+z t));
    * a real map is histogrammed on its values (the shipped code histograms the
      complexified map).
    ``acorr=True`` fits the basis over the histogram of z(r') + conj(z(r))
    (for the Toeplitz Gram), the reference's commented branch.
    Returns (B (L, nt) complex128, C (L, *zmap.shape) complex128).
    """
    zmap = np.asarray(zmap)
    t = np.asarray(t, np.float64)
    if not isinstance(bins, (list, tuple)):
        bins = (bins, 5)
    if np.isrealobj(zmap):
        z = 2 * math.pi * 1j * zmap.astype(np.float64)
        hk, ze = np.histogram(2 * math.pi * zmap.ravel().astype(np.float64), bins=int(bins[0]))
        c0 = 0.5 * (ze[1:] + ze[:-1])
        if acorr:
            hk, zk = _acorr_hist(hk.astype(np.float64), c0)
        else:
            zk = 1j * c0
    else:
        z = 2 * math.pi * zmap.astype(np.complex128)
        zz = z.ravel()
        hk, e0, e1 = np.histogram2d(zz.imag, zz.real, bins=[int(bins[0]), int(bins[1])])
        c0, c1 = 0.5 * (e0[1:] + e0[:-1]), 0.5 * (e1[1:] + e1[:-1])
        if acorr:
            hk, zk = _acorr_hist(hk.astype(np.float64), c0, c1)
        else:
            zk = (1j * c0[:, None] + c1[None, :])
    hk = hk.ravel().astype(np.float64)
    zk = zk.ravel()
    tl = np.linspace(0, L, L) / L * t[-1]
    ch = np.exp(-tl[:, None] * zk[None, :])  # (L, K)
    w = np.diag(hk ** 0.5)
    p = np.linalg.pinv(w @ ch.T) @ w  # (L, K)
    b = p @ np.exp(-zk[:, None] * t[None, :])  # (L, nt)
    ct = np.exp(-tl.reshape([L] + [1] * z.ndim) * z[None])
    ct = np.nan_to_num(ct, nan=0.0, posinf=0.0, neginf=0.0)
    return b, ct


# --------------------------------------------------------------------------------------
# Plan and operators
# --------------------------------------------------------------------------------------
@dataclass
class OraclePlan:
    ndim: int
    oversamp: tuple
    width: tuple
    beta: tuple
    os_shape: tuple
    shape: tuple
    index: tuple
    value: tuple
    scale: float
    nframes: int
    dshape: tuple
    zmap_t_kernel: object = None
    zmap_s_kernel: object = None
    zmap_batch_size: int = None
    c_os: object = None
    is_cart: tuple = None


def plan_nufft(coord, shape, width=4, oversamp=1.25, zmap=None, L=6, nbins=(40, 40), dt=None,
               T=None, L_batch_size=None):
    """_nufft/_plan.py:20-199.

    Coordinates are taken in cycles/FOV in [-N/2, N/2): ``normalize_coordinates``
    (_traj.py:10-53) is the identity for such input by its documented contract;
    the shipped version divides each sample by its own radius.
    """
    coord = np.asarray(coord, np.float32)
    ndim = coord.shape[-1]
    width = np.asarray([width] * ndim if np.isscalar(width) else width, np.int16)
    oversamp = np.asarray([oversamp] * ndim if np.isscalar(oversamp) else oversamp, np.float32)
    beta = beta_f32(width, oversamp)
    shape = np.asarray([shape] * ndim if np.isscalar(shape) else list(shape)[-ndim:], np.int64)
    is_cart = np.asarray([np.allclose(coord[..., ax], np.round(coord[..., ax]))
                          for ax in range(ndim)][::-1])
    oversamp[is_cart] = 1.0
    width[is_cart] = 1
    os_shape = oversamp_shape(shape, oversamp)
    c_os = scale_coord(coord, shape[::-1], oversamp[::-1])
    cs = list(c_os.shape[:-1])
    while len(cs) < 3:
        cs = [1] + cs
    nframes = cs[0]
    dshape = tuple(coord.shape[-3:-1]) if coord.ndim >= 3 else tuple(coord.shape[-2:-1])
    c3 = c_os.reshape(nframes, -1, ndim)
    index, value = prepare_tables(c3, os_shape, width, beta, is_cart)
    w_eff = [1 if is_cart[a] else int(width[a]) for a in range(ndim)]
    scale = kernel_scaling([float(b) for b in beta], w_eff)
    zt = zs = None
    if zmap is not None:
        if T is None:
            T = dt * np.arange(coord.shape[-2], dtype=np.float32)
        zt, zs = mri_exp_approx(zmap, T, L, nbins)
        if L_batch_size is None:
            L_batch_size = L
    return OraclePlan(ndim, tuple(oversamp), tuple(width), tuple(beta), tuple(os_shape),
                      tuple(int(s) for s in shape), index, value, scale, nframes, dshape,
                      zt, zs, L_batch_size, c3, tuple(bool(v) for v in is_cart))


def _cart2noncart(kgrid, plan, basis):
    """_grid/_cart2noncart/__init__.py:25-110 (batch shape per the ndim-aware intent)."""
    nd, F = plan.ndim, plan.nframes
    has_c = F > 1 or basis is not None
    batch_shape = kgrid.shape[: kgrid.ndim - nd - (1 if has_c else 0)]
    B = int(np.prod(batch_shape))
    C = basis.shape[1] if basis is not None else F
    g = kgrid.reshape(B, C, *plan.os_shape).swapaxes(0, 1)
    y = interp(g, plan.index, plan.value, plan.os_shape, F, basis)
    if F == 1:
        y = y[0].reshape(*batch_shape, *plan.dshape)
    else:
        y = y.swapaxes(0, 1).reshape(*batch_shape, F, *plan.dshape)
    return (y / np.float32(plan.scale)).astype(np.complex64)


def _noncart2cart(kspace, plan, basis):
    """_grid/_noncart2cart/__init__.py:25-119."""
    nd, F = plan.ndim, plan.nframes
    batch_shape = kspace.shape[: kspace.ndim - len(plan.dshape) - (1 if F > 1 else 0)]
    B = int(np.prod(batch_shape))
    y = kspace.reshape(B, F, -1).swapaxes(0, 1)
    bkf = None if basis is None else np.ascontiguousarray(basis.conj().T)
    g = spread(y, plan.index, plan.value, plan.os_shape, bkf)
    if F == 1 and basis is None:
        g = g[0].reshape(*batch_shape, *plan.os_shape)
    else:
        g = g.swapaxes(0, 1).reshape(*batch_shape, g.shape[0], *plan.os_shape)
    return (g / np.float32(plan.scale)).astype(np.complex64)


def _do_nufft(image, plan, basis, norm):
    """_nufft/_nufft.py:218-251."""
    nd = plan.ndim
    x = apodize(image, nd, plan.oversamp, plan.width, plan.beta)
    x = resize(x, plan.os_shape)
    k = fft_c(x, nd, norm)
    return _cart2noncart(k, plan, basis)


def _do_nufft_adj(kspace, plan, basis, norm):
    """_nufft/_nufft.py:254-287."""
    nd = plan.ndim
    g = _noncart2cart(kspace, plan, basis)
    x = ifft_c(g, nd, norm)
    x = resize(x, plan.shape)
    return apodize(x, nd, plan.oversamp, plan.width, plan.beta)


def _readout_len(plan):
    return plan.dshape[-1]


def nufft_fwd(image, plan, basis=None, weight=None, norm=None):
    """_nufft/_nufft.py:11-90.  The B0 branch sums each segment chunk once (the
    shipped loop adds every chunk twice, :80-84)."""
    image = np.asarray(image, np.complex64)
    if plan.zmap_s_kernel is None:
        k = _do_nufft(image, plan, basis, norm)
    else:
        Lseg = plan.zmap_s_kernel.shape[0]
        k = 0.0
        for start in range(0, Lseg, plan.zmap_batch_size):
            stop = min(Lseg, start + plan.zmap_batch_size)
            C = plan.zmap_s_kernel[start:stop].astype(np.complex64)
            itmp = C.reshape(C.shape[0], *([1] * (image.ndim - plan.ndim)), *C.shape[1:]) * image[None]
            ktmp = _do_nufft(itmp.astype(np.complex64), plan, basis, norm)  # (l, ..., nv, ns)
            Bt = plan.zmap_t_kernel[start:stop].astype(np.complex64)  # (l, ns)
            Bt = Bt.reshape(Bt.shape[0], *([1] * (ktmp.ndim - 2)), Bt.shape[1])
            k = k + (Bt * ktmp).sum(axis=0)
        k = k.astype(np.complex64)
    if weight is not None:
        k = (weight * k).astype(np.complex64)
    return k


def nufft_adj(kspace, plan, basis=None, weight=None, norm=None):
    """_nufft/_nufft.py:93-169."""
    kspace = np.asarray(kspace, np.complex64)
    if weight is not None:
        kspace = (weight * kspace).astype(np.complex64)
    if plan.zmap_s_kernel is None:
        return _do_nufft_adj(kspace, plan, basis, norm)
    Lseg = plan.zmap_s_kernel.shape[0]
    img = 0.0
    for start in range(0, Lseg, plan.zmap_batch_size):
        stop = min(Lseg, start + plan.zmap_batch_size)
        Bt = plan.zmap_t_kernel[start:stop].astype(np.complex64)
        Bt = Bt.reshape(Bt.shape[0], *([1] * (kspace.ndim - 1)), Bt.shape[1])
        ktmp = (Bt.conj() * kspace[None]).astype(np.complex64)
        itmp = _do_nufft_adj(ktmp, plan, basis, norm)  # (l, ..., N)
        C = plan.zmap_s_kernel[start:stop].astype(np.complex64)
        C = C.reshape(C.shape[0], *([1] * (itmp.ndim - 1 - plan.ndim)), *C.shape[1:])
        img = img + (C.conj() * itmp).sum(axis=0)
    return img.astype(np.complex64)


# --------------------------------------------------------------------------------------
# Toeplitz Gram
# --------------------------------------------------------------------------------------
@dataclass
class OracleGram:
    value: object  # (F, *os) elementwise, or (nvox, K, K) per-voxel matrices; leading L with a field map
    shape: tuple
    ndim: int
    islowrank: bool
    zmap_s_kernel: object = None  # (L, *shape) spatial B0 coefficients C_l


def apod_vector64(n, oversamp, width, beta):
    """apod_vector in float64 throughout (the plan-time float64 PSF)."""
    os_i = float(np.ceil(np.float32(oversamp) * np.float32(n)))
    idx = np.arange(n, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        a = np.sqrt(float(beta) ** 2 - (math.pi * int(width) * (idx - n // 2) / os_i) ** 2)
        a = a / np.sinh(a)
        a = a / a[n // 2]
    return np.nan_to_num(a, nan=1.0)


def spread_f64(values, plan):
    """Float64 spread on a plan's grid: values (F, B, M) -> (F, B, *os) complex128,
    taps in float64 (orc_grid_f64), not divided by the kernel scale."""
    F, M, nd = plan.c_os.shape
    B = values.shape[1]
    v = np.ascontiguousarray(values, np.complex128).reshape(F, B, M)
    out = np.zeros((F, B, *plan.os_shape), np.complex128)
    cxyz = np.ascontiguousarray(plan.c_os, np.float32)
    w = (ctypes.c_int * nd)(*[int(x) for x in plan.width[::-1]])
    bt = (ctypes.c_double * nd)(*[float(x) for x in plan.beta[::-1]])
    no = (ctypes.c_int * nd)(*[int(x) for x in plan.os_shape[::-1]])
    ca = (ctypes.c_int * nd)(*[int(bool(x)) for x in (plan.is_cart or (False,) * nd)[::-1]])
    lib().orc_grid_f64(_p(out), _p(v), _p(cxyz), nd, F, B, M, w, bt, no, ca)
    return out


def nufft_adj_f64(kspace, plan):
    """The adjoint NUFFT of a single-frame plan (norm None) with the reference's
    taps and kernel but float64 arithmetic throughout: float64 spread
    (orc_grid_f64), complex128 centred inverse FFT, crop, float64 deapodisation.
    kspace (B, M) -> (B, *shape) complex128.  A precision reference: the
    reference's float32 serial sums (_noncart2cart/_3D.py:29-50) drift from it on
    crowded trajectories (about 7e-4 rel-L2 at the 3D radial 200^3 / 8 M-sample
    size), an algorithm in float64 does not."""
    nd = plan.ndim
    k = np.asarray(kspace, np.complex128)
    B = k.shape[0]
    G = spread_f64(k.reshape(1, B, -1), plan)[0] / plan.scale
    x = ifft_c(G, nd, None)
    x = resize(x, plan.shape)
    for n in range(1, nd + 1):
        ax = -n
        if int(plan.width[ax]) != 1:
            a = apod_vector64(x.shape[ax], plan.oversamp[ax], plan.width[ax], plan.beta[ax])
            x = x * a.reshape([x.shape[ax]] + [1] * (n - 1))
    return x


def psf_f64(values, pplan, os_shape, basis=None):
    """The Toeplitz PSF in float64 (plan time): the adjoint NUFFT of the per-sample
    values on the PSF plan ``pplan`` (2x coordinates), cropped to ``os_shape``.

    values (L, F, M): per B0 segment l the sample weights (times B_l(t)).  With a
    basis (F, K) the subspace projection of the reference's PSF
    (delta[k1, f] = basis[f, k1], spread with conj(basis[f, k2]),
    _sparsegram/_plan.py:201-208 with _noncart2cart/_2D_subspace.py:49-53) is
    taken after the per-frame spread, by linearity: P[l, k1, k2] = sum_f
    basis[f, k1] conj(basis[f, k2]) G[l, f].  The rest of the adjoint (division
    by the kernel scale, centred inverse FFT with norm None, crop, float64
    deapodisation) follows _nufft/_nufft.py:254-287.  Returns (L, K, K, *os) or
    (L, F, *os) complex128."""
    nd = pplan.ndim
    Ls, F = values.shape[:2]
    G = spread_f64(np.moveaxis(values, 0, 1), pplan) / pplan.scale  # (F, L, *os_psf)
    G = np.moveaxis(G, 1, 0)  # (L, F, ...)
    if basis is not None:
        b = np.asarray(basis, np.complex128)
        G = np.einsum("fa,fb,lf...->lab...", b, b.conj(), G)
    x = ifft_c(G, nd, None)
    x = resize(x, os_shape)
    for n in range(1, nd + 1):
        ax = -n
        if int(pplan.width[ax]) != 1:
            a = apod_vector64(x.shape[ax], pplan.oversamp[ax], pplan.width[ax], pplan.beta[ax])
            x = x * a.reshape([x.shape[ax]] + [1] * (n - 1))
    return x


def plan_spgram(coord, shape, basis=None, weight=None, width=6, normalize="reference", zmap=None, L=6,
                nbins=(40, 40), dt=None, T=None):
    """_sparsegram/_plan.py:20-249 with its intent fixes.

    PSF = adjoint NUFFT of ``weight * delta`` at 2x coordinates onto the 2N
    grid (:201-208, with the keyword intent restored), computed in float64
    (``psf_f64``; the reference uses its complex64 NUFFT), then a centred
    orthonormal FFT and ifftshift (:211, :226).  With a basis the per-voxel
    matrix is value[v][k2][k1] = T[k1, k2](v) (so out = value[v] @ in, the
    evident intent of _bmatvec/_bdot.py).  ``normalize="reference"`` divides by
    mean(|T| over T != 0) (:242); ``normalize=None`` scales T so that the Gram
    equals A^H W A with A = nufft(norm=None) and A^H its exact adjoint.
    With a field map (:162-182, :26-53 of _sparsegram.py) there is one kernel per
    time segment, built with the sample weights B_l(t), and the apply is
    sum_l conj(C_l) G_l(C_l x); B and C come from the autocorrelated histogram
    (``mri_exp_approx(..., acorr=True)``), which approximates the pairwise
    phase exp(-(z(r') + conj(z(r))) t) that the Gram needs.
    """
    coord = np.asarray(coord, np.float32)
    ndim = coord.shape[-1]
    shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in list(shape)[-ndim:]]
    is_cart = [np.allclose(shape[::-1][ax] * coord[..., ax], np.round(shape[::-1][ax] * coord[..., ax]))
               for ax in range(ndim)][::-1]
    osf = np.asarray([1.0 if c else 2.0 for c in is_cart], np.float32)
    os_shape = oversamp_shape(shape, osf)
    wgt = np.ones(coord.shape[:-1], np.float32) if weight is None else np.asarray(weight, np.float32)
    if basis is not None:
        basis = np.asarray(basis, np.complex64)
    Cl = None
    vals = wgt.astype(np.complex128)[None]  # (L = 1, F, ...)
    if zmap is not None:
        if T is None:
            T = dt * np.arange(coord.shape[-2], dtype=np.float32)
        Bt, Cl = mri_exp_approx(zmap, T, L, nbins, acorr=True)
        # segment l weights each sample by B_l(t) of its readout position (last axis)
        vals = vals * Bt.astype(np.complex128).reshape(L, *([1] * (vals.ndim - 2)), Bt.shape[-1])
        Cl = Cl.astype(np.complex64)
    pplan = plan_nufft(coord * osf[::-1], os_shape, width=width, oversamp=1.25)
    # the PSF in float64 at plan time (the reference builds it with its complex64
    # adjoint NUFFT, _sparsegram/_plan.py:201-208); applies stay complex64
    Fp = pplan.nframes
    psf = psf_f64(vals.reshape(vals.shape[0], Fp, -1), pplan, os_shape, basis)
    G_os = float(np.prod(pplan.os_shape))
    if normalize is None:
        T = fft_c(psf * G_os, ndim, norm=None)
    else:
        T = fft_c(psf, ndim, norm="ortho")
    nlead = 1 if zmap is not None else 0
    if not nlead:
        T = T[0]
    if basis is None and T.ndim > ndim + nlead and T.shape[nlead] == 1:
        T = T[:, 0] if nlead else T[0]
    T = np.fft.ifftshift(T, axes=tuple(range(-ndim, 0)))
    if basis is not None:
        K = basis.shape[1]
        T = T.reshape(-1, K, K, int(np.prod(os_shape)))
        T = np.ascontiguousarray(T.transpose(0, 3, 2, 1))  # (L, nvox, k2, k1)
        if not nlead:
            T = T[0]
    if normalize == "reference":
        nz = T[T != 0]
        T = T / np.mean(np.abs(nz))
    T = np.nan_to_num(T).astype(np.complex64)
    return OracleGram(T, tuple(os_shape), ndim, basis is not None, Cl)


def sparse_gram(image, gram, norm=None):
    """_sparsegram/_sparsegram.py:11-81 with the per-voxel product out = T[v] @ in;
    with a field map sum_l conj(C_l) G_l(C_l x)."""
    image = np.asarray(image, np.complex64)
    if gram.zmap_s_kernel is not None:
        C = gram.zmap_s_kernel
        nd = gram.ndim
        out = 0
        for l in range(C.shape[0]):
            gl = OracleGram(gram.value[l], gram.shape, gram.ndim, gram.islowrank)
            out = out + np.conj(C[l]) * _sparse_gram1(C[l] * image, gl, norm)
        return np.asarray(out, np.complex64)
    return _sparse_gram1(image, gram, norm)


def _sparse_gram1(image, gram, norm=None):
    image = np.asarray(image, np.complex64)
    nd = gram.ndim
    shape = image.shape[-nd:]
    x = resize(image, gram.shape)
    k = fft_c(x, nd, norm, centered=False)
    if gram.islowrank:
        K = gram.value.shape[-1]
        kk = k.reshape(-1, K, int(np.prod(gram.shape)))  # (nb, K, nvox)
        out = np.einsum("vij,bjv->biv", gram.value, kk)
        k = out.reshape(k.shape).astype(np.complex64)
    else:
        k = (gram.value * k).astype(np.complex64)
    x = ifft_c(k, nd, norm, centered=False)
    return resize(x, shape).astype(np.complex64)


# --------------------------------------------------------------------------------------
# Cartesian (dense) Gram
# --------------------------------------------------------------------------------------
def plan_gram(mask, shape, basis=None, zmap=None, T=None, L=6, nbins=(40, 40)):
    """_gram/_plan.py:19-157 with its intent fixes.

    The kernel is the sampling mask (centred, DC at N // 2) moved to FFT order
    with ``ifftshift`` (both branches; the shipped code shifts only the low-rank
    kernel, with ``fftshift``, :133-135).  With a basis (:122-135) the per-voxel
    matrix is value[v][k2][k1] = sum_t mask_t(v) B[t, k1] conj(B[t, k2]).  A 1D
    mask (ny,) is (1, ny, 1) and a 2D one has one frame (:90-94); mask planes
    broadcast to ``shape``.  With a field map (:114-125, :138-145) the spatial
    coefficients are not folded into the k-space kernel: segment l weights mask
    point p by B_l(T[p]) (``mri_exp_approx(..., acorr=True)`` over the distinct
    sampling times) and the apply is sum_l conj(C_l) G_l(C_l x), as for the
    Toeplitz Gram.
    """
    shape = tuple(int(s) for s in shape)
    assert len(shape) == 2, "dense Gram FFT is 2D (or separable 3D) only (_plan.py:86-88)"
    m = np.asarray(mask, np.float64)
    if m.ndim == 1:
        m = m[None, :, None]
    elif m.ndim == 2:
        m = m[None]
    m = np.broadcast_to(m, (m.shape[0], *shape))
    nt = m.shape[0]
    m = np.fft.ifftshift(m, axes=(-2, -1))
    Cl = None
    if zmap is not None:
        t = np.fft.ifftshift(np.broadcast_to(np.asarray(T, np.float32), m.shape), axes=(-2, -1))
        tu, inv = np.unique(t.astype(np.float64).ravel(), return_inverse=True)
        Bt, Cl = mri_exp_approx(zmap, tu, L, nbins, acorr=True)
        wl = Bt[:, inv].reshape(L, *m.shape)
        Cl = Cl.astype(np.complex64)
    else:
        wl = np.ones((1, *m.shape))
    mw = wl * m[None]  # (L, nt, ny, nx)
    nvox = int(np.prod(shape))
    if basis is not None:
        B = np.asarray(basis, np.complex128)
        assert B.shape[0] == nt
        K = B.shape[1]
        val = np.zeros((mw.shape[0], nvox, K, K), np.complex128)
        for t_ in range(nt):
            outer = np.conj(B[t_])[:, None] * B[t_][None, :]  # [k2, k1]
            val += mw[:, t_].reshape(mw.shape[0], nvox, 1, 1) * outer
    else:
        val = mw
    if zmap is None:
        val = val[0]
    return OracleGram(val.astype(np.complex64), shape, 2, basis is not None, Cl)


def gram(image, gram_matrix, norm=None):
    """_gram/_gram.py:11-133: uncentred FFT, per-voxel product with the kernel,
    uncentred inverse FFT (no embedding: the grid is the image); with a field map
    sum_l conj(C_l) G_l(C_l x)."""
    return sparse_gram(image, gram_matrix, norm)


# --------------------------------------------------------------------------------------
# Sparse (Cartesian-subsampled) FFT
# --------------------------------------------------------------------------------------
def _sparse_index(indexes, shape):
    """(frames, npts, ndim) integer grid indexes in (z, y, x) order (centred input,
    any entry negative, shifted by N // 2, the intent of _traj.py:36-53), and dshape."""
    idx = np.rint(np.asarray(indexes, np.float64)).astype(np.int64)
    nd = idx.shape[-1]
    if (idx < 0).any():
        idx = idx + np.asarray([s // 2 for s in shape[::-1]])
    ds = list(idx.shape[:-1])
    while len(ds) < 3:
        ds = [1] + ds
    return idx.reshape(ds[0], -1, nd)[..., ::-1], tuple(ds[1:])


def dense_to_sparse(dense, idx, basis_adj=None):
    """_mask/_dense2sparse/_{2,3}D[_subspace].py (``_mask_nb``): gather the sampled grid
    points.  dense (F, B, *N) (or (K, B, *N) with a basis), idx (F, npts, d) in (z, y, x)
    order; returns (F, B, npts): sparse[f, b, p] = dense[f, b, idx[f, p]], or
    sum_k basis_adj[f, k] dense[k, b, idx[f, p]] accumulated over k in order."""
    dense = np.asarray(dense, np.complex64)
    F, npts, d = idx.shape
    B = dense.shape[1]
    out = np.zeros((F, B, npts), np.complex64)
    for f in range(F):
        sel = tuple(idx[f, :, a] for a in range(d))
        if basis_adj is None:
            out[f] = dense[f][(slice(None),) + sel]
        else:
            for k in range(dense.shape[0]):
                out[f] += np.complex64(basis_adj[f, k]) * dense[k][(slice(None),) + sel]
    return out


def sparse_to_dense(sparse, idx, shape, basis=None):
    """_mask/_sparse2dense/_{2,3}D[_subspace].py (``_zerofill_nb``): scatter-add the samples
    (repeated points add, frame by frame and point by point).  sparse (F, B, npts), idx
    (F, npts, d) (z, y, x); returns (F, B, *shape), or with basis (K, F) the projection
    dense[k] += basis[k, f] sparse[f] -> (K, B, *shape)."""
    sparse = np.asarray(sparse, np.complex64)
    F, B, npts = sparse.shape
    d = idx.shape[-1]
    C = F if basis is None else basis.shape[0]
    out = np.zeros((C, B, *shape), np.complex64)
    for c in range(C):
        for b in range(B):
            for f in range(F):
                if basis is None and f != c:
                    continue
                sel = tuple(idx[f, :, a] for a in range(d))
                v = sparse[f, b] if basis is None else np.complex64(basis[c, f]) * sparse[f, b]
                np.add.at(out[c, b], sel, v)
    return out


def sparse_fftn(image, indexes, shape, basis=None, norm=None):
    """src/pyfourier/_sparsefft/_sparsefft.py:98-108: centred FFT, then the masking gather
    (``dense_to_sparse``; with a basis the adjoint projection sum_k basis[f, k] X[k])."""
    nd = len(shape)
    idx, ds = _sparse_index(indexes, shape)
    F = idx.shape[0]
    X = fft_c(np.asarray(image, np.complex64), nd, norm)
    C = X.shape[-nd - 1] if (basis is not None or F > 1) else 1
    X = X.reshape(-1, C, *shape)
    if basis is None and C == 1 and F > 1:
        X = np.broadcast_to(X, (X.shape[0], F, *shape))
    dense = np.ascontiguousarray(np.swapaxes(X, 0, 1))  # (C, B, *N)
    out = dense_to_sparse(dense, idx, None if basis is None else np.asarray(basis, np.complex64))
    return np.ascontiguousarray(np.swapaxes(out, 0, 1))  # (B, F, npts)


def sparse_ifftn(kspace, indexes, shape, basis=None, norm=None):
    """src/pyfourier/_sparsefft/_sparsefft.py:111-121: the masking scatter-add
    (``sparse_to_dense``; with a basis the conj-transposed projection), then the centred
    inverse FFT."""
    nd = len(shape)
    idx, ds = _sparse_index(indexes, shape)
    F = idx.shape[0]
    y = np.asarray(kspace, np.complex64).reshape(-1, F, idx.shape[1])
    bt = None if basis is None else np.ascontiguousarray(np.asarray(basis, np.complex64).conj().T)
    grid = sparse_to_dense(np.ascontiguousarray(np.swapaxes(y, 0, 1)), idx, tuple(shape), bt)
    return ifft_c(np.ascontiguousarray(np.swapaxes(grid, 0, 1)), nd, norm)


# --------------------------------------------------------------------------------------
# Pipe-Menon density compensation
# --------------------------------------------------------------------------------------
def pipe_menon_dcf(coord, shape, niter=30, width=6, oversamp=1.5):
    """src/pyfourier/_dcomp/pipemenon.py:9-96: w = ones(coord.shape[:-1]); the plan
    with (width, oversamp); niter times w = w / |nufft(nufft_adj(w, ortho), ortho)|
    (_GHG, :99-115).  float32 like the reference's weights."""
    coord = np.asarray(coord, np.float32)
    w = np.ones(coord.shape[:-1], np.float32)
    plan = plan_nufft(coord, shape, width=width, oversamp=oversamp)
    for _ in range(niter):
        ghg = nufft_fwd(nufft_adj(w.astype(np.complex64), plan, norm="ortho"), plan, norm="ortho")
        w = (w / np.abs(ghg)).astype(np.float32)
    return w


# --------------------------------------------------------------------------------------
# GROG pre-interpolation
# --------------------------------------------------------------------------------------
def grog_operators(calib, ndim, lamda=0.01):
    """_preinterp/_grog.py:253-356 (``_calc_grappaop``, ``_grappa_op_2d/3d``) in complex128.

    Per axis the GRAPPA operator G solving (S^H S + l0 I) G = S^H T, with source rows S
    the calibration coil vectors and targets T their neighbours one step further along
    the axis, l0 = lamda * ||S||_F / nc.  2D: one operator per calibration slice,
    (nz, nc, nc); 3D: (nc, nc).  Returned in (x, y[, z]) order.  (The shipped helpers
    take their array backend from the builtin ``input``, :288, :326, :359; the
    calibration array's is the evident intent.)
    """
    c = np.asarray(calib, np.complex128)
    if c.ndim == 3:
        c = c[:, None]
    c = np.moveaxis(c, 0, -1)  # (nz, ny, nx, nc)
    nc = c.shape[-1]

    def train(S, T):
        Sh = np.conj(np.swapaxes(S, -1, -2))
        l0 = lamda * np.linalg.norm(Sh, axis=(-2, -1)) / nc
        A = Sh @ S + l0[..., None, None] * np.eye(nc)
        return np.linalg.solve(A, Sh @ T)

    nz = c.shape[0]
    if ndim == 2:
        gy = train(c[:, :-1].reshape(nz, -1, nc), c[:, 1:].reshape(nz, -1, nc))
        gx = train(c[:, :, :-1].reshape(nz, -1, nc), c[:, :, 1:].reshape(nz, -1, nc))
        return [gx, gy]
    gz = train(c[:-1].reshape(-1, nc), c[1:].reshape(-1, nc))
    gy = train(c[:, :-1].reshape(-1, nc), c[:, 1:].reshape(-1, nc))
    gx = train(c[:, :, :-1].reshape(-1, nc), c[:, :, 1:].reshape(-1, nc))
    return [gx, gy, gz]


def _fractional_powers(A, deltas):
    """_grog.py:369-396 (``_weight_grid``): A^d = V diag(L^d) V^-1, principal branch."""
    L, V = np.linalg.eig(A)
    Vi = np.linalg.inv(V)
    return np.stack([(V * (L ** d)[..., None, :]) @ Vi for d in deltas])  # (nsteps, ..., nc, nc)


def grog_table(ops, nsteps=11):
    """_grog.py:131-170: G[(iz n + iy) n + ix] = Gx^dx @ Gy^dy (@ Gz^dz), the steps
    d = (i - (n - 1) / 2) / (n - 1).  2D: (n^2, nz, nc, nc); 3D: (n^3, nc, nc)."""
    n = 2 * (nsteps // 2) + 1
    deltas = (np.arange(n) - (n - 1) // 2) / (n - 1)
    P = [_fractional_powers(o, deltas) for o in ops]
    if len(ops) == 2:
        G = P[0][None, :] @ P[1][:, None]  # [iy, ix] = Gx[ix] @ Gy[iy]
        return G.reshape(n * n, *G.shape[2:])
    G = (P[0][None, None, :] @ P[1][None, :, None]) @ P[2][:, None, None]
    return G.reshape(n ** 3, *G.shape[3:])


def grog_lut(coord, nsteps=11):
    """_grog.py:172-182: indexes = round(coord) (float32, half to even); per axis the step
    floor((n - 1) * (index - coord)) + n // 2, combined as sum_a step_a n^a over (x, y, z).
    The shipped code scales by a literal 10, which is n - 1 for the default n = 11."""
    n = 2 * (nsteps // 2) + 1
    c = np.asarray(coord, np.float32)
    idx = np.round(c)
    d = idx - c
    st = np.floor(d * np.float32(n - 1)).astype(np.int64) + n // 2
    w = np.array([1, n, n * n], np.int64)[: c.shape[-1]]
    return idx, (st.reshape(-1, c.shape[-1]) * w).sum(-1)


def grog_interp(input, calib, coord, shape, lamda=0.01, nsteps=11):
    """_preinterp/_grog.py:22-250 with its intent fixes: returns (output, indexes, weights).

    input (..., nc, *coord.shape[:-1]); calib (nc, [nz,] ny, nx) (2D: one operator set per
    calibration slice, the leading input axes being those slices) or (nc, nz, ny, nx) (3D).
    Each sample's coil vector is moved to its nearest grid point by the GRAPPA operator of
    its quantised offset, out = in @ G[lut] (the shipped ``_dot_product``, :406-412, adds
    G[i][j] * in[j], i.e. in * colsum(G); the 3D branch treats the sample axis as a batch
    axis, :205-207).  Indexes are round(coord) + N // 2; weights 1 / (occurrences of each
    flattened index over all samples, before clipping); samples outside the grid are zeroed
    and their indexes clipped (:224-236).
    """
    coord = np.asarray(coord, np.float32)
    ndim = coord.shape[-1]
    shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in list(shape)[-ndim:]]
    cal = np.asarray(calib)
    cal = cal / np.linalg.norm(cal)
    G = grog_table(grog_operators(cal, ndim, lamda), nsteps).astype(np.complex64)
    idx, lut = grog_lut(coord, nsteps)
    x = np.asarray(input, np.complex64)
    M = int(np.prod(coord.shape[:-1]))
    nc = cal.shape[0]
    ishape = x.shape
    rows = np.swapaxes(x.reshape(-1, nc, M), 1, 2)  # (B, M, nc)
    out = np.empty_like(rows)
    nsl = G.shape[1] if ndim == 2 else 1
    if nsl > 1 and rows.shape[0] != nsl:
        raise ValueError("2D GROG with per-slice operators needs one input slice per calibration slice")
    for b in range(rows.shape[0]):
        Gb = (G[:, b if nsl > 1 else 0] if ndim == 2 else G)[lut]
        out[b] = np.einsum("mi,mij->mj", rows[b], Gb)
    out = np.swapaxes(out, 1, 2).reshape(ishape)
    n_xyz = shape[::-1]
    ind = (idx + np.array([s // 2 for s in n_xyz], np.float32)).astype(np.int64)
    unfold = np.array([1, n_xyz[0], n_xyz[0] * (n_xyz[1] if ndim > 1 else 1)], np.int64)[:ndim]
    flat = (ind * unfold).sum(-1).ravel()
    _, inv, counts = np.unique(flat, return_inverse=True, return_counts=True)
    weights = (1.0 / counts[inv].astype(np.float32)).reshape(ind.shape[:-1]).astype(np.float32)
    outside = np.zeros(ind.shape[:-1], bool)
    for a in range(ndim):
        outside |= (ind[..., a] < 0) | (ind[..., a] >= n_xyz[a])
        ind[..., a] = np.clip(ind[..., a], 0, n_xyz[a] - 1)
    out[..., outside] = 0
    return out, ind, weights


# --------------------------------------------------------------------------------------
# FP64 references
# --------------------------------------------------------------------------------------
def pixel_grid(shape_zyx):
    """Centred pixel positions r in [-N//2, N - N//2) per axis, returned in (x, y, z) order."""
    axes = [np.arange(n) - n // 2 for n in shape_zyx]
    mesh = np.meshgrid(*axes, indexing="ij")
    return np.stack(mesh[::-1], axis=-1).reshape(-1, len(shape_zyx)).astype(np.float64)


def nudft_fwd(image, coord, shape_zyx):
    """y_m = sum_r x(r) exp(-2 pi i k_m . r / N) in float64.

    image (..., *N) ; coord (M, d) in cycles/FOV (x, y, z order) -> (..., M).
    """
    r = pixel_grid(shape_zyx)
    n_xyz = np.asarray(shape_zyx[::-1], np.float64)
    ph = -2j * np.pi * (np.asarray(coord, np.float64) / n_xyz) @ r.T  # (M, P)
    E = np.exp(ph)
    x = np.asarray(image).reshape(*image.shape[: image.ndim - len(shape_zyx)], -1).astype(np.complex128)
    return x @ E.T


def nudft_adj(kspace, coord, shape_zyx):
    """x(r) = sum_m y_m exp(+2 pi i k_m . r / N) in float64 (true adjoint of nudft_fwd)."""
    r = pixel_grid(shape_zyx)
    n_xyz = np.asarray(shape_zyx[::-1], np.float64)
    E = np.exp(2j * np.pi * r @ (np.asarray(coord, np.float64) / n_xyz).T)  # (P, M)
    y = np.asarray(kspace).astype(np.complex128)
    return (y @ E.T).reshape(*y.shape[:-1], *shape_zyx)


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
