"""B0 / R2* time-segmentation basis (plan time, float64).

Restates ``mri_exp_approx`` (src/pyfourier/_subroutines/_b0.py:10-135), the
histogram-weighted least-squares fit of MIRT's mri_exp_approx, with three
intent fixes:

* histogram bin centres are the midpoints of the bin edges (the shipped
  ``ze[1:] - ze[1] / 2`` subtracts half of an edge value);
* the temporal basis fits ``exp(-z t)``, the sign of the spatial coefficients
  ``C_l = exp(-z t_l)`` (the shipped code fits ``exp(+z t)``);
* a real (B0-only) map is histogrammed on its values.

The model approximated is ``exp(-z(r) t) ~= sum_l B_l(t) C_l(r)`` with
``z = 2*pi*(R2* + 1j*B0)`` (a real map is B0 in Hz).
"""

from __future__ import annotations

import math

import numpy as np
import torch


def _pair_histogram(hk, c0, c1=None):
    """Histogram of z(r') + conj(z(r)) over pixel pairs, from the histogram of z:
    differences of the B0 values (an autocorrelation of the histogram) and sums
    of the R2* values (a self-convolution).  Returns (counts, complex values)."""
    if c1 is None:
        h = np.correlate(hk, hk, mode="full")
        zk = 1j * (c0[1] - c0[0]) * np.arange(-(len(c0) - 1), len(c0))
        return h, zk
    n0, n1 = hk.shape
    h = np.zeros((2 * n0 - 1, 2 * n1 - 1))
    for a0, a1 in zip(*np.nonzero(hk)):
        h[a0 - np.arange(n0)[:, None] + n0 - 1, a1 + np.arange(n1)[None, :]] += hk[a0, a1] * hk
    d1 = (c1[1] - c1[0]) if n1 > 1 else 0.0
    zk = 1j * (c0[1] - c0[0]) * np.arange(-(n0 - 1), n0)[:, None] + (2 * c1[0] + d1 * np.arange(2 * n1 - 1))[None, :]
    return h, zk


def mri_exp_approx(zmap, t, lseg=6, bins=(40, 40), mask=None, acorr=False):
    """Return ``(B, C)``: B (lseg, nt) complex128 and C (lseg, *zmap.shape) complex128.

    ``zmap`` and ``t`` may be numpy arrays or torch tensors; B is returned as a
    numpy array, C as a torch tensor on zmap's device (numpy if zmap is numpy).
    ``acorr=True`` fits B over the pair histogram of z(r') + conj(z(r)) instead
    of the histogram of z, the form the Toeplitz Gram needs (the reference
    keeps this branch commented out, src/pyfourier/_subroutines/_b0.py:86-106).
    """
    is_torch = isinstance(zmap, torch.Tensor)
    zt = zmap if is_torch else torch.as_tensor(np.asarray(zmap))
    tt = torch.as_tensor(np.asarray(t.detach().cpu() if isinstance(t, torch.Tensor) else t),
                         dtype=torch.float64)
    if not isinstance(bins, (list, tuple)):
        bins = (bins, 5)
    zc = zt.detach().cpu().numpy()
    if mask is not None:
        mask = np.asarray(mask.detach().cpu() if isinstance(mask, torch.Tensor) else mask, bool)
    if not np.iscomplexobj(zc):
        vals = 2 * math.pi * np.asarray(zc, np.float64)
        vals = vals[mask] if mask is not None else vals.ravel()
        hk, ze = np.histogram(vals, bins=int(bins[0]))
        c0 = 0.5 * (ze[1:] + ze[:-1])
        if acorr:
            hk, zk = _pair_histogram(np.asarray(hk, np.float64), c0)
        else:
            zk = 1j * c0
    else:
        z = 2 * math.pi * np.asarray(zc, np.complex128)
        z = z[mask] if mask is not None else z.ravel()
        hk, e0, e1 = np.histogram2d(z.imag, z.real, bins=[int(bins[0]), int(bins[1])])
        c0, c1 = 0.5 * (e0[1:] + e0[:-1]), 0.5 * (e1[1:] + e1[:-1])
        if acorr:
            hk, zk = _pair_histogram(np.asarray(hk, np.float64), c0, c1)
        else:
            zk = 1j * c0[:, None] + c1[None, :]
    hk = np.asarray(hk, np.float64).ravel()
    zk = np.asarray(zk, np.complex128).ravel()
    t64 = tt.numpy()
    tl = np.linspace(0, lseg, lseg) / lseg * t64[-1]
    ch = np.exp(-tl[:, None] * zk[None, :])  # (L, K)
    w = np.diag(hk ** 0.5)
    p = np.linalg.pinv(w @ ch.T) @ w
    b = p @ np.exp(-zk[:, None] * t64[None, :])  # (L, nt)

    dev = zt.device
    if torch.is_complex(zt):
        z_full = 2 * math.pi * zt.to(torch.complex128)
    else:
        z_full = 2j * math.pi * zt.to(torch.float64)
    tl_t = torch.as_tensor(tl, dtype=torch.float64, device=dev)
    ct = torch.exp(-tl_t.reshape([lseg] + [1] * zt.ndim) * z_full[None])
    ct = torch.nan_to_num(ct, nan=0.0, posinf=0.0, neginf=0.0)
    if not is_torch:
        ct = ct.numpy()
    return b, ct
