"""Cartesian (dense) Gram operator: ``plan_gram``, ``gram``.

Mirrors src/pyfourier/_gram (``_plan.py:19-177``, ``_gram.py:11-133``,
``_fwd.py:17-111``): for Cartesian sampling the normal operator A^H A of the
sparse FFT is exactly circulant, so it is an uncentred FFT, a per-voxel product
with the sampling mask (each frame's plane) or, with a subspace basis, with the
K x K matrix sum_t mask_t(v) B[t, k1] conj(B[t, k2]), and the inverse FFT.  It
runs on libpfb200's Gram apply with the grid equal to the image (no embedding).

Intent fixes relative to the shipped reference, which cannot run as written:
* the apply reads ``gram_matrix.st_kernel`` (_gram.py:19, :115-117), a field
  ``GramMatrix`` does not have; here the kernel is ``GramMatrix.value``;
* the mask is given centred (DC at N // 2) and the transform is uncentred, so
  the kernel is the ``ifftshift``-ed mask in both branches (the shipped code
  shifts only the low-rank kernel, with ``fftshift``, _plan.py:133-135);
* with a field map the spatial coefficients C_l are not multiplied into the
  k-space kernel (_plan.py:139-145); as for the Toeplitz Gram there is one
  kernel per time segment, mask_t(k) w_l(T_t(k)), and the apply is
  sum_l conj(C_l) G_l(C_l x) (_gram.py:26-52), with w_l and C_l fitted over the
  pair histogram of the field map.
Only 2D grids (or separable 3D processed as 2D planes), as in the reference
(_plan.py:86-88).
"""

from __future__ import annotations

import numpy as np
import torch

from ._b0 import mri_exp_approx
from ._gram import GramMatrix, sparse_gram
from ._plan import _as_tensor, resolve_device


def _dense_kernel(m, shape, basis, zmap, T, L, nbins):
    """The Gram kernel on ``m``'s device: (value, C_l or None, islowrank).

    value: (nframes, ny, nx) planes, or (ny*nx, K, K) matrices [k2][k1]; with a
    field map a leading segment axis (L, ...)."""
    dev = m.device
    m = m.to(torch.float32)
    if m.ndim == 1:  # (ny,) -> (1, ny, 1) (_plan.py:90-94)
        m = m[None, :, None]
    elif m.ndim == 2:
        m = m[None]
    try:
        m = torch.broadcast_to(m, (m.shape[0], *shape))
    except RuntimeError as e:
        raise ValueError(f"mask planes {tuple(m.shape[1:])} do not broadcast to shape {shape}") from e
    nt = m.shape[0]
    m = torch.fft.ifftshift(m, dim=(-2, -1))  # centred mask -> FFT order
    # per-segment sample weights w_l (L, nt, ny, nx), or one segment of ones
    zs = None
    if zmap is not None:
        if T is None:
            raise ValueError("T (sampling time of every mask point) is required with a field map")
        t = torch.broadcast_to(_as_tensor(T).to(dev, torch.float32), m.shape)
        t = torch.fft.ifftshift(t, dim=(-2, -1)).reshape(-1).cpu().numpy().astype(np.float64)
        tu, inv = np.unique(t, return_inverse=True)  # fit over the distinct sampling times
        bt, zs = mri_exp_approx(_as_tensor(zmap).to(dev), tu, L, nbins, acorr=True)
        wl = torch.as_tensor(bt[:, inv], dtype=torch.complex64, device=dev).reshape(L, *m.shape)
        zs = zs.to(torch.complex64).contiguous()
    else:
        wl = torch.ones((1, *m.shape), dtype=torch.complex64, device=dev)
    mw = wl * m[None].to(torch.complex64)  # (L, nt, ny, nx)
    if basis is not None:
        B = _as_tensor(basis).to(dev, torch.complex64)
        if B.shape[0] != nt:
            raise ValueError("basis needs one row per mask frame")
        # value[l, v, k2, k1] = sum_t mw[l, t, v] B[t, k1] conj(B[t, k2])
        outer = B[:, None, :] * B.conj()[:, :, None]  # (t, k2, k1)
        value = torch.einsum("ltv,tab->lvab", mw.reshape(mw.shape[0], nt, -1), outer)
        islowrank = True
    else:
        value = mw
        islowrank = False
    if zs is None:
        value = value[0]
    return value.to(torch.complex64).contiguous(), zs, islowrank


def plan_gram(mask, shape, basis=None, zmap=None, L=6, nbins=(40, 40), T=None, L_batch_size=None, oversamp=None,
              width=6, device="cpu"):
    """Cartesian Gram kernel (src/pyfourier/_gram/_plan.py:19-157).

    mask: (ncontrasts, ny, nx) sampling mask (non-zero = sampled; values are used
    as weights), centred; (ny, nx) for one frame, (ny,) for (1, ny, 1); planes
    broadcast to ``shape`` (e.g. (ncontrasts, ny, 1)).  shape: (ny, nx).  basis:
    (ncontrasts, K).  With ``zmap``, ``T`` gives the sampling time of every mask
    point (broadcastable to the mask).  ``oversamp`` and ``width`` are accepted for
    compatibility and not used.
    """
    shape = tuple(int(s) for s in shape)
    if len(shape) != 2:
        raise ValueError("we support dense Gram FFT for 2D or separable 3D imaging (i.e., FFT along readout) only")
    m = _as_tensor(mask)
    dev = resolve_device(device, m.device)
    value, zs, islowrank = _dense_kernel(m.to(dev), shape, basis, zmap, T, L, nbins)
    return GramMatrix(value, shape, 2, islowrank, zs, L_batch_size, dev, image_shape=shape)


def gram(image, gram_matrix, norm=None, device="cpu"):
    """Apply the Cartesian Gram (src/pyfourier/_gram/_fwd.py:17-80): image
    (..., [ncontrasts or ncoeff], ny, nx) -> same.  ``norm`` does not change the
    result (the forward and inverse scalings multiply to 1 / (ny nx))."""
    return sparse_gram(image, gram_matrix, norm=norm, device=device)
