"""Sparse (Cartesian-subsampled) FFT: ``plan_spfft``, ``sparse_fftn``, ``sparse_ifftn``.

Mirrors src/pyfourier/_sparsefft (``_plan.py:16-146``, ``_fwd.py:17-200``,
``_adj.py:17-200``, ``_sparsefft.py:11-144``) and its masking kernels
(src/pyfourier/_subroutines/_mask/_dense2sparse, _sparse2dense): the forward is
the centred FFT of the image followed by a gather of the sampled grid points
(with the adjoint subspace projection and the B0 segments of the NUFFT), the
adjoint a scatter-add of the samples (duplicates add) followed by the centred
inverse FFT.

That is exactly this package's NUFFT on a plan whose axes are all Cartesian:
integer positions, kernel width 1, no oversampling, unit weights and scale, no
deapodisation (_apod.py:26 skips width-1 axes).  So the plan here is a NUFFT
plan built from ``indexes - shape // 2`` (grid indexes in [0, N) to centred
integer coordinates), and the operators are the library's NUFFT pipelines:
the gather is the interpolation with one tap, the scatter the spread.
Intent fix: the reference maps indexes through ``normalize_coordinates``
(_traj.py:36-53), which divides every point by its own radius; grid indexes in
[0, N) are used as given, and negative entries mark centred coordinates.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from ._nufft import nufft, nufft_adj
from ._plan import _as_tensor, plan_nufft


@dataclass
class FFTPlan:
    """Fields as src/pyfourier/_subroutines/_mask/_plan.py:13-76 (``index`` in (z, y, x)
    order, each (nframes, npts)); ``nufft_plan`` is the device plan that runs it."""

    indexes: object
    dshape: tuple
    ishape: tuple
    ndim: int
    zmap_t_kernel: object
    zmap_s_kernel: object
    zmap_batch_size: int
    nufft_plan: object
    sparse: bool = True

    @property
    def index(self):
        idx = self.indexes.reshape(-1, int(np.prod(self.dshape)), self.ndim).to(torch.int32)
        return tuple(idx[..., a] for a in range(self.ndim))[::-1]

    @property
    def device(self):
        return self.nufft_plan.device

    def to(self, device):
        self.nufft_plan.to(device)
        return self


def plan_spfft(indexes, shape, zmap=None, L=6, nbins=(40, 40), dt=None, T=None, L_batch_size=None, device=None):
    """Precompute a sparse FFT plan (src/pyfourier/_sparsefft/_plan.py:16-146).

    ``indexes``: sampled grid points, (ncontrasts, nviews, nsamples, ndim) or fewer
    leading axes, axes (x, y, z), integer-valued: grid indexes in [0, N) (or centred
    coordinates in [-N/2, N/2) when any entry is negative).  ``shape``: grid size,
    (z, y, x) or a scalar.
    """
    idx = _as_tensor(indexes, torch.float32)
    ndim = int(idx.shape[-1])
    shape = [int(shape)] * ndim if np.isscalar(shape) else [int(s) for s in list(shape)[-ndim:]]
    if not bool(torch.all(idx == torch.round(idx))):
        raise ValueError("Input coordinates must lie on Cartesian grid, got non-uniform coord! "
                         "Please use NUFFT instead.")
    shift = torch.as_tensor([s // 2 for s in shape[::-1]], dtype=torch.float32, device=idx.device)
    coord = idx if bool((idx < 0).any()) else idx - shift
    # every axis is detected Cartesian (width 1, no oversampling); width 2 only keeps beta finite
    plan = plan_nufft(coord, shape, width=2, oversamp=1.0, zmap=zmap, L=L, nbins=nbins, dt=dt, T=T,
                      L_batch_size=L_batch_size, device=device)
    ds = list(idx.shape[:-1])
    while len(ds) < 3:
        ds = [1] + ds
    return FFTPlan(idx.to(plan.device), tuple(ds[1:]), tuple(shape), ndim, plan.zmap_t_kernel, plan.zmap_s_kernel,
                   plan.zmap_batch_size, plan)


def _plan_for(indexes, shape, plan, zmap, L, nbins, dt, T, L_batch_size):
    if plan is None:
        if indexes is None:
            raise ValueError("indexes or plan is required")
        plan = plan_spfft(indexes, shape, zmap, L, nbins, dt, T, L_batch_size)
    return plan


def sparse_fftn(image, indexes=None, shape=None, plan=None, basis=None, zmap=None, L=6, nbins=(40, 40), dt=None,
                T=None, L_batch_size=None, weight=None, norm=None, device="cpu", threadsperblock=128):
    """N-dimensional sparse FFT (src/pyfourier/_sparsefft/_fwd.py:17-200): image
    (..., [ncontrasts], *shape) -> kspace (..., [ncontrasts], nviews, nsamples)."""
    if plan is None and shape is None:
        nd = _as_tensor(indexes).shape[-1]
        shape = tuple(_as_tensor(image).shape[-nd:])
    plan = _plan_for(indexes, shape, plan, zmap, L, nbins, dt, T, L_batch_size)
    return nufft(image, nufft_plan=plan.nufft_plan, basis=basis, weight=weight, norm=norm, device=device,
                 threadsperblock=threadsperblock)


def sparse_ifftn(kspace, indexes=None, shape=None, plan=None, basis=None, zmap=None, L=6, nbins=(40, 40), dt=None,
                 T=None, L_batch_size=None, weight=None, norm=None, device="cpu", threadsperblock=128):
    """N-dimensional inverse sparse FFT (src/pyfourier/_sparsefft/_adj.py:17-200):
    kspace (..., [ncontrasts], nviews, nsamples) -> image (..., [ncontrasts], *shape)."""
    if plan is None and shape is None:
        raise ValueError("shape is required without a plan")
    plan = _plan_for(indexes, shape, plan, zmap, L, nbins, dt, T, L_batch_size)
    return nufft_adj(kspace, nufft_plan=plan.nufft_plan, basis=basis, weight=weight, norm=norm, device=device,
                     threadsperblock=threadsperblock)
