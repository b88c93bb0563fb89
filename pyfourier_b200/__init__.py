"""pyfourier_b200: the NUFFT hot path of pyfourier, B200-native (sm_100a CUDA + cuFFT).

Drop-in entry points (same names, arguments and shape conventions as
pyfourier): ``nufft``, ``nufft_adj``, ``plan_nufft`` / ``NUFFTPlan``,
``plan_spgram`` / ``sparse_gram`` / ``GramMatrix``, ``plan_spfft`` /
``sparse_fftn`` / ``sparse_ifftn``, ``plan_gram`` / ``gram`` (Cartesian
Gram), ``grog_interp`` (GROG pre-interpolation, also as
``_preinterp.grog_interp``), ``pipe_menon_dcf`` (also
as ``pipemenon.pipe_menon_dcf``).  Everything computes in
``libpfb200.so`` through its C ABI (include/pfb200.h); there is no CPU
fallback and importing an operator without the library raises.
"""

from . import _lib
from ._autotune import autotune
from ._b0 import mri_exp_approx
from ._cgram import gram, plan_gram
from ._dcf import pipe_menon_dcf
from ._gram import GramMatrix, plan_spgram, sparse_gram
from ._nufft import nufft, nufft_adj
from ._preinterp import GrogPlan, grog_interp
from ._plan import Interpolator, NUFFTPlan, plan_nufft, release_cached_memory
from ._sparsefft import FFTPlan, plan_spfft, sparse_fftn, sparse_ifftn
from . import pipemenon  # noqa: E402  (module path of the reference: pyfourier.pipemenon)

__version__ = "0.1.0"

__all__ = [
    "nufft", "nufft_adj", "plan_nufft", "NUFFTPlan", "Interpolator",
    "plan_spgram", "sparse_gram", "GramMatrix", "mri_exp_approx", "autotune", "pipe_menon_dcf",
    "pipemenon", "plan_spfft", "sparse_fftn", "sparse_ifftn", "FFTPlan", "plan_gram", "gram",
    "grog_interp", "GrogPlan", "release_cached_memory",
]
