"""The package has no CPU fallback: a missing library and a machine without a CUDA
device both raise instead of computing anything on the host."""

import os
import subprocess
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_missing_library_raises_import_error():
    # a fresh interpreter: the library object is cached per process once loaded
    code = ("import sys; sys.path.insert(0, sys.argv[1])\n"
            "from pyfourier_b200 import _lib\n"
            "try:\n"
            "    _lib.load('/nonexistent/libpfb200.so')\n"
            "except ImportError as e:\n"
            "    print('ImportError', e)\n")
    p = subprocess.run([sys.executable, "-c", code, ROOT], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.startswith("ImportError") and "no CPU fallback" in p.stdout


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")
def test_operators_without_cuda_raise():
    import pyfourier_b200 as pf

    N = 16
    rng = np.random.default_rng(0)
    coord = ((rng.random((50, 2)) - 0.5) * N).astype(np.float32)
    x = (rng.standard_normal((2, N, N)) + 1j * rng.standard_normal((2, N, N))).astype(np.complex64)
    with pytest.raises(RuntimeError, match="CUDA"):
        pf.nufft(x, coord, (N, N))
    with pytest.raises(RuntimeError, match="CUDA"):
        pf.nufft_adj(np.zeros((2, 50), np.complex64), coord, (N, N))
    with pytest.raises(RuntimeError, match="CUDA"):
        pf.plan_nufft(coord, (N, N))
