"""Host logic of bench.py that needs no GPU: the clock sampler against a fake NVML,
the byte accounting of the roofline and the float64 checkers."""

import sys
import time
import types

import numpy as np
import pytest

import bench


def _fake_nvml(reason_bits, clocks=(1965, 1950, 1965)):
    """A stand-in for pynvml: fixed max clock, SM clocks cycling through ``clocks``,
    clock-event reasons ``reason_bits``; the UUID lookup fails (no CUDA device here)
    so the sampler falls back to the device index."""
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    calls = {"init": 0, "by_index": [], "n": 0}

    class NVMLError(Exception):
        pass

    def init():
        calls["init"] += 1

    def by_uuid(u):
        raise NVMLError("no such device")

    def by_index(i):
        calls["by_index"].append(i)
        return ("handle", i)

    def max_clock(h, kind):
        assert kind == nv.NVML_CLOCK_SM
        return 1965

    def clock(h, kind):
        calls["n"] += 1
        return clocks[calls["n"] % len(clocks)]

    nv.NVMLError = NVMLError
    nv.nvmlInit = init
    nv.nvmlDeviceGetHandleByUUID = by_uuid
    nv.nvmlDeviceGetHandleByIndex = by_index
    nv.nvmlDeviceGetMaxClockInfo = max_clock
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reason_bits
    return nv, calls


@pytest.mark.parametrize("bits, names", [
    (0, []),
    (0x4, ["sw_power_cap"]),
    (0x8 | 0x40, ["hw_slowdown", "hw_thermal_slowdown"]),
    (0x20 | 0x80, ["hw_power_brake_slowdown", "sw_thermal_slowdown"]),
    (0x1 | 0x2, []),  # idle / application-clock bits are not slowdowns
])
def test_clock_sampler_nvml(monkeypatch, bits, names):
    nv, calls = _fake_nvml(bits)
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    cs = bench.ClockSampler(3)
    cs.start()
    time.sleep(0.06)
    out = cs.stop()
    assert calls["init"] == 1 and calls["by_index"] == [3]
    assert out["source"].startswith("nvml")
    assert out["sm_max_mhz"] == 1965.0
    assert out["samples"] >= 2 and out["samples"] == calls["n"]
    assert out["sm_mhz"] in (1950.0, 1965.0)
    assert out["reasons"] == names


def test_clock_sampler_without_nvml_or_smi(monkeypatch):
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("driver not loaded")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setenv("PATH", "")
    cs = bench.ClockSampler(0)
    cs.start()
    out = cs.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]


# --------------------------------------------------------------------------------------
# byte accounting and the float64 checkers of the bench (CPU)
# --------------------------------------------------------------------------------------
def _fake_plan(shape, os_shape, M):
    from types import SimpleNamespace

    return SimpleNamespace(ndim=len(shape), shape=tuple(shape), os_shape=tuple(os_shape),
                           interpolator=SimpleNamespace(total_samples=M))


def test_stage_bytes_3d_matches_pass_formulas():
    N, n, M, B = 200, 250, 8_000_000, 32
    sb = bench.stage_bytes(_fake_plan((N, N, N), (n, n, n), M), B)
    e = 8 * B
    assert sb["pad"] == e * (N ** 3 + n * N ** 2)
    assert sb["fft"] == e * (n * N ** 2 + n ** 2 * N)
    assert sb["transpose"] == e * (n ** 2 * N + n ** 3)
    assert sb["ifft"] == e * (n ** 3 + 2 * n ** 2 * N + n * N ** 2)
    assert sb["crop"] == e * (n * N ** 2 + N ** 3)
    coords = M * 20
    assert sb["spread"] == B * M * 8 + B * n ** 3 * 8 + coords
    assert sb["interp"] == sb["spread"]
    assert sb["out"] == sb["vals"] == 2 * B * M * 8


def test_stage_bytes_2d_with_frames_and_segments():
    N, n, M, B, F, L = 192, 240, 500_000, 12, 64, 8
    sb = bench.stage_bytes(_fake_plan((N, N), (n, n), M), B, F, L)
    img, gp = B * F * N * N * 8, B * F * L * 8
    assert sb["fft"] == 0
    assert sb["pad"] == img + gp * N * n
    assert sb["transpose"] == gp * (N * n + n * n)
    assert sb["crop"] == gp * N * n + img
    # channels per sample: coils x segments (frames are groups, not channels)
    assert sb["vals"] == B * M * 8 + B * L * M * 8


def test_nudft_fp64_matches_the_oracle_2d_and_3d():
    import torch

    from oracle import nufft_oracle as orc

    rng = np.random.default_rng(0)
    for shp in [(6, 8, 10), (12, 9)]:
        x = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
        c = ((rng.random((50, len(shp))) - 0.5) * np.array(shp[::-1])).astype(np.float32)
        got = bench.nudft_fwd_fp64(torch, torch.as_tensor(x), c, chunk=17).numpy()
        assert orc.rel_l2(got, orc.nudft_fwd(x, c, shp)) < 1e-12


def test_exact_subspace_normal_operator_matches_the_oracle_definition():
    import torch

    from oracle import nufft_oracle as orc

    rng = np.random.default_rng(1)
    N, F, K = 10, 4, 2
    coord = ((rng.random((F, 3, 7, 2)) - 0.5) * N).astype(np.float32)
    basis = np.linalg.qr(rng.standard_normal((F, K)) + 1j * rng.standard_normal((F, K)))[0].astype(np.complex64)
    x = (rng.standard_normal((K, N, N)) + 1j * rng.standard_normal((K, N, N))).astype(np.complex64)
    got = bench.nudft2_normal_subspace_fp64(torch, torch.as_tensor(x), coord, basis, chunk=5).numpy()
    ref = np.zeros((K, N, N), np.complex128)
    for f in range(F):
        cf = coord[f].reshape(-1, 2)
        yf = sum(basis[f, k] * orc.nudft_fwd(x[k], cf, (N, N)) for k in range(K))
        af = orc.nudft_adj(yf, cf, (N, N))
        for k in range(K):
            ref[k] += np.conj(basis[f, k]) * af
    assert orc.rel_l2(got, ref) < 1e-12


def test_exact_off_resonance_model():
    import torch

    rng = np.random.default_rng(2)
    N = 8
    x = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    b0 = rng.uniform(-200, 200, (N, N))
    c = ((rng.random((30, 2)) - 0.5) * N).astype(np.float32)
    t = rng.uniform(0, 5e-3, 30)
    got = bench.b0_exact_fp64(torch, torch.as_tensor(x), c, t, b0, chunk=7).numpy()
    yy, xx = np.mgrid[:N, :N] - N // 2
    ref = np.array([np.sum(x * np.exp(-2j * np.pi * (c[m, 0] * xx / N + c[m, 1] * yy / N + t[m] * b0)))
                    for m in range(30)])
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
