"""Plan autotuner.

Chooses, for one plan and one batch shape, the tile extent (the binning of
the samples and the owner tile of the spread) and the number of samples per
spread work item, by timing a forward + adjoint NUFFT on synthetic data with
CUDA events.  The best choice is cached on disk per problem signature (GPU
name, dimensions, oversampled grid, kernel widths, sample count bucket,
frames, batch, coefficients, B0 segments), so later plans of the same problem
reuse it without timing.

Cache file: ``$PYFOURIER_B200_CACHE`` or ``~/.cache/pyfourier_b200/autotune.json``.
"""

from __future__ import annotations

import json
import math
import os
import threading

import torch

_LOCK = threading.Lock()


def cache_path():
    return os.environ.get("PYFOURIER_B200_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "pyfourier_b200", "autotune.json")


def _load_cache():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(cache):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home directory only disables the cache


def signature(plan, batch, ncoeff, nseg):
    ip = plan.interpolator
    mb = int(round(math.log2(max(ip.total_samples, 1))))
    return "|".join([
        torch.cuda.get_device_name(plan.device), f"d{ip.ndim}", "os" + "x".join(map(str, ip.ishape)),
        "w" + "x".join(map(str, ip.width)), f"m2^{mb}", f"f{ip.nframes}", f"b{batch}", f"c{ncoeff}",
        f"l{nseg}"])


def default_candidates(ndim):
    if ndim == 3:
        tiles = [(6, 6, 6), (8, 8, 8), (4, 8, 8), (5, 10, 10)]
    elif ndim == 2:
        tiles = [(16, 16), (24, 24), (32, 32), (16, 64)]
    else:
        tiles = [(64,), (256,), (1024,)]
    # visits per spread work item (a crowded tile is split over interleaved items)
    return tiles, ([2048, 4096, 8192] if ndim == 3 else [1024, 2048, 4096])


def _time_pair(fwd, adj, iters):
    fwd()
    adj()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(iters):
        fwd()
        adj()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / iters


def apply_choice(plan, tile, chunk):
    plan.interpolator.retile(tile)
    plan.interpolator.set_tuning(chunk=chunk)


def autotune(plan, batch=1, basis=None, iters=3, tiles=None, chunks=None, use_cache=True):
    """Tune `plan` in place for `batch` coils (and `basis`, if given) and return
    the chosen ``{"tile": ..., "chunk": ..., "ms": ...}``."""
    from ._nufft import _Ctx, adj_core, fwd_core

    ip = plan.interpolator
    C = basis.shape[1] if basis is not None else ip.nframes
    nseg = plan.zmap_s_kernel.shape[0] if plan.zmap_s_kernel is not None else 1
    key = signature(plan, batch, C, nseg)
    if use_cache:
        with _LOCK:
            hit = _load_cache().get(key)
        if hit is not None:
            apply_choice(plan, tuple(hit["tile"]), int(hit["chunk"]))
            return dict(hit, cached=True)
    d_tiles, d_chunks = default_candidates(ip.ndim)
    tiles = tiles or d_tiles
    chunks = chunks or d_chunks
    dev = plan.device
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.complex(torch.randn(batch, C, *plan.shape, generator=g),
                      torch.randn(batch, C, *plan.shape, generator=g)).to(dev)
    y = torch.complex(torch.randn(batch, ip.total_samples, generator=g),
                      torch.randn(batch, ip.total_samples, generator=g)).to(dev)
    bas = basis.to(dev, torch.complex64).contiguous() if basis is not None else None
    best = None
    for tile in tiles:
        try:
            ip.retile(tile)
        except ValueError:
            continue
        for chunk in chunks:
            ip.set_tuning(chunk=chunk)
            ctx = _Ctx(plan, bas, None, 0)
            ms = _time_pair(lambda: fwd_core(ctx, x), lambda: adj_core(ctx, y), iters)
            if best is None or ms < best["ms"]:
                best = {"tile": list(ip.tile), "chunk": chunk, "ms": ms}
    apply_choice(plan, tuple(best["tile"]), best["chunk"])
    if use_cache:
        with _LOCK:
            cache = _load_cache()
            cache[key] = best
            _save_cache(cache)
    return dict(best, cached=False)
