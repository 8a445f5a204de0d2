"""Autotuner for the banded-SW launch shape (lanes per pair x cells per lane).

For a band class, every shape whose G*K covers 2*band+1 is installed in turn, the
caller's workload is run, and the banded-SW DP stage time (CUDA events of the
library's stage timer) is read back; the fastest shape stays installed on the
context. Results are cached per (device name, band class) for the process.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable

from . import _abi as A

_CACHE: dict = {}


def shapes() -> list:
    """(lanes per pair, cells per lane) of every launch shape, by index."""
    L = A.lib()
    n = L.kira_gpu_bsw_shapes(None, None, None, 0)
    g = (C.c_int * n)()
    k = (C.c_int * n)()
    L.kira_gpu_bsw_shapes(g, k, None, n)
    return [(int(g[i]), int(k[i])) for i in range(n)]


def packed() -> list:
    """Per shape: True for the packed int16 score lanes."""
    L = A.lib()
    n = L.kira_gpu_bsw_shapes(None, None, None, 0)
    p = (C.c_int * n)()
    L.kira_gpu_bsw_shapes(None, None, p, n)
    return [bool(p[i]) for i in range(n)]


def covering(band: int) -> list:
    need = 2 * max(band, 1) + 1
    return [i for i, (g, k) in enumerate(shapes()) if g * k >= need]


def tune_bsw_shape(ctx, band: int, run_once: Callable[[], None], repeats: int = 3,
                   device_name: str = "") -> dict:
    """Times every covering shape on `run_once` (which must run one verification
    or banded-SW call on `ctx`) and installs the fastest. Returns the timings."""
    key = (device_name, band)
    L = A.lib()
    if key in _CACHE:
        ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, band, _CACHE[key]["best"]))
        return _CACHE[key]
    ctx.check(L.kira_gpu_profile(ctx.handle, 1))
    timings = {}
    try:
        for s in covering(band):
            ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, band, s))
            run_once()  # warm the shape (allocation, module load)
            best = float("inf")
            for _ in range(repeats):
                run_once()
                buf = (C.c_float * 8)()
                n = L.kira_gpu_stage_times(ctx.handle, buf, 8)
                if n > 2:
                    best = min(best, float(buf[2]))
            timings[s] = best
    finally:
        ctx.check(L.kira_gpu_profile(ctx.handle, 0))
    best_shape = min(timings, key=timings.get)
    ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, band, best_shape))
    res = {"best": best_shape, "shape": shapes()[best_shape],
           "dp_ms": {f"{shapes()[s][0]}x{shapes()[s][1]}#{s}": round(t, 4)
                     for s, t in timings.items()}}
    _CACHE[key] = res
    return res
