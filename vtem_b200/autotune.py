"""Autotuner for the tensor-core GEMM's output tile width.

``vtb_tc_gemm_bf16_bn`` is built for output tiles of 128 rows by BN columns
with BN in :data:`CANDIDATES` (320: two 160-column accumulators that share
each A tile).  The best BN depends on the problem: the Kronecker Gram of the
decoder has only (Mt + 1)(2 Mt + 1) * 2 columns (306 at Mt = 8), where one
tile across all of them loads every A tile once, while the RF projection has
hundreds of RF columns and many rows.  ``tile_for`` times
every candidate on the caller's own operands (CUDA events, a few launches
each) the first time a shape class (exact column count, row and reduction
lengths rounded to powers of two) is seen, and reuses the choice afterwards;
the choices are kept per process and, when ``VTB_AUTOTUNE_CACHE`` names a file,
in that JSON file across processes.  ``VTB_AUTOTUNE=0`` disables tuning
(BN = 128).  Tuning launches and synchronises, so it must not run inside a
CUDA graph capture: callers run once eagerly before capturing.
"""
from __future__ import annotations

import json
import os
import threading

import torch

from ._abi import call

CANDIDATES = (64, 96, 128, 160, 192, 256, 320)
DEFAULT_BN = 128

_lock = threading.Lock()
_cache = {}
_loaded = False
timings = {}      # shape -> {bn: ms}, for reports


def _bucket(x):
    return max(0, int(x - 1).bit_length())


def _key(M, N, K, out_f64, x3=False):
    """Shape class: the exact column count (the tile waste depends on it) and
    the row and reduction lengths rounded up to powers of two; the
    three-product mode is its own class."""
    k = "%d,%d,%d,%d" % (_bucket(M), N, _bucket(K), int(bool(out_f64)))
    return k + ",x3" if x3 else k


_frozen = threading.local()


class frozen(object):
    """Within this context (per thread) no tuning runs: shapes already tuned
    keep their width, others get DEFAULT_BN.  For concurrent users such as a
    serving loop, where timing launches would both stall and be distorted by
    the other threads' work."""

    def __enter__(self):
        self._prev = getattr(_frozen, "on", False)
        _frozen.on = True
        return self

    def __exit__(self, *exc):
        _frozen.on = self._prev
        return False


def _load():
    global _loaded
    if _loaded:
        return
    _loaded = True
    path = os.environ.get("VTB_AUTOTUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                _cache.update({k: int(v) for k, v in json.load(f).items()})
        except (OSError, ValueError):
            pass


def _save():
    path = os.environ.get("VTB_AUTOTUNE_CACHE")
    if not path:
        return
    try:
        with open(path, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)
    except OSError:
        pass


def tile_for(M, N, K, out_f64, launch, reps=3, x3=False):
    """BN for the GEMM (M x K) @ (N x K)^T; ``launch(bn)`` issues one GEMM
    with tile width bn on the current stream (raising on a bad status)."""
    if os.environ.get("VTB_AUTOTUNE", "1") == "0":
        return DEFAULT_BN
    key = _key(M, N, K, out_f64, x3)
    with _lock:
        _load()
        if key in _cache:
            return _cache[key]
    if torch.cuda.is_current_stream_capturing() or getattr(_frozen, "on", False):
        return DEFAULT_BN
    res = {}
    for bn in CANDIDATES:
        if bn > 2 * max(N, 64) and bn != DEFAULT_BN:
            continue          # wider than twice the problem: only padding
        launch(bn)            # warm-up (kernel attributes, instruction cache)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            launch(bn)
        e1.record()
        e1.synchronize()
        res[bn] = e0.elapsed_time(e1) / reps
    best = min(res, key=res.get)
    with _lock:
        _cache[key] = best
        timings[key] = res
        _save()
    return best


def gemm_bf16_tuned(A3, M, B3, N, K, C, c_m, c_n, out_f64, alpha, accumulate, err_ptr, stream, x3=False):
    """vtb_tc_gemm_bf16_bn (or, with ``x3``, the three-product
    vtb_tc_gemm_bf16x3_bn on [hi | lo] operands, K the width of one part)
    with the tuned tile width for this shape."""
    name = "vtb_tc_gemm_bf16x3_bn" if x3 else "vtb_tc_gemm_bf16_bn"

    def launch(bn):
        call(name, A3, M, B3, N, K, C, c_m, c_n, int(out_f64), float(alpha), int(accumulate), err_ptr, int(bn), stream)

    if accumulate:
        # tuning launches repeatedly: only a non-accumulating GEMM may be tuned
        with _lock:
            _load()
            bn = _cache.get(_key(M, N, K, out_f64, x3), DEFAULT_BN)
    else:
        bn = tile_for(M, N, K, out_f64, launch, x3=x3)
    launch(bn)
    return bn
