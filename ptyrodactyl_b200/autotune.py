"""Autotuner for the multislice engine's launch shapes.

For a job geometry (grid edge, slices, probes, modes, kind) it times the candidate
launch configurations on the device — probes per batch and the pass kernels'
register/occupancy variant — and keeps the fastest in a JSON cache keyed by the
geometry and the GPU name, so later calls (the server, the benchmarks) reuse it.
Timing uses CUDA events on the launching stream after a warm-up, median of 3.
"""

from __future__ import annotations

import ctypes
import json
import os
import statistics
import threading
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import torch

from . import _lib
from .simulations import _stream_ptr, ms_params

CACHE_ENV = "PTYRO_B200_TUNE_CACHE"
_DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "ptyrodactyl_b200", "tune.json")
_lock = threading.Lock()
_memo: Dict[str, dict] = {}


@dataclass(frozen=True)
class TuneKey:
    n: int
    num_slices: int
    num_probes: int
    num_modes: int = 1

    def key(self, gpu: str) -> str:
        # probe counts are bucketed to powers of two: the best batch depends on the scale only
        p = 1
        while p < self.num_probes:
            p *= 2
        return f"{gpu}|n{self.n}|s{self.num_slices}|p{p}|m{self.num_modes}"


def _cache_path() -> str:
    return os.environ.get(CACHE_ENV, _DEFAULT_CACHE)


def _load_cache() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(data: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home directory only loses the cache, not the result


def candidates(n: int, num_probes: int, num_modes: int) -> list:
    """(batch, tune) pairs worth timing for this geometry."""
    slot = 8 * n * n * num_modes
    batches = set()
    for mib in (16, 32, 64, 128, 256):
        b = max(1, min(num_probes, (mib << 20) // slot))
        batches.add(b)
    tunes = (0, 3, 19, 83, 147, 211) + ((2259, 6355, 22739) if n == 256 else ()) if n <= 256 else ((3, 259, 771, 2307, 18691) if n == 512 else (0, 3))
    return [(b, t) for b in sorted(batches) for t in tunes]


def tune_forward(slices: torch.Tensor, modes: torch.Tensor, weights: torch.Tensor, positions: torch.Tensor,
                 slice_thickness: float, voltage_kv: float, calib_ang: float, force: bool = False,
                 windows: Optional[torch.Tensor] = None) -> Tuple[int, int]:
    """Best (batch, tune) for this forward geometry, timed on the device on first use."""
    lib = _lib.load()
    dev = slices.device
    n = modes.shape[0]
    key = TuneKey(n, slices.shape[2], positions.shape[0], modes.shape[2]).key(torch.cuda.get_device_name(dev))
    with _lock:
        if not force:
            if key in _memo:
                r = _memo[key]
                return int(r["batch"]), int(r["tune"])
            cache = _load_cache()
            if key in cache:
                _memo[key] = cache[key]
                return int(cache[key]["batch"]), int(cache[key]["tune"])
    results = []
    out = torch.empty((positions.shape[0], n, n), dtype=torch.float32, device=dev)
    st = _stream_ptr(dev)
    f = slices.shape[0]
    for batch, tune in candidates(n, positions.shape[0], modes.shape[2]):
        prm = ms_params(n, slices.shape[2], modes.shape[2], positions.shape[0], voltage_kv, slice_thickness,
                        calib_ang, calib_ang, slices.stride(), modes.stride(), batch, tune, f, windows)
        nbytes = lib.ptyro_ms_workspace_bytes(ctypes.byref(prm))
        try:
            ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        except torch.cuda.OutOfMemoryError:
            continue

        def run():
            _lib.check(lib.ptyro_ms_forward(ctypes.byref(prm), slices.data_ptr(), modes.data_ptr(),
                                            weights.data_ptr(), positions.data_ptr(), out.data_ptr(),
                                            ws.data_ptr(), nbytes, st))

        run()
        ts = []
        for _ in range(3):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            run()
            e.record()
            torch.cuda.synchronize(dev)
            ts.append(s.elapsed_time(e))
        results.append((statistics.median(ts), batch, tune))
        del ws
    if not results:
        raise RuntimeError("autotune: no candidate fits in device memory")
    best = min(results)
    entry = {"batch": best[1], "tune": best[2], "ms": best[0],
             "timings": [[round(t, 4), b, u] for t, b, u in sorted(results)]}
    with _lock:
        _memo[key] = entry
        cache = _load_cache()
        cache[key] = entry
        _store_cache(cache)
    return best[1], best[2]
