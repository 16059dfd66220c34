"""Project autotuner for the float engine.

The tunable tile of the float path is the FFT register tile: complex values per thread of the cross
FFT (fused with pass 2) and of the range FFT, 8, 16 or 32, which sets the CTA size (line length / tile)
and so the register/occupancy/barrier trade-off.  ``tune_float`` times every candidate on the device
for one scene shape (CUDA events, median of ``reps`` frames after a warm-up) and returns the fastest.
Results are cached per (pow2 m, pow2 n, interpolators) in memory and in a JSON file
(``PFA_TUNE_CACHE``, default ``~/.cache/pfa_b200/tune.json``); pass ``use_cache=False`` to re-measure.
"""
from __future__ import annotations

import json
import os
import statistics
from pathlib import Path

from .engine import FloatPlan
from .geometry import pow2

CANDIDATES = ((16, 16), (8, 16), (16, 8), (8, 8), (16, 32))
_MEM: dict = {}


def _cache_path() -> Path:
    return Path(os.environ.get("PFA_TUNE_CACHE", Path.home() / ".cache" / "pfa_b200" / "tune.json"))


def _key(m, n, range_sinc, az_sinc) -> str:
    return f"{pow2(m)}x{pow2(n)}:{'s' if range_sinc else 'l'}{'s' if az_sinc else 'l'}"


def _load():
    p = _cache_path()
    if not _MEM and p.is_file():
        try:
            _MEM.update(json.loads(p.read_text()))
        except (OSError, ValueError):
            pass


def _store():
    p = _cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(json.dumps(_MEM, indent=1))
    except OSError:
        pass


def tune_float(tables, signal, range_sinc=False, az_sinc=False, device=0, candidates=CANDIDATES, reps=5,
               use_cache=True):
    """Fastest (cross, range) FFT tile for this scene shape.  signal: (m, n) complex64 CUDA tensor.
    Returns (tile, {tile: ms})."""
    import torch
    m, n = tuple(signal.shape)
    key = _key(m, n, range_sinc, az_sinc)
    if use_cache:
        _load()
        if key in _MEM:
            hit = _MEM[key]
            return tuple(hit["tile"]), {tuple(map(int, k.split(","))): v for k, v in hit["ms"].items()}
    times = {}
    for tile in candidates:
        with FloatPlan(m, n, range_sinc, az_sinc, device=device, tile=tile) as plan:
            plan.set_tables(tables)
            img = torch.empty((plan.m2, plan.n2), dtype=torch.float32, device=signal.device)
            plan.form(signal, out=img)
            torch.cuda.synchronize()
            samples = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                plan.form(signal, out=img)
                e1.record()
                torch.cuda.synchronize()
                samples.append(e0.elapsed_time(e1))
            times[tuple(tile)] = statistics.median(samples)
    best = min(times, key=times.get)
    _MEM[key] = {"tile": list(best), "ms": {f"{a},{b}": v for (a, b), v in times.items()}}
    _store()
    return best, times
