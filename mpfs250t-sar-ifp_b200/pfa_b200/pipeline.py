"""The reference's storage-to-storage scene pipeline over the B200 engine
(mpfs/host/sar_pipeline.py:118-163; accel.AccelBackend, mpfs/host/accel.py:23-78).

    *_CPHD.cphd -> [host] CPHD header, PVP and tables (O(m + n))
                -> signal read straight into pinned host memory -> device
                -> [B200] resample, window, 2-D FFT, |z|, display scaling
                -> [host] UTM affine + GeoTIFF (*_detected.tif)

``B200Backend`` is the ``AccelBackend`` of the engine (``focus(signal, tables) -> detected``, float32
|img| on the pow2 raster as ``NumpyBackend.focus`` returns it); ``process_scene`` and ``watch`` mirror the
reference's functions of the same names.  Plans are cached per scene shape, so a queue of same-shaped
scenes allocates once.
"""
from __future__ import annotations

import time
from pathlib import Path

import numpy as np

from . import cphd, geocode, geometry
from .engine import FloatPlan


class B200Backend:
    """accel.AccelBackend over the engine (mpfs/host/accel.py:23-44): float path, lerp passes as
    form_image_pfa, optionally the split-precision tensor-core FFTs (``mixed``)."""
    name = "b200"

    def __init__(self, device: int = 0, mixed: bool = False):
        self.device, self.mixed = device, mixed
        self._plans = {}

    def plan(self, m, n):
        key = (m, n)
        if key not in self._plans:
            self._plans[key] = FloatPlan(m, n, mixed=self.mixed, device=self.device)
        return self._plans[key]

    def focus_device(self, signal, tables):
        """signal: (m, n) complex64 CUDA tensor.  Returns the float32 |img| CUDA tensor."""
        p = self.plan(*tuple(signal.shape))
        p.set_tables(tables)
        return p.form(signal)

    def focus(self, signal, tables):
        import torch
        x = torch.from_numpy(np.ascontiguousarray(signal, np.complex64)).to(f"cuda:{self.device}")
        return self.focus_device(x, tables).cpu().numpy()

    def close(self):
        for p in self._plans.values():
            p.close()
        self._plans.clear()


def make_backend(name: str = "b200", **kw):
    """accel.make_backend (mpfs/host/accel.py:73-78) for the engine's backend."""
    if name != "b200":
        raise ValueError(f"unknown backend {name}")
    return B200Backend(**kw)


def load_scene(cphd_path, deci_pulse=1, deci_sample=1):
    """CPHD header, PVP and tables, and the signal read straight into pinned host memory (the host half
    of sar_pipeline.process_scene, :123-131).  Returns (tables, pinned complex64 torch tensor)."""
    import torch
    with cphd.open_phase_history(cphd_path) as reader:
        meta = reader.cphd_meta
        if meta.Global.DomainType != "FX":
            raise ValueError("expects FX-domain CPHD")
        tables = geometry.prepare_tables_fast(reader, meta, deci_pulse, deci_sample)
        m, n = tables["dims"]
        mu, nu = tables["deci"]
        s0 = tables["samp0"]
        host = torch.empty((m, n), dtype=torch.complex64).pin_memory()
        reader.read_signal_into(host.numpy(), rows=(0, tables["n_vec"], mu), cols=(s0, s0 + n * nu, nu))
    return tables, host


def _out_path(cphd_path, out_dir):
    return Path(out_dir) / (Path(cphd_path).stem.replace("_CPHD", "") + "_detected.tif")


def form_scene(loaded, out_tif, backend, epsg="auto", flip_col=False, flip_row=False, dtype="uint8"):
    """The device half: signal to the device, focus, display scaling, GeoTIFF (:132-148)."""
    import torch
    tables, host = loaded
    sig = host.to(f"cuda:{backend.device}", non_blocking=True)
    mag = backend.focus_device(sig, tables)
    geocode.save_detected_geotiff(mag, tables, out_tif, epsg, flip_col, flip_row, dtype)
    torch.cuda.synchronize()
    return out_tif


def process_scene(cphd_path, out_dir, backend=None, deci_pulse=1, deci_sample=1, epsg="auto",
                  flip_col=False, flip_row=False, dtype="uint8"):
    """One CPHD file to a detected GeoTIFF (sar_pipeline.process_scene, :118-148).  Returns the path."""
    cphd_path, out_dir = Path(cphd_path), Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    backend = backend or B200Backend()
    t0 = time.perf_counter()
    out_tif = form_scene(load_scene(cphd_path, deci_pulse, deci_sample), _out_path(cphd_path, out_dir), backend,
                         epsg, flip_col, flip_row, dtype)
    print(f"  [b200] {cphd_path.name} -> {out_tif.name} ({time.perf_counter() - t0:.2f} s)")
    return out_tif


def watch(in_dir, out_dir, backend=None, poll=5.0, deci_pulse=1, deci_sample=1, once=False, **kw):
    """Batch daemon (sar_pipeline.watch, :151-163): every *_CPHD.cphd dropped into in_dir, once each;
    a failing scene is reported and skipped.  The next file of a sweep is read (CPHD parse, tables,
    signal into pinned memory) on a host thread while the current one is on the device.
    ``once``: one sweep, then return the processed paths."""
    from concurrent.futures import ThreadPoolExecutor
    in_dir, out_dir = Path(in_dir), Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    backend = backend or B200Backend()
    done, outs = set(), []
    with ThreadPoolExecutor(max_workers=1, thread_name_prefix="pfa-cphd-read") as ex:
        while True:
            todo = [f for f in sorted(in_dir.glob("**/*_CPHD.cphd")) if f not in done]
            nxt = ex.submit(load_scene, todo[0], deci_pulse, deci_sample) if todo else None
            for i, f in enumerate(todo):
                t0 = time.perf_counter()
                fut = nxt
                nxt = ex.submit(load_scene, todo[i + 1], deci_pulse, deci_sample) if i + 1 < len(todo) else None
                try:
                    out_tif = form_scene(fut.result(), _out_path(f, out_dir), backend, **kw)
                    print(f"  [b200] {f.name} -> {out_tif.name} ({time.perf_counter() - t0:.2f} s)")
                    outs.append(out_tif)
                except Exception as e:          # keep the queue alive
                    print(f"  !! {f.name} failed: {e}")
                done.add(f)
            if once:
                return outs
            time.sleep(poll)
