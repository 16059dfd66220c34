"""Host-side mirror of the reference's focusing interfaces, over the C ABI.

* ``FixedPlan`` / ``form_image_fixed``: the datapath of ``silicon_emulator.form_image`` after the CPHD
  read (mpfs/host/silicon_emulator.py:226-249), with its knobs ``grid``, ``range_sinc``, ``az_sinc``
  (``--grid --range-sinc --az-sinc``; ``--deci`` is applied by ``prepare_tables``).  Returns the same
  uint16 (grid, grid) image the emulator returns.
* ``FloatPlan`` / ``focus_float``: ``form_image_pfa.pfa`` + detection (src/form_image_pfa.py:243-246,
  mpfs/host/accel.py:39-44).

Device memory and streams come from PyTorch; the arithmetic is entirely in libpfa_b200.so.  Tensors
may be passed directly (CUDA tensors, no copy) or as NumPy arrays (copied in and out).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import geometry


def _torch():
    import torch
    return torch


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _stream_handle(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _frame_ptrs(arrays):
    return (C.c_void_p * max(len(arrays), 1))(*[a.ctypes.data for a in arrays])


def _checked_frames(arrays, shape, dtype, what):
    """Host frames must be C-contiguous with the exact dtype/shape: the library writes through the raw
    pointers, so a silent copy here would lose the caller's output (or its pinned input)."""
    for a in arrays:
        if not isinstance(a, np.ndarray) or a.dtype != dtype or a.shape != shape or not a.flags.c_contiguous:
            raise ValueError(f"{what} frames must be C-contiguous {np.dtype(dtype).name} {shape}")
    return list(arrays)


class _Plan:
    def __init__(self, cfg: _lib.Config):
        self._lib = _lib.load()
        h = C.c_void_p()
        _lib.check(self._lib.pfa_plan_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.cfg = cfg

    @property
    def handle(self):
        return self._h

    @property
    def workspace_bytes(self) -> int:
        return int(self._lib.pfa_plan_workspace_bytes(self._h))

    def set_profiling(self, enable: bool = True):
        _lib.check(self._lib.pfa_set_profiling(self._h, 1 if enable else 0), self._h)

    def stage_times(self) -> dict:
        """{stage name: ms} of the last frame (needs set_profiling(True) before the frame)."""
        ms = (C.c_float * 16)()
        cnt = C.c_int32(0)
        names = C.create_string_buffer(512)
        _lib.check(self._lib.pfa_get_stage_times(self._h, ms, 16, C.byref(cnt), names, 512), self._h)
        keys = names.value.decode().split(",") if cnt.value else []
        return {k: float(ms[i]) for i, k in enumerate(keys)}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pfa_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class FixedPlan(_Plan):
    """Bit-exact fixed-point frame former for an (m, n) scene on a (grid, grid) raster."""

    INTERP = {"lerp": _lib.LERP, "sinc": _lib.SINC, "cubic": _lib.CUBIC}
    DETECT_ORDER = {"emulator": _lib.DETECT_ORDER_EMULATOR, "fused": _lib.DETECT_ORDER_FUSED}

    def __init__(self, m: int, n: int, grid: int, range_sinc: bool = False, az_sinc: bool = False, device: int = 0,
                 range_interp: str | None = None, az_interp: str | None = None, detect_order: str = "emulator"):
        """``range_interp`` / ``az_interp`` ("lerp", "sinc", "cubic") override the two flags; "cubic" and
        ``detect_order="fused"`` are the silicon A/B variants (gen_resample_vectors.gather_cubic,
        model_detect_fusion.order_B_fused)."""
        ri = self.INTERP[range_interp or ("sinc" if range_sinc else "lerp")]
        ai = self.INTERP[az_interp or ("sinc" if az_sinc else "lerp")]
        cfg = _lib.Config(mode=_lib.MODE_FIXED, m=m, n=n, grid=grid, range_interp=ri, az_interp=ai, device=device,
                          detect_order=self.DETECT_ORDER[detect_order])
        super().__init__(cfg)
        self.m, self.n, self.grid, self.device = m, n, grid, device

    def set_tables(self, tables: dict):
        """Upload the job derived from ``prepare_tables`` output (mpfs/host/sar_pipeline.py:36-115)."""
        return self.set_job(self.job_for(tables))

    def job_for(self, tables: dict) -> dict:
        """The job of ``tables`` (host only, no device work: safe on another host thread)."""
        return geometry.fixed_job(tables, self.grid)

    def set_job(self, job: dict):
        inv_order = np.empty(job["m"], np.int32)
        inv_order[job["order"]] = np.arange(job["m"], dtype=np.int32)
        keep = dict(f0=job["f0"], df=job["df"], pr=job["pr"], tan_s=job["tan_s"], inv_order=inv_order,
                    kr=job["krp"], kc=job["kcp"], hr=np.ascontiguousarray(job["hamr"], np.int32),
                    hc=np.ascontiguousarray(job["hamc"], np.int32),
                    tw=np.ascontiguousarray(job["twiddle"], np.int16),
                    sinc=None if job.get("sinc_q15") is None else np.ascontiguousarray(job["sinc_q15"], np.int16))
        fj = _lib.FixedJob(_ptr(keep["f0"]), _ptr(keep["df"]), _ptr(keep["pr"]), _ptr(keep["tan_s"]),
                           _ptr(keep["inv_order"]), _ptr(keep["kr"]), _ptr(keep["kc"]), _ptr(keep["hr"]),
                           _ptr(keep["hc"]), _ptr(keep["tw"]), _ptr(keep["sinc"]))
        _lib.check(self._lib.pfa_set_fixed_job(self._h, C.byref(fj)), self._h)
        self._job = keep

    def form(self, signal, out=None, stream=None):
        """signal: (m, n) complex64 CUDA tensor (or NumPy array).  Returns a uint16 (grid, grid) image
        [range bin][cross bin] -- a CUDA tensor for tensor input, a NumPy array for NumPy input."""
        torch = _torch()
        host = isinstance(signal, np.ndarray)
        sig = torch.from_numpy(np.ascontiguousarray(signal, np.complex64)).to(f"cuda:{self.device}") if host \
            else signal.contiguous()
        if sig.dtype != torch.complex64 or tuple(sig.shape) != (self.m, self.n):
            raise ValueError(f"signal must be complex64 {(self.m, self.n)}, got {sig.dtype} {tuple(sig.shape)}")
        img = out if out is not None else torch.empty((self.grid, self.grid), dtype=torch.uint16, device=sig.device)
        _lib.check(self._lib.pfa_form_fixed(self._h, C.c_void_p(sig.data_ptr()), C.c_void_p(img.data_ptr()),
                                            _stream_handle(stream)), self._h)
        if host:
            return img.cpu().numpy()
        return img

    def form_iq16(self, sig_iq, out=None, stream=None):
        """sig_iq: (m, n, 2) int16 CUDA tensor (quantised I/Q, the board's sig.bin layout)."""
        torch = _torch()
        img = out if out is not None else torch.empty((self.grid, self.grid), dtype=torch.uint16, device=sig_iq.device)
        _lib.check(self._lib.pfa_form_fixed_iq16(self._h, C.c_void_p(sig_iq.data_ptr()), C.c_void_p(img.data_ptr()),
                                                 _stream_handle(stream)), self._h)
        return img

    def form_host(self, signal: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        """End-to-end through host buffers (pfa_form_fixed_host): copy in, form, copy out, sync."""
        sig = np.ascontiguousarray(signal, np.complex64)
        img = out if out is not None else np.empty((self.grid, self.grid), np.uint16)
        _lib.check(self._lib.pfa_form_fixed_host(self._h, _ptr(sig), _ptr(img)), self._h)
        return img

    def form_host_frames(self, signals, outs=None):
        """Pipelined end-to-end frames (pfa_form_fixed_host_frames): uploads, frames and downloads of
        consecutive host frames overlap on three streams.  Pass pinned (page-locked) arrays for full
        PCIe bandwidth.  Returns the list of (grid, grid) uint16 images."""
        sigs = _checked_frames(signals, (self.m, self.n), np.complex64, "signal")
        imgs = outs if outs is not None else [np.empty((self.grid, self.grid), np.uint16) for _ in sigs]
        imgs = _checked_frames(imgs, (self.grid, self.grid), np.uint16, "image")
        if len(imgs) != len(sigs):
            raise ValueError("one output per signal")
        _lib.check(self._lib.pfa_form_fixed_host_frames(self._h, _frame_ptrs(sigs), _frame_ptrs(imgs),
                                                        len(sigs)), self._h)
        return imgs

    def exponents(self):
        """(e_range[n], e_az[grid], q0_exp) of the last frame (fft_pass_bfp's per-row exponents)."""
        er = np.zeros(self.n, np.int32)
        ea = np.zeros(self.grid, np.int32)
        q0 = C.c_int32(0)
        _lib.check(self._lib.pfa_get_fixed_exponents(self._h, _ptr(er), _ptr(ea), C.byref(q0)), self._h)
        return er, ea, int(q0.value)


class FloatPlan(_Plan):
    """Float PFA frame former: form_image_pfa.pfa + detection for an (m, n) scene onto the
    (pow2(m), pow2(n)) raster, rows = cross, cols = range, centred as the reference (or natural)."""

    DETECT = {"mag": _lib.DETECT_MAG, "power": _lib.DETECT_POWER, "complex": _lib.DETECT_COMPLEX}

    def __init__(self, m: int, n: int, range_sinc: bool = False, az_sinc: bool = False, mixed: bool = False,
                 device: int = 0, tile: tuple = (0, 0), test_wait_polls: int = 0):
        """``tile``: complex values per thread of the (cross, range) FFTs, 8, 16 or 32, 0 = the library's
        automatic choice (the autotuner's knob).  ``test_wait_polls``: the test hook of pfa_config (0 in
        normal use)."""
        cfg = _lib.Config(mode=_lib.MODE_MIXED if mixed else _lib.MODE_FLOAT32, m=m, n=n, grid=0,
                          range_interp=_lib.SINC if range_sinc else _lib.LERP,
                          az_interp=_lib.SINC if az_sinc else _lib.LERP, device=device,
                          fft_ept_cross=int(tile[0]), fft_ept_range=int(tile[1]),
                          test_wait_polls=int(test_wait_polls))
        super().__init__(cfg)
        self.m, self.n, self.device, self.tile = m, n, device, tuple(tile)
        self.m2, self.n2 = geometry.pow2(m), geometry.pow2(n)

    def set_tables(self, tables: dict, window: bool = True, centred: bool = True):
        """Upload the job derived from ``prepare_tables`` output (mpfs/host/sar_pipeline.py:36-115)."""
        return self.set_job(self.job_for(tables), window, centred)

    def job_for(self, tables: dict) -> dict:
        """The job of ``tables`` (host only, no device work: safe on another host thread)."""
        return geometry.float_job(tables)

    def set_job(self, job: dict, window: bool = True, centred: bool = True):
        keep = dict(f0=job["f0"], df=job["df"], fl=job["f_last"], pr=job["pr"], tan_s=job["tan_s"],
                    order=job["order"], kr=job["KR"], kc=job["KC"], hm=np.ascontiguousarray(job["ham_m"]),
                    hn=np.ascontiguousarray(job["ham_n"]))
        fj = _lib.FloatJob(_ptr(keep["f0"]), _ptr(keep["df"]), _ptr(keep["fl"]), _ptr(keep["pr"]), _ptr(keep["tan_s"]),
                           _ptr(keep["order"]), _ptr(keep["kr"]), _ptr(keep["kc"]),
                           _ptr(keep["hm"]) if window else None, _ptr(keep["hn"]) if window else None,
                           int(job["sgn"]), _lib.LAYOUT_CENTRED if centred else _lib.LAYOUT_NATURAL)
        _lib.check(self._lib.pfa_set_float_job(self._h, C.byref(fj)), self._h)
        self._job = keep

    def form(self, signal, out=None, detect: str = "mag", stream=None):
        """signal: (m, n) complex64 CUDA tensor (or NumPy array).  Returns (m2, n2) float32 |img|
        (``detect="power"``: |img|^2, ``"complex"``: complex64 img)."""
        torch = _torch()
        host = isinstance(signal, np.ndarray)
        sig = torch.from_numpy(np.ascontiguousarray(signal, np.complex64)).to(f"cuda:{self.device}") if host \
            else signal.contiguous()
        if sig.dtype != torch.complex64 or tuple(sig.shape) != (self.m, self.n):
            raise ValueError(f"signal must be complex64 {(self.m, self.n)}, got {sig.dtype} {tuple(sig.shape)}")
        dt = torch.complex64 if detect == "complex" else torch.float32
        img = out if out is not None else torch.empty((self.m2, self.n2), dtype=dt, device=sig.device)
        _lib.check(self._lib.pfa_form_float(self._h, C.c_void_p(sig.data_ptr()), C.c_void_p(img.data_ptr()),
                                            self.DETECT[detect], _stream_handle(stream)), self._h)
        return img.cpu().numpy() if host else img

    def form_host(self, signal: np.ndarray, out: np.ndarray | None = None, detect: str = "mag") -> np.ndarray:
        sig = np.ascontiguousarray(signal, np.complex64)
        dt = np.complex64 if detect == "complex" else np.float32
        img = out if out is not None else np.empty((self.m2, self.n2), dt)
        _lib.check(self._lib.pfa_form_float_host(self._h, _ptr(sig), _ptr(img), self.DETECT[detect]), self._h)
        return img


    def form_host_frames(self, signals, outs=None, detect: str = "mag"):
        """Pipelined end-to-end frames (pfa_form_float_host_frames); see FixedPlan.form_host_frames."""
        sigs = _checked_frames(signals, (self.m, self.n), np.complex64, "signal")
        dt = np.complex64 if detect == "complex" else np.float32
        imgs = outs if outs is not None else [np.empty((self.m2, self.n2), dt) for _ in sigs]
        imgs = _checked_frames(imgs, (self.m2, self.n2), dt, "image")
        if len(imgs) != len(sigs):
            raise ValueError("one output per signal")
        _lib.check(self._lib.pfa_form_float_host_frames(self._h, _frame_ptrs(sigs), _frame_ptrs(imgs),
                                                        self.DETECT[detect], len(sigs)), self._h)
        return imgs

def form_host_scenes(plan, scenes, prepare, outs=None, **form_kw):
    """A queue of scenes with a new geometry each, through the host-buffer entry point (the reference's
    scene loop, mpfs/host/sar_pipeline.py:151-163).

    ``prepare(scene) -> (tables, signal)`` (CPHD read, ``prepare_tables``) and the job derivation of scene
    i + 1 run on a host thread while scene i is formed: the library call releases the interpreter lock,
    so table preparation leaves the critical path and each scene costs its frame plus the one-copy job
    upload.  ``outs``: output arrays reused in turn (the caller consumes each image before its buffer
    comes round again); default a new array per scene.  Returns the images in scene order."""
    from concurrent.futures import ThreadPoolExecutor

    def stage(sc):
        tables, signal = prepare(sc)
        return plan.job_for(tables), signal

    scenes = list(scenes)
    images = []
    with ThreadPoolExecutor(max_workers=1, thread_name_prefix="pfa-scene-prep") as ex:
        nxt = ex.submit(stage, scenes[0]) if scenes else None
        for i in range(len(scenes)):
            job, signal = nxt.result()
            if i + 1 < len(scenes):
                nxt = ex.submit(stage, scenes[i + 1])
            plan.set_job(job)
            out = outs[i % len(outs)] if outs else None
            images.append(plan.form_host(signal, out, **form_kw))
    return images


def focus_float(signal, tables, range_sinc=False, az_sinc=False, mixed=False, device=0):
    """Drop-in for ``accel.NumpyBackend.focus`` (mpfs/host/accel.py:39-44): float32 |img|."""
    m, n = np.asarray(signal).shape if isinstance(signal, np.ndarray) else tuple(signal.shape)
    with FloatPlan(m, n, range_sinc, az_sinc, mixed, device) as plan:
        plan.set_tables(tables)
        return plan.form(signal)


def form_image_fixed(signal, tables, grid, range_sinc=False, az_sinc=False, device=0):
    """Drop-in for the emulator datapath: ``img = form_image_fixed(signal, tables, grid, rs, az)``
    replaces silicon_emulator.py:226-249 (Q0 quantise .. detect_fixed) and returns the same uint16
    (grid, grid) image."""
    m, n = tables["dims"] if "dims" in tables else np.asarray(signal).shape
    with FixedPlan(m, n, grid, range_sinc, az_sinc, device) as plan:
        plan.set_tables(tables)
        return plan.form(signal)
