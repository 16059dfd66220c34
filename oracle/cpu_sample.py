"""ORACLE timing harness (used only by bench.py's cpu_baseline leg and its reference arm).

Times the CPU restatement of the reference's fixed-point datapath (``fixed_emulator``, which follows
mpfs/host/silicon_emulator.py line for line) on a bounded, evenly spaced sample of the lines of every
stage of one frame, and scales each stage to the full frame:

  Q0 quantise      whole signal (cheap)
  pass 1           S of the m pulses                 -> x m/S
  pass 2 + window  S of the G range rows             -> x G/S   (the emulator loops over all G rows)
  FFT-1            S of the G rows (13 BFP stages)   -> x G/S
  FFT-2            S of the G columns                -> x G/S
  detect           S of the G rows                   -> x G/S

The sampled lines are split over ``workers`` spawned processes (one chunk each) when workers > 1.

``fixed_frame_full`` runs the WHOLE frame instead (every pulse, row and column of every stage), with
each stage's lines split over the spawned workers and int16 planes passed between stages, and returns
the uint16 image with its timing: the reference arm's timed step.
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp

import numpy as np

from . import fixed_emulator as fe


def _pass1_chunk(args):
    sr, si, geo, rows, sinc = args          # sr/si hold only the sampled pulses, in `rows` order
    t = time.perf_counter()
    n = geo["n"]
    for r, i in enumerate(rows):
        idx, wq = fe.bracket_q15(geo["KRp"], fe.pass1_coords(geo, i))
        if sinc:
            fe.gather_sinc(sr[r], si[r], idx, wq, n)
        else:
            fe.gather_lerp(sr[r], si[r], idx, wq, f32_product=True)
    return time.perf_counter() - t


def _pass2_chunk(args):
    rowr, rowi, geo, rows, sinc = args
    t = time.perf_counter()
    m, G = geo["m"], geo["grid"]
    hr = fe.hamming_q15(geo["n"], G)
    hc = fe.hamming_q15(m, G)
    for j in rows:
        src = geo["KRp"][j] * geo["tan_s"]
        idx, wq = fe.bracket_q15(geo["KCp"], src)
        if sinc:
            r, i = fe.gather_sinc(rowr, rowi, idx, wq, m)
        else:
            r, i = fe.gather_lerp(rowr, rowi, idx, wq)
        cw = fe.wrap16((hr[j] * hc) >> 15)
        fe.sat16(fe.wrap16((r * cw) >> 15))
        fe.sat16(fe.wrap16((i * cw) >> 15))
    return time.perf_counter() - t


def _fft_chunk(args):
    xr, xi = args
    t = time.perf_counter()
    fe.fft_bfp_rows(xr, xi)
    return time.perf_counter() - t


def _detect_chunk(args):
    xr, xi = args
    t = time.perf_counter()
    fe.detect_q(xr, xi)
    return time.perf_counter() - t


def _full_p1(args):
    sr, si, geo, rows, mode = args          # int16 planes of the chunk's pulses, in `rows` order
    n = geo["n"]
    out_r = np.empty((len(rows), geo["grid"]), np.int16)
    out_i = np.empty_like(out_r)
    for r, i in enumerate(rows):
        idx, wq = fe.bracket_q15(geo["KRp"], fe.pass1_coords(geo, i))
        a, b = fe._gather(mode, sr[r].astype(np.int64), si[r].astype(np.int64), idx, wq, n, True)
        out_r[r], out_i[r] = a, b
    return out_r, out_i


def _full_p2(args):
    tr, ti, geo, rows, mode = args          # int16 range-bin rows of the corner-turned scratch, [:, :m]
    m, n, G = geo["m"], geo["n"], geo["grid"]
    hr = fe.hamming_q15(n, G)
    hc = fe.hamming_q15(m, G)
    out_r = np.empty((len(rows), G), np.int16)
    out_i = np.empty_like(out_r)
    for r, j in enumerate(rows):
        src = geo["KRp"][j] * geo["tan_s"]
        idx, wq = fe.bracket_q15(geo["KCp"], src)
        a, b = fe._gather(mode, tr[r].astype(np.int64), ti[r].astype(np.int64), idx, wq, m, False)
        cw = fe.wrap16((hr[j] * hc) >> 15)                       # window_fixed, row j
        out_r[r] = fe.sat16(fe.wrap16((a * cw) >> 15))
        out_i[r] = fe.sat16(fe.wrap16((b * cw) >> 15))
    return out_r, out_i


def _full_fft(args):
    xr, xi = args
    yr, yi, e = fe.fft_bfp_rows(xr.astype(np.int64), xi.astype(np.int64))
    return yr.astype(np.int16), yi.astype(np.int16), e


def _full_detect(args):
    yr, yi, sh = args                       # FFT-2 rows (cross bins) and their renorm shifts
    return fe.detect_q(fe.sat16(yr.astype(np.int64) >> sh[:, None]), fe.sat16(yi.astype(np.int64) >> sh[:, None]))


def fixed_frame_full(signal, tables, grid, range_sinc=True, az_sinc=True, workers=1, pool=None):
    """One whole fixed-point frame of the oracle (``fixed_emulator.form_image``'s stages, every line),
    each stage split over ``workers`` spawned processes.  Returns (uint16 image [range][cross], dict of
    stage seconds).  The per-line arithmetic is the oracle's; int16 planes carry the stage outputs
    between processes (every stage output is saturated to int16)."""
    stage = {}
    rmode = "sinc" if range_sinc else "lerp"
    amode = "sinc" if az_sinc else "lerp"
    t = time.perf_counter()
    sr, si, _ = fe.quantize_q0(np.asarray(signal, np.complex64))
    sr, si = sr.astype(np.int16), si.astype(np.int16)
    stage["q0"] = time.perf_counter() - t
    geo = fe.fixed_geometry(tables, grid)
    m, n, G = geo["m"], geo["n"], grid
    own = False
    ex = pool
    if workers > 1 and ex is None:
        ex, own = make_pool(workers), True
    mapper = ex.map if workers > 1 else map

    def chunks(count):
        return [c for c in np.array_split(np.arange(count), max(1, 2 * workers)) if len(c)]

    try:
        t = time.perf_counter()
        s1r = np.zeros((G, G), np.int16)
        s1i = np.zeros((G, G), np.int16)
        cs = chunks(m)
        for c, (a, b) in zip(cs, mapper(_full_p1, [(sr[c], si[c], geo, c, rmode) for c in cs])):
            s1r[geo["inv_order"][c]] = a
            s1i[geo["inv_order"][c]] = b
        stage["pass1"] = time.perf_counter() - t
        t = time.perf_counter()
        tr = np.ascontiguousarray(s1r.T[:, :m])
        ti = np.ascontiguousarray(s1i.T[:, :m])
        wr = np.empty((G, G), np.int16)
        wi = np.empty((G, G), np.int16)
        cs = chunks(G)
        for c, (a, b) in zip(cs, mapper(_full_p2, [(tr[c], ti[c], geo, c, amode) for c in cs])):
            wr[c], wi[c] = a, b
        stage["pass2_window"] = time.perf_counter() - t

        def fft_pass(xr, xi):
            yr = np.empty_like(xr)
            yi = np.empty_like(xi)
            e = np.empty(xr.shape[0], np.int64)
            for c, (a, b, ee) in zip(cs, mapper(_full_fft, [(xr[c], xi[c]) for c in cs])):
                yr[c], yi[c], e[c] = a, b, ee
            return yr, yi, e

        t = time.perf_counter()
        y1r, y1i, e1 = fft_pass(wr, wi)
        sh = (int(e1.max()) - e1)[:, None]
        y1r = fe.sat16(y1r.astype(np.int64) >> sh).astype(np.int16)
        y1i = fe.sat16(y1i.astype(np.int64) >> sh).astype(np.int16)
        stage["fft1"] = time.perf_counter() - t
        t = time.perf_counter()
        y2r, y2i, e2 = fft_pass(np.ascontiguousarray(y1r.T), np.ascontiguousarray(y1i.T))
        stage["fft2"] = time.perf_counter() - t
        t = time.perf_counter()
        sh2 = int(e2.max()) - e2
        det = np.empty((G, G), np.uint16)
        for c, d in zip(cs, mapper(_full_detect, [(y2r[c], y2i[c], sh2[c]) for c in cs])):
            det[c] = d
        img = np.ascontiguousarray(det.T)
        stage["detect"] = time.perf_counter() - t
    finally:
        if own:
            ex.shutdown()
    return img, {k: round(v, 4) for k, v in stage.items()}


def make_pool(workers: int):
    """Spawned worker pool for fixed_frame_estimate (reuse it across calls)."""
    return ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn"))


def fixed_frame_estimate(signal, tables, grid, range_sinc=True, az_sinc=True, sample=64, workers=1, seed=0,
                         pool=None):
    """Estimated single-frame time (ms) of the oracle, from `sample` lines per stage."""
    rng = np.random.default_rng(seed)
    stage = {}
    t = time.perf_counter()
    sr, si, _ = fe.quantize_q0(np.asarray(signal, np.complex64))
    stage["q0"] = time.perf_counter() - t
    geo = fe.fixed_geometry(tables, grid)
    m, n, G = geo["m"], geo["n"], grid
    s1 = min(sample, m)
    s2 = min(sample, G)
    p1_rows = np.linspace(0, m - 1, s1).astype(int)
    p2_rows = np.linspace(0, n - 1, s2).astype(int)
    # representative pass-2 source row and FFT operands (timing does not depend on the values)
    rowr = rng.integers(-2000, 2000, m).astype(np.int64)
    rowi = rng.integers(-2000, 2000, m).astype(np.int64)
    fr = rng.integers(-2000, 2000, (s2, G)).astype(np.int64)
    fi = rng.integers(-2000, 2000, (s2, G)).astype(np.int64)

    def split(rows):
        return [c for c in np.array_split(rows, workers) if len(c)]

    own = False
    if workers > 1:
        ex = pool
        if ex is None:
            ex, own = make_pool(workers), True
        run = lambda fn, jobs: max(ex.map(fn, jobs)) if jobs else 0.0   # noqa: E731
    else:
        ex = None
        run = lambda fn, jobs: sum(map(fn, jobs))                          # noqa: E731
    try:
        if ex is not None:          # warm the workers (imports) outside the timed stages
            list(ex.map(_fft_chunk, [(fr[:1, :64], fi[:1, :64])] * workers))
        stage["pass1"] = run(_pass1_chunk, [(sr[c], si[c], geo, c, range_sinc) for c in split(p1_rows)]) * m / s1
        stage["pass2_window"] = run(_pass2_chunk, [(rowr, rowi, geo, c, az_sinc) for c in split(p2_rows)]) * G / s2
        fc = [(fr[c], fi[c]) for c in split(np.arange(s2))]
        stage["fft1"] = run(_fft_chunk, fc) * G / s2
        stage["fft2"] = run(_fft_chunk, fc) * G / s2
        stage["detect"] = run(_detect_chunk, fc) * G / s2
    finally:
        if own:
            ex.shutdown()
    total = sum(stage.values())
    return dict(ms_per_frame=1000.0 * total, stage_seconds={k: round(v, 4) for k, v in stage.items()},
                sample=f"{s1} of {m} pulses, {s2} of {G} rows/columns per FFT/resample stage, "
                       f"scaled to the full frame", workers=workers)


def available_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _float_p1_chunk(args):
    rows, kr, KR = args                      # rows: sampled pulses (complex64), kr: their wavenumbers
    from . import float_pfa as fp
    t = time.perf_counter()
    for r in range(rows.shape[0]):
        xp, row = kr[r], rows[r]
        if xp[0] > xp[-1]:
            xp, row = xp[::-1], row[::-1]
        fp._interp(KR, xp, row, "lerp").astype(np.complex64)
    return time.perf_counter() - t


def _float_p2_chunk(args):
    cols, KRs, tan_s, KC = args              # cols: (S, m) sorted-pulse columns of g1
    from . import float_pfa as fp
    t = time.perf_counter()
    for c in range(cols.shape[0]):
        fp._interp(KC, KRs[c] * tan_s, cols[c], "lerp").astype(np.complex64)
    return time.perf_counter() - t


def _float_fft_chunk(args):
    x = args
    t = time.perf_counter()
    np.fft.fft(x, axis=-1)
    return time.perf_counter() - t


def float_frame_estimate(signal, tables, sample=64, workers=1, pool=None, seed=0):
    """Estimated time (ms) of the reference-precision float PFA (form_image_pfa.resample_kspace + focus
    + |.|, restated in oracle/float_pfa.py) for one frame, from `sample` lines per stage."""
    from . import float_pfa as fp
    rng = np.random.default_rng(seed)
    g = fp.geometry(tables["freq"], tables["ax"], tables["ay"])
    m, n = g["m"], g["n"]
    m2, n2 = fp.to_pow2(m), fp.to_pow2(n)
    s1, s2 = min(sample, m), min(sample, n)
    p1_rows = np.linspace(0, m - 1, s1).astype(int)
    p2_rows = np.linspace(0, n - 1, s2).astype(int)
    cols = (rng.standard_normal((s2, m)) + 1j * rng.standard_normal((s2, m))).astype(np.complex64)
    tan_s = g["tan_phi"][g["order"]]
    fr = (rng.standard_normal((min(sample, m2), n2)) + 1j * rng.standard_normal((min(sample, m2), n2))).astype(np.complex64)
    fc = (rng.standard_normal((min(sample, n2), m2)) + 1j * rng.standard_normal((min(sample, n2), m2))).astype(np.complex64)

    def split(rows):
        return [c for c in np.array_split(rows, workers) if len(c)]

    own = False
    if workers > 1:
        ex = pool
        if ex is None:
            ex, own = make_pool(workers), True
        run = lambda fn, jobs: max(ex.map(fn, jobs)) if jobs else 0.0   # noqa: E731
    else:
        ex = None
        run = lambda fn, jobs: sum(map(fn, jobs))                          # noqa: E731
    stage = {}
    try:
        if ex is not None:
            list(ex.map(_float_fft_chunk, [fr[:1, :64]] * workers))
        stage["pass1"] = run(_float_p1_chunk, [(np.asarray(signal)[c], g["kr"][c], g["KR"]) for c in split(p1_rows)]) * m / s1
        stage["pass2"] = run(_float_p2_chunk, [(cols[c], g["KR"][p2_rows[c]], tan_s, g["KC"]) for c in split(np.arange(s2))]) * n / s2
        t = time.perf_counter()
        _ = np.asarray(signal[:s1]) * np.float32(1.0)                 # window multiply, sampled
        stage["window"] = (time.perf_counter() - t) * m / s1
        stage["fft_rows"] = run(_float_fft_chunk, [fr[c] for c in split(np.arange(fr.shape[0]))]) * m2 / fr.shape[0]
        stage["fft_cols"] = run(_float_fft_chunk, [fc[c] for c in split(np.arange(fc.shape[0]))]) * n2 / fc.shape[0]
        t = time.perf_counter()
        np.abs(fr).astype(np.float32)
        stage["detect"] = (time.perf_counter() - t) * m2 / fr.shape[0]
    finally:
        if own:
            ex.shutdown()
    total = sum(stage.values())
    return dict(ms_per_frame=1000.0 * total, stage_seconds={k: round(v, 4) for k, v in stage.items()},
                sample=f"{s1} of {m} pulses, {s2} of {n} range bins, {fr.shape[0]} of {m2} FFT rows and "
                       f"{fc.shape[0]} of {n2} FFT columns, scaled to the full frame", workers=workers)


# ----------------------------------------------------------------------------- C restatement
_CLIB = None


def _c_oracle():
    """ctypes handle of oracle/lib/libfixed_oracle.so (built by oracle/Makefile)."""
    global _CLIB
    if _CLIB is None:
        import ctypes as C
        from pathlib import Path
        path = Path(__file__).resolve().parent / "lib" / "libfixed_oracle.so"
        if not path.is_file():
            raise RuntimeError(f"{path} not built: run `make -C oracle`")
        lib = C.CDLL(str(path))
        P = C.c_void_p
        lib.pfa_oracle_fixed_frame.restype = C.c_int
        lib.pfa_oracle_fixed_frame.argtypes = [P, C.c_int, C.c_int, C.c_int] + [P] * 12 + [C.c_int] * 3 + [P] * 4
        _CLIB = lib
    return _CLIB


def c_fixed_frame(signal, tables, grid, range_sinc=True, az_sinc=True, threads=0):
    """One whole fixed-point frame of the C restatement (oracle/fixed_frame.c) on ``threads`` host threads
    (0 = all).  Returns (uint16 image [range][cross], dict(q0_exp, e_range, e_az))."""
    import ctypes as C
    lib = _c_oracle()
    sig = np.ascontiguousarray(signal, np.complex64)
    m, n = sig.shape
    geo = fe.fixed_geometry(tables, grid)
    wr, wi = fe.twiddles_q15(grid)
    arrs = [np.ascontiguousarray(a) for a in (
        geo["f0"], geo["df"], geo["fac"], np.asarray(geo["inv_order"], np.int32), geo["tan_s"], geo["KRp"],
        geo["KCp"], fe.hamming_q15(n, grid).astype(np.int32), fe.hamming_q15(m, grid).astype(np.int32),
        wr.astype(np.int32), wi.astype(np.int32), fe._tab().astype(np.int16))]
    img = np.empty((grid, grid), np.uint16)
    e1 = np.empty(grid, np.int32)
    e2 = np.empty(grid, np.int32)
    q0 = np.zeros(1, np.int32)
    ptr = lambda a: C.c_void_p(a.ctypes.data)   # noqa: E731
    st = lib.pfa_oracle_fixed_frame(ptr(sig), m, n, grid, *[ptr(a) for a in arrs], int(bool(range_sinc)),
                                    int(bool(az_sinc)), int(threads), ptr(img), ptr(e1), ptr(e2), ptr(q0))
    if st != 0:
        raise MemoryError("C oracle: host allocation failed")
    return img, dict(q0_exp=int(q0[0]), e_range=e1, e_az=e2)
