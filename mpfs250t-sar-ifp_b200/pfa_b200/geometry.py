"""Host-side FP64 geometry: the tables the PFA engine consumes.

``prepare_tables`` mirrors ``mpfs/host/sar_pipeline.py:36-115`` (same NumPy expressions in the same
order, so its outputs are bit-identical): per-pulse in-plane look vector (ax, ay), the (m, n) RF
frequency table, the uniform output grids KR/KC and tan(phi).  It stays on the CPU in float64, as in the
reference; the engine receives only O(m + n) vectors derived from it.

``fixed_job`` derives the fixed-point job vectors exactly as ``silicon_emulator.resample_fixed`` and
``window_fixed`` do (mpfs/host/silicon_emulator.py:131-141, 185-188), i.e. the board's staged job
(f0, df, pr, sorted tan(phi), pulse permutation, padded KR/KC grids, Q15 tapers; the 10-role DDR
format of mpfs/host/serialize_inputs.py:1-30, with the emulator's floor tapers).

``float_job`` derives the float-mode vectors of ``form_image_pfa.resample_kspace``
(src/form_image_pfa.py:177-211) without materialising the (m, n) wavenumber table: per pulse the
frequency row is affine in the sample index, so its extreme wavenumbers are its end points.
"""
from __future__ import annotations

import functools
import math

import numpy as np

C_LIGHT = 299_792_458.0


def prepare_tables(reader, meta, deci_pulse=1, deci_sample=1, crop_sample=0):
    """sar_pipeline.prepare_tables restated (mpfs/host/sar_pipeline.py:36-115)."""
    mu, nu = max(1, deci_pulse), max(1, deci_sample)
    n_vec, n_samp = reader.get_data_size_as_tuple()[0]
    sgn = int(meta.Global.SGN)
    tx = reader.read_pvp_variable("TxPos", 0)[::mu]
    rcv = reader.read_pvp_variable("RcvPos", 0)[::mu]
    srp = reader.read_pvp_variable("SRPPos", 0)[::mu]
    sc0 = reader.read_pvp_variable("SC0", 0)[::mu]
    scss = reader.read_pvp_variable("SCSS", 0)[::mu]
    apc = 0.5 * (tx + rcv)
    plan = meta.SceneCoordinates.ReferenceSurface.Planar
    uiax = np.array([plan.uIAX.X, plan.uIAX.Y, plan.uIAX.Z])
    uiay = np.array([plan.uIAY.X, plan.uIAY.Y, plan.uIAY.Z])
    los = srp - apc
    u = los / np.linalg.norm(los, axis=1, keepdims=True)
    ax = u @ uiax
    ay = u @ uiay
    m = len(range(0, n_vec, mu))
    n = len(range(0, n_samp, nu))
    d0 = 0
    if crop_sample and crop_sample < n:
        d0 = (n - crop_sample) // 2
        n = crop_sample
    samp0 = d0 * nu
    k = d0 + np.arange(n)
    freq = sc0[:, None] + k[None, :] * (scss[:, None] * nu)
    kmag = 2.0 * freq / C_LIGHT
    dx, dy = ax.mean(), ay.mean()
    dn = np.hypot(dx, dy)
    dx, dy = dx / dn, dy / dn
    cx, cy = -dy, dx
    pr = ax * dx + ay * dy
    pc = ax * cx + ay * cy
    kr = kmag * pr[:, None]
    tan_phi = pc / pr
    kr_lo, kr_hi = kr.max(axis=1).min(), kr.min(axis=1).max()
    if kr_lo > kr_hi:
        kr_lo, kr_hi = kr.min(), kr.max()
    KR = np.linspace(kr_lo, kr_hi, n)
    kc_max = np.abs(KR[:, None] * tan_phi[None, :]).max()
    KC = np.linspace(-kc_max, kc_max, m)
    window = np.outer(np.hamming(m), np.hamming(n)).astype(np.float32)
    geo = {"dc": 1.0 / (KC[-1] - KC[0]), "dr": 1.0 / (KR[-1] - KR[0]),
           "dhat": (dx, dy), "chat": (cx, cy)}
    return {"ax": ax, "ay": ay, "freq": freq, "sgn": sgn, "KR": KR, "KC": KC, "tan_phi": tan_phi,
            "window": window, "geo": geo, "center_ecef": srp[0], "uiax": uiax, "uiay": uiay,
            "dims": (m, n), "deci": (mu, nu), "n_vec": n_vec, "n_samp": n_samp, "samp0": samp0}


class AffineFreq:
    """The (m, n) RF frequency table of prepare_tables, freq[i, k] = sc0_i + k * step_i (k = k0 + column),
    without materialising it: columns and rows are computed on demand with the same float64 operations
    as the NumPy broadcast (so every element is bit-identical), ``np.asarray`` builds the full array."""

    def __init__(self, sc0: np.ndarray, step: np.ndarray, k0: int, n: int):
        self.sc0 = np.asarray(sc0, np.float64)
        self.step = np.asarray(step, np.float64)
        self.k0, self.n = int(k0), int(n)
        self.shape = (len(self.sc0), self.n)
        self.ndim, self.dtype = 2, np.dtype(np.float64)

    def column(self, c: int) -> np.ndarray:
        c = c + self.n if c < 0 else c
        return self.sc0 + np.float64(self.k0 + c) * self.step

    def __getitem__(self, idx):
        if isinstance(idx, tuple) and len(idx) == 2 and idx[0] == slice(None) and isinstance(idx[1], (int, np.integer)):
            return self.column(int(idx[1]))
        return np.asarray(self)[idx]

    def __array__(self, dtype=None, copy=None):
        k = self.k0 + np.arange(self.n)
        a = self.sc0[:, None] + k[None, :] * self.step[:, None]
        return a if dtype is None else a.astype(dtype)


def prepare_tables_fast(reader, meta, deci_pulse=1, deci_sample=1, crop_sample=0):
    """prepare_tables in O(m + n) with bit-identical outputs (mpfs/host/sar_pipeline.py:36-115).

    The reference materialises (m, n) float64 arrays (freq, 2 freq / c, kr, KR x tan(phi)) only to take
    row extremes and a global max.  Every one of them is monotone: fl(k * step) and fl(sc0 + x) are
    monotone in k, so are fl(2 f / c) and fl(kmag * pr), hence each pulse's kr extremes are its end
    samples; and fl(|a| |b|) is monotone in both factors, hence max |KR x tan(phi)| is the rounded product
    of the two largest magnitudes.  ``freq`` is returned as an ``AffineFreq`` view; the (m, n) float32
    window of the reference is not built (the engine applies the two Hamming tapers on the fly).
    """
    mu, nu = max(1, deci_pulse), max(1, deci_sample)
    n_vec, n_samp = reader.get_data_size_as_tuple()[0]
    sgn = int(meta.Global.SGN)
    tx = reader.read_pvp_variable("TxPos", 0)[::mu]
    rcv = reader.read_pvp_variable("RcvPos", 0)[::mu]
    srp = reader.read_pvp_variable("SRPPos", 0)[::mu]
    sc0 = reader.read_pvp_variable("SC0", 0)[::mu]
    scss = reader.read_pvp_variable("SCSS", 0)[::mu]
    apc = 0.5 * (tx + rcv)
    plan = meta.SceneCoordinates.ReferenceSurface.Planar
    uiax = np.array([plan.uIAX.X, plan.uIAX.Y, plan.uIAX.Z])
    uiay = np.array([plan.uIAY.X, plan.uIAY.Y, plan.uIAY.Z])
    los = srp - apc
    u = los / np.linalg.norm(los, axis=1, keepdims=True)
    ax = u @ uiax
    ay = u @ uiay
    m = len(range(0, n_vec, mu))
    n = len(range(0, n_samp, nu))
    d0 = 0
    if crop_sample and crop_sample < n:
        d0 = (n - crop_sample) // 2
        n = crop_sample
    samp0 = d0 * nu
    freq = AffineFreq(sc0, scss * nu, d0, n)
    dx, dy = ax.mean(), ay.mean()
    dn = np.hypot(dx, dy)
    dx, dy = dx / dn, dy / dn
    cx, cy = -dy, dx
    pr = ax * dx + ay * dy
    pc = ax * cx + ay * cy
    tan_phi = pc / pr
    ka = (2.0 * freq.column(0) / C_LIGHT) * pr
    kb = (2.0 * freq.column(n - 1) / C_LIGHT) * pr
    rmax, rmin = np.maximum(ka, kb), np.minimum(ka, kb)
    kr_lo, kr_hi = rmax.min(), rmin.max()
    if kr_lo > kr_hi:
        kr_lo, kr_hi = rmin.min(), rmax.max()
    KR = np.linspace(kr_lo, kr_hi, n)
    kc_max = np.abs(KR[np.argmax(np.abs(KR))] * tan_phi[np.argmax(np.abs(tan_phi))])
    KC = np.linspace(-kc_max, kc_max, m)
    geo = {"dc": 1.0 / (KC[-1] - KC[0]), "dr": 1.0 / (KR[-1] - KR[0]),
           "dhat": (dx, dy), "chat": (cx, cy)}
    return {"ax": ax, "ay": ay, "freq": freq, "sgn": sgn, "KR": KR, "KC": KC, "tan_phi": tan_phi,
            "geo": geo, "center_ecef": srp[0], "uiax": uiax, "uiay": uiay,
            "dims": (m, n), "deci": (mu, nu), "n_vec": n_vec, "n_samp": n_samp, "samp0": samp0}


def prepare_tables_from_scene_fast(scene, deci=1):
    from .synth import FakeReader
    rd = FakeReader(scene)
    return prepare_tables_fast(rd, rd.cphd_meta, deci, deci)


def prepare_tables_from_scene(scene, deci=1):
    from .synth import FakeReader
    rd = FakeReader(scene)
    return prepare_tables(rd, rd.cphd_meta, deci, deci)


def pow2(v: int) -> int:
    return 1 << int(math.ceil(math.log2(max(int(v), 1))))


@functools.lru_cache(maxsize=64)
def hamming_q15_floor(length: int, size: int) -> np.ndarray:
    """floor(hamming(length) * 32768) zero-padded to ``size`` (int32; the odd-length centre is 32768).
    Cached per (length, size): a queue of same-shaped scenes builds it once (read-only array)."""
    h = np.zeros(size)
    h[:length] = np.hamming(length)
    out = np.floor(h * 32768).astype(np.int32)
    out.flags.writeable = False
    return out


@functools.lru_cache(maxsize=16)
def twiddles_q15(n: int) -> np.ndarray:
    """(n/2, 2) int16: floor(exp(-2 pi j k/n) * 32768) clipped to int16 (src/fixedpoint.py:277).
    Cached per n (read-only array)."""
    w = np.exp(-2j * np.pi * np.arange(n // 2) / n)
    out = np.empty((n // 2, 2), np.int16)
    out[:, 0] = np.clip(np.floor(w.real / 2.0 ** -15), -32768, 32767)
    out[:, 1] = np.clip(np.floor(w.imag / 2.0 ** -15), -32768, 32767)
    out.flags.writeable = False
    return out


def fixed_job(tables: dict, grid: int) -> dict:
    """Fixed-point job vectors, exactly as silicon_emulator.resample_fixed/window_fixed build them."""
    ax, ay, freq = tables["ax"], tables["ay"], tables["freq"]
    KR = np.asarray(tables["KR"])
    KC = np.asarray(tables["KC"])
    tan_phi = np.asarray(tables["tan_phi"])
    m, n = freq.shape
    if grid < m or grid < n:
        raise ValueError(f"grid {grid} must be >= the scene dims {m}x{n}")
    f0 = freq[:, 0].astype(np.float32)
    df = (freq[:, 1] - freq[:, 0]).astype(np.float32)
    dx, dy = ax.mean(), ay.mean()
    dn = math.hypot(dx, dy)
    pr = (ax * (dx / dn) + ay * (dy / dn)).astype(np.float32)
    order = np.argsort(tan_phi)
    tan_s = tan_phi[order].astype(np.float32)
    oob_r = float(KR.max() + (KR.max() - KR.min()) + 1.0)
    oob_c = float(KC.max() + (KC.max() - KC.min()) + 1.0)
    krp = np.full(grid, oob_r, np.float32)
    krp[:n] = KR
    kcp = np.full(grid, oob_c, np.float32)
    kcp[:m] = KC
    return dict(m=m, n=n, grid=grid,
                f0=np.ascontiguousarray(f0), df=np.ascontiguousarray(df), pr=np.ascontiguousarray(pr),
                tan_s=np.ascontiguousarray(tan_s), order=order.astype(np.int32),
                krp=krp, kcp=kcp,
                hamr=hamming_q15_floor(n, grid), hamc=hamming_q15_floor(m, grid),
                twiddle=twiddles_q15(grid))


def float_job(tables: dict) -> dict:
    """Float-mode vectors of form_image_pfa.resample_kspace (src/form_image_pfa.py:177-217).

    f0/df describe each pulse's frequency row (freq[i, k] = f0_i + k df_i, as prepare_tables builds it);
    pr is the radial projection; KR/KC, tan(phi) order and the two Hamming tapers are computed as the
    reference computes them.
    """
    ax, ay, freq = tables["ax"], tables["ay"], tables["freq"]
    m, n = freq.shape
    f0 = np.ascontiguousarray(freq[:, 0], np.float64)
    df = np.ascontiguousarray((freq[:, -1] - freq[:, 0]) / max(n - 1, 1), np.float64)
    dx, dy = ax.mean(), ay.mean()
    dn = math.hypot(dx, dy)
    dx, dy = dx / dn, dy / dn
    cx, cy = -dy, dx
    pr = ax * dx + ay * dy
    pc = ax * cx + ay * cy
    tan_phi = pc / pr
    # kr[i, k] = (2 freq[i, k] / c) pr_i is monotone in k, so its row extremes are the end points
    ka = (2.0 * freq[:, 0] / C_LIGHT) * pr
    kb = (2.0 * freq[:, -1] / C_LIGHT) * pr
    rmax, rmin = np.maximum(ka, kb), np.minimum(ka, kb)
    kr_lo, kr_hi = rmax.min(), rmin.max()
    if kr_lo > kr_hi:
        kr_lo, kr_hi = rmin.min(), rmax.max()
    KR = np.asarray(tables.get("KR", np.linspace(kr_lo, kr_hi, n)), np.float64)
    kc_max = max(abs(KR[0]), abs(KR[-1])) * np.abs(tan_phi).max()
    KC = np.asarray(tables.get("KC", np.linspace(-kc_max, kc_max, m)), np.float64)
    order = np.argsort(tan_phi)
    f_last = np.ascontiguousarray(freq[:, -1], np.float64)
    return dict(m=m, n=n, m2=pow2(m), n2=pow2(n), f0=f0, df=df, f_last=f_last, pr=np.ascontiguousarray(pr),
                tan_s=np.ascontiguousarray(tan_phi[order]), order=order.astype(np.int32),
                KR=np.ascontiguousarray(KR), KC=np.ascontiguousarray(KC),
                ham_m=np.hamming(m), ham_n=np.hamming(n), sgn=int(tables.get("sgn", -1)))
