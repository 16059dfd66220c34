"""ORACLE (test infrastructure, never shipped or measured as the product).

CPU restatement, in vectorised integer numpy, of the reference's bit-accurate fixed-point PFA
datapath ``mpfs/host/silicon_emulator.py`` (``form_image`` :216-253) and the pieces it imports:

* Q0 quantiser            silicon_emulator.py:226-229, src/fixedpoint.py:19-26 (fit_scale)
* fixed geometry          silicon_emulator.py:131-141
* bracket + Q15 weight    mpfs/host/serialize_inputs.py:67-94 (interp_coeffs)
* 2-tap lerp gather       silicon_emulator.py:60-71 (apply_fixed)
* 32-tap sinc gather      silicon_emulator.py:88-122 (apply_sinc), table gen_resample_vectors.py:206-254
* two-pass resample       silicon_emulator.py:125-156 (resample_fixed)
* Q15 2-D Hamming         silicon_emulator.py:165-195 (window_fixed)
* per-row BFP FFT         src/fixedpoint.py:266-289 (fft1d_bfp_hw_perrow) + renorm silicon_emulator.py:198-205
* detect                  silicon_emulator.py:208-213 (detect_fixed)

All values are carried as int64 real/imag planes, so every step is exact integer arithmetic; the
float64 steps of the reference (coordinate search, fraction, Q15 rounding) are reproduced with the
same float64 operations in the same order.  Pinned against the reference in
``tests/test_oracle_pins.py`` (CRC equality of whole frames and equality of every intermediate).
"""
from __future__ import annotations

import math
import zlib
from fractions import Fraction

import numpy as np

C_LIGHT = 299792458.0
I16_MIN, I16_MAX = -32768, 32767


# ----------------------------------------------------------------------------- small helpers
def sat16(x):
    return np.clip(x, I16_MIN, I16_MAX)


def wrap16(x):
    """C ``(int16_t)`` conversion: keep the low 16 bits, two's complement."""
    x = np.asarray(x, np.int64) & 0xFFFF
    return np.where(x >= 0x8000, x - 0x10000, x)


def frame_crc(img: np.ndarray) -> int:
    """CRC-32 (zlib / IEEE 802.3) of the little-endian uint16 image bytes, C order."""
    return zlib.crc32(np.ascontiguousarray(img, dtype="<u2").tobytes()) & 0xFFFFFFFF


# ----------------------------------------------------------------------------- Q0 quantiser
def q0_exponent(signal: np.ndarray) -> int:
    """Block exponent of ``fit_scale(signal, 16)`` (fixedpoint.py:19-26): ceil(log2(max|.|/32767))."""
    big = max(float(np.abs(signal.real).max()), float(np.abs(signal.imag).max()))
    if big == 0.0:
        return 0
    return math.ceil(math.log2(big / 32767))


def quantize_q0(signal: np.ndarray):
    """silicon_emulator.py:226-229: floor(x / 2^e) in float32, saturate to int16."""
    e = q0_exponent(signal)
    lsb = np.float32(2.0 ** e)
    re = sat16(np.floor(signal.real.astype(np.float32) / lsb)).astype(np.int64)
    im = sat16(np.floor(signal.imag.astype(np.float32) / lsb)).astype(np.int64)
    return re, im, e


# ----------------------------------------------------------------------------- sinc table
def sinc_table_q15(phases: int = 256, taps: int = 32) -> np.ndarray:
    """DC-normalised truncated-sinc polyphase table in Q15 (gen_resample_vectors.py:206-254).

    Exact rationals: each tap is the float64 sin value over the float64 pi times the exact offset,
    normalised by the exact sum and rounded half-up to Q15; then the int16-clamped taps receive the
    unity-gain residual largest-magnitude first, limited by each tap's int16 headroom.
    """
    first = 1 - taps // 2
    pi_q = Fraction(math.pi)
    rows = []
    for ph in range(phases):
        mu = Fraction(ph, phases)
        coef = []
        for t in range(taps):
            d = mu - (first + t)
            coef.append(Fraction(1) if d == 0 else Fraction(math.sin(math.pi * float(d))) / (pi_q * d))
        total = sum(coef)
        q = [math.floor(cf / total * 32768 + Fraction(1, 2)) for cf in coef]
        q = [min(max(v, I16_MIN), I16_MAX) for v in q]
        resid = 32768 - sum(q)
        for t in sorted(range(taps), key=lambda u: -abs(q[u])):
            if resid == 0:
                break
            room = (I16_MAX - q[t]) if resid > 0 else (I16_MIN - q[t])
            step = resid if abs(resid) <= abs(room) else room
            q[t] += step
            resid -= step
        if resid != 0:
            raise ValueError("sinc table cannot reach unity gain within int16")
        rows.append(q)
    return np.asarray(rows, np.int64)


_TAB = None


def _tab():
    global _TAB
    if _TAB is None:
        _TAB = sinc_table_q15()
    return _TAB


# ----------------------------------------------------------------------------- coefficients
def bracket_q15(query, xp):
    """Lower-bound bracket + Q15 weight of a 1-D linear resample (serialize_inputs.py:67-94).

    Returns (idx int64, wq int64): idx in xp's natural order, -1 for queries outside the span.
    """
    xp = np.asarray(xp, np.float64)
    q = np.asarray(query, np.float64)
    n = xp.size
    ascending = xp[-1] >= xp[0]
    xa = xp if ascending else xp[::-1]
    k = np.searchsorted(xa, q, side="left") - 1
    ok = (k >= 0) & (k < n - 1)
    kc = np.clip(k, 0, n - 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        fa = (q - xa[kc]) / (xa[kc + 1] - xa[kc])
    if ascending:
        idx, w = kc, fa
    else:
        idx, w = (n - 2) - kc, 1.0 - fa
    with np.errstate(invalid="ignore"):
        wq = np.clip(np.round(w * 32768.0), 0, 32767)
    idx = np.where(ok, idx, -1).astype(np.int64)
    wq = np.where(ok, wq, 0).astype(np.int64)
    return idx, wq


# ----------------------------------------------------------------------------- gathers
def _lerp_step(d, wq, f32_product):
    """floor((b - a) wq / 2^15).  With ``f32_product`` the product is first rounded to float32, as
    it is in the emulator's pass 1, whose quantised signal is complex64 (silicon_emulator.py:227-229
    make float32 planes, so ``(b.real - a.real) * wq`` at :66 is a float32 multiply)."""
    if f32_product:
        p = d.astype(np.float32) * wq.astype(np.float32)
        return np.floor(p / np.float32(32768.0)).astype(np.int64)
    return (d * wq) >> 15


def gather_lerp(src_re, src_im, idx, wq, f32_product=False):
    """2-tap truncating lerp (silicon_emulator.py:60-71): a + floor((b-a) wq / 2^15), sat16, 0 if idx<0."""
    sn = src_re.shape[-1]
    j = np.clip(idx, 0, sn - 2)
    ar = np.take_along_axis(src_re, j, -1)
    br = np.take_along_axis(src_re, j + 1, -1)
    ai = np.take_along_axis(src_im, j, -1)
    bi = np.take_along_axis(src_im, j + 1, -1)
    rr = sat16(ar + _lerp_step(br - ar, wq, f32_product))
    ri = sat16(ai + _lerp_step(bi - ai, wq, f32_product))
    live = idx >= 0
    return np.where(live, rr, 0), np.where(live, ri, 0)


def gather_sinc(src_re, src_im, idx, wq, sn):
    """32-tap polyphase sinc (silicon_emulator.py:88-122).

    Interior brackets (15 <= idx <= sn-17): sum_t tab[wq>>7][t] x[idx-15+t], round half up (+2^14,
    >>15), sat16.  Other live brackets fall back to the truncating 2-tap lerp; idx<0 gives 0.
    """
    tab = _tab()
    taps, first = 32, -15
    lr, li = gather_lerp(src_re, src_im, idx, wq)
    interior = (idx >= -first) & (idx <= sn - (taps + first))
    if not interior.any():
        return lr, li
    base = np.where(interior, idx + first, 0)                    # window start
    coef = tab[(wq * 256) >> 15]                                  # (..., 32)
    acc_r = np.zeros(idx.shape, np.int64)
    acc_i = np.zeros(idx.shape, np.int64)
    for t in range(taps):
        pos = base + t
        acc_r += coef[..., t] * np.take_along_axis(src_re, pos, -1)
        acc_i += coef[..., t] * np.take_along_axis(src_im, pos, -1)
    sr = sat16((acc_r + (1 << 14)) >> 15)
    si = sat16((acc_i + (1 << 14)) >> 15)
    return np.where(interior, sr, lr), np.where(interior, si, li)


def lagrange_taps_q15(w):
    """4-point cubic Lagrange taps at mu = w / 2^15 in Q15 (gen_resample_vectors.lagrange_taps_q15,
    mpfs/fpga/tb/gen_resample_vectors.py:177-195): exact rationals, one round-half-up per tap.
    Vectorised over integer w; each tap is floor((2 N + D) / (2 D)) with N/D the exact value x 2^15."""
    w = np.asarray(w, np.int64)
    a, b = w + 32768, w - 32768
    c = w - 65536
    nums = (-(w * b * c), a * b * c, -(a * w * c), a * w * b)
    dens = (6 << 30, 1 << 31, 1 << 31, 6 << 30)
    return np.stack([(2 * nn + d) // (2 * d) for nn, d in zip(nums, dens)], -1)


def gather_cubic(src_re, src_im, idx, wq, sn):
    """4-tap cubic Lagrange gather (gen_resample_vectors.gather_cubic, :298-325): taps at idx-1..idx+2
    where 1 <= idx <= sn-3, sum >> 15 (floor), sat16; other live brackets use the integer 2-tap lerp
    (no saturation needed: it stays between its two samples); idx < 0 gives 0."""
    lr, li = gather_lerp(src_re, src_im, idx, wq)
    interior = (idx >= 1) & (idx <= sn - 3)
    if not interior.any():
        return lr, li
    base = np.where(interior, idx - 1, 0)
    coef = lagrange_taps_q15(np.where(interior, wq, 0))
    acc_r = np.zeros(idx.shape, np.int64)
    acc_i = np.zeros(idx.shape, np.int64)
    for t in range(4):
        pos = base + t
        acc_r += coef[..., t] * np.take_along_axis(src_re, pos, -1)
        acc_i += coef[..., t] * np.take_along_axis(src_im, pos, -1)
    return np.where(interior, sat16(acc_r >> 15), lr), np.where(interior, sat16(acc_i >> 15), li)


def _gather(mode, src_re, src_im, idx, wq, sn, f32_product):
    if mode == "sinc":
        return gather_sinc(src_re, src_im, idx, wq, sn)
    if mode == "cubic":
        return gather_cubic(src_re, src_im, idx, wq, sn)
    return gather_lerp(src_re, src_im, idx, wq, f32_product=f32_product)


# ----------------------------------------------------------------------------- geometry
def fixed_geometry(tables: dict, grid: int) -> dict:
    """Per-pulse fixed-point geometry (silicon_emulator.py:131-141), NumPy-2 dtype rules included."""
    ax, ay, freq = tables["ax"], tables["ay"], tables["freq"]
    KR = np.asarray(tables["KR"])
    KC = np.asarray(tables["KC"])
    tan_phi = np.asarray(tables["tan_phi"])
    m, n = freq.shape
    f0 = freq[:, 0].astype(np.float32)
    df = (freq[:, 1] - freq[:, 0]).astype(np.float32)
    mx, my = ax.mean(), ay.mean()
    nrm = math.hypot(mx, my)
    pr = (ax * (mx / nrm) + ay * (my / nrm)).astype(np.float32)
    order = np.argsort(tan_phi)
    tan_s = tan_phi[order].astype(np.float32)
    inv_order = np.argsort(order)
    oob_r = float(KR.max() + (KR.max() - KR.min()) + 1.0)
    oob_c = float(KC.max() + (KC.max() - KC.min()) + 1.0)
    KRp = np.full(grid, oob_r, np.float32)
    KRp[:n] = KR
    KCp = np.full(grid, oob_c, np.float32)
    KCp[:m] = KC
    # pass-1 source scale: f32(f32(2 pr) / f32(c))  (NumPy 2 keeps the python scalars weak)
    fac = (np.float32(2.0) * pr) / np.float32(C_LIGHT)
    return dict(m=m, n=n, grid=grid, f0=f0, df=df, pr=pr, fac=fac, order=order, tan_s=tan_s,
                inv_order=inv_order, KRp=KRp, KCp=KCp)


def pass1_coords(geo: dict, i: int) -> np.ndarray:
    """kr_i[k] = f64(fac_i) * (f64(f0_i) + f64(k) * f64(df_i))  (silicon_emulator.py:144)."""
    n = geo["n"]
    return np.float64(geo["fac"][i]) * (np.float64(geo["f0"][i])
                                        + np.arange(n, dtype=np.float64) * np.float64(geo["df"][i]))


# ----------------------------------------------------------------------------- resample
def resample_two_pass(sig_re, sig_im, geo, range_sinc=False, az_sinc=False, range_mode=None, az_mode=None):
    """resample_fixed (silicon_emulator.py:125-156).

    Returns g2 planes of shape (grid, grid): rows = range bins, cols = cross bins; and the
    pass-1 scratch planes (grid, grid) rows = tan(phi)-sorted pulse slots, cols = range bins.
    ``range_mode`` / ``az_mode`` ("lerp", "sinc", "cubic") override the two booleans; the cubic
    variant is gen_resample_vectors.gather_cubic in both passes (integer edge lerp in pass 1 too).
    """
    rmode = range_mode or ("sinc" if range_sinc else "lerp")
    amode = az_mode or ("sinc" if az_sinc else "lerp")
    m, n, G = geo["m"], geo["n"], geo["grid"]
    if G < m or G < n:
        raise ValueError(f"grid {G} smaller than scene {m}x{n}")
    s1r = np.zeros((G, G), np.int64)
    s1i = np.zeros((G, G), np.int64)
    for i in range(m):
        idx, wq = bracket_q15(geo["KRp"], pass1_coords(geo, i))
        r, im = _gather(rmode, sig_re[i], sig_im[i], idx, wq, n, True)
        s1r[geo["inv_order"][i]] = r
        s1i[geo["inv_order"][i]] = im
    tr = s1r.T
    ti = s1i.T
    g2r = np.zeros((G, G), np.int64)
    g2i = np.zeros((G, G), np.int64)
    for j in range(G):
        src = geo["KRp"][j] * geo["tan_s"]                      # float32 * float32 -> float32
        idx, wq = bracket_q15(geo["KCp"], src)
        row_r = np.ascontiguousarray(tr[j, :m])
        row_i = np.ascontiguousarray(ti[j, :m])
        r, im = _gather(amode, row_r, row_i, idx, wq, m, False)
        g2r[j] = r
        g2i[j] = im
    return g2r, g2i, s1r, s1i


# ----------------------------------------------------------------------------- window
def hamming_q15(length: int, size: int) -> np.ndarray:
    """floor(hamming(length) * 32768) zero-padded to ``size`` (silicon_emulator.py:185-188)."""
    h = np.zeros(size)
    h[:length] = np.hamming(length)
    return np.floor(h * 32768).astype(np.int64)


def window_q15(gr, gi, m, n):
    """window_fixed (silicon_emulator.py:165-195): cw = (int16)((hr_j hc_k) >> 15), out = (int16)((x cw) >> 15)."""
    G0, G1 = gr.shape
    hr = hamming_q15(n, G0)
    hc = hamming_q15(m, G1)
    cw = wrap16((hr[:, None] * hc[None, :]) >> 15)
    return sat16(wrap16((gr * cw) >> 15)), sat16(wrap16((gi * cw) >> 15))


# ----------------------------------------------------------------------------- BFP FFT
def bitrev_perm(n: int) -> np.ndarray:
    bits = n.bit_length() - 1
    p = np.zeros(n, np.int64)
    for b in range(bits):
        p |= ((np.arange(n) >> b) & 1) << (bits - 1 - b)
    return p


def twiddles_q15(n: int):
    """floor(exp(-2 pi j k / n) * 32768) clipped to int16, k < n/2 (fixedpoint.py:277, quant trunc).

    The stage-s table (length 2^(s-1)) equals this length-n/2 table at stride n/2^s: the float64
    angle -2 pi k / 2^s is bit-identical to -2 pi (k n/2^s) / n because the factors are powers of 2.
    """
    w = np.exp(-2j * np.pi * np.arange(n // 2) / n)
    return (np.clip(np.floor(w.real / 2.0 ** -15), I16_MIN, I16_MAX).astype(np.int64),
            np.clip(np.floor(w.imag / 2.0 ** -15), I16_MIN, I16_MAX).astype(np.int64))


def stage_shift(mx):
    """max(0, ceil(log2((mx + 1) / 32767))) evaluated exactly on integers (fixedpoint.py:286)."""
    mx = np.asarray(mx, np.int64)
    sh = np.zeros(mx.shape, np.int64)
    lim = np.full(mx.shape, 32767, np.int64)
    while True:
        over = (mx + 1) > lim
        if not over.any():
            return sh
        sh += over
        lim = np.where(over, lim * 2, lim)


def fft_bfp_rows(xr, xi, tw=None):
    """fft1d_bfp_hw_perrow(x, 16, 16, bitrev) (fixedpoint.py:266-289) on int planes, per row.

    Returns (yr, yi, e_row).
    """
    R, n = xr.shape
    stages = n.bit_length() - 1
    wr_all, wi_all = tw if tw is not None else twiddles_q15(n)
    perm = bitrev_perm(n)
    xr = sat16(xr[:, perm])
    xi = sat16(xi[:, perm])
    e = np.zeros(R, np.int64)
    for s in range(1, stages + 1):
        blk = 1 << s
        half = blk >> 1
        wr = wr_all[:: n // blk][:half]
        wi = wi_all[:: n // blk][:half]
        vr = xr.reshape(R, n // blk, blk)
        vi = xi.reshape(R, n // blk, blk)
        ar, ai = vr[..., :half], vi[..., :half]
        br, bi = vr[..., half:], vi[..., half:]
        tr = sat16((wr * br - wi * bi) >> 15)
        ti = sat16((wr * bi + wi * br) >> 15)
        xr = np.concatenate([ar + tr, ar - tr], axis=-1).reshape(R, n)
        xi = np.concatenate([ai + ti, ai - ti], axis=-1).reshape(R, n)
        mx = np.maximum(np.abs(xr).max(axis=1), np.abs(xi).max(axis=1))
        sh = stage_shift(mx)
        xr = sat16(xr >> sh[:, None])
        xi = sat16(xi >> sh[:, None])
        e += sh
    return xr, xi, e


def fft_pass_raw(xr, xi, tw=None, chunk=1024):
    """The per-row BFP FFTs of fft_pass_bfp before the global renormalisation: (y_re, y_im, e_row)."""
    R, n = xr.shape
    yr = np.empty_like(xr)
    yi = np.empty_like(xi)
    e = np.empty(R, np.int64)
    for r0 in range(0, R, chunk):
        r1 = min(R, r0 + chunk)
        yr[r0:r1], yi[r0:r1], e[r0:r1] = fft_bfp_rows(xr[r0:r1], xi[r0:r1], tw)
    return yr, yi, e


def fft_pass(xr, xi, tw=None, chunk=1024):
    """fft_pass_bfp (silicon_emulator.py:198-205): per-row BFP FFT, then >> (emax - e_row), sat16."""
    yr, yi, e = fft_pass_raw(xr, xi, tw, chunk)
    emax = int(e.max())
    sh = (emax - e)[:, None]
    return sat16(yr >> sh), sat16(yi >> sh), e


# ----------------------------------------------------------------------------- detect
def detect_q(re, im):
    """detect_fixed (silicon_emulator.py:208-213): floor(sqrt(re^2 + im^2)) as uint16."""
    re = sat16(re)
    im = sat16(im)
    mag = np.floor(np.sqrt((re * re + im * im).astype(np.float64)))
    return np.clip(mag, 0, 0xFFFF).astype(np.uint16)


def detect_fused(yr, yi, e):
    """Silicon-order detect (model_detect_fusion.order_B_fused, mpfs/host/model_detect_fusion.py:56-71):
    the magnitude at each row's native exponent, then the (emax - e_row) shift of the magnitude:
    floor(sqrt(re^2 + im^2) / 2^s), clipped to uint16.  For these integer inputs this is
    isqrt(re^2 + im^2) >> s (the float64 sqrt of an integer < 2^53 never rounds across an integer)."""
    emax = int(e.max())
    sh = (emax - e)[:, None]
    mag = np.floor(np.sqrt((yr * yr + yi * yi).astype(np.float64))).astype(np.int64)
    return np.clip(mag >> sh, 0, 0xFFFF).astype(np.uint16)


# ----------------------------------------------------------------------------- whole frame
def form_image(signal, tables, grid, range_sinc=False, az_sinc=False, keep=False, range_mode=None, az_mode=None,
               detect_order="emulator"):
    """The datapath of silicon_emulator.form_image after the CPHD read (:226-249).

    Returns (img uint16 (grid, grid) [range bin][cross bin], diag dict).  Variants for comparison with
    board captures: ``range_mode``/``az_mode`` "cubic" (gen_resample_vectors.gather_cubic) and
    ``detect_order`` "fused" (detect at the native row exponent, model_detect_fusion.order_B_fused).
    """
    sr, si, q0e = quantize_q0(np.asarray(signal, np.complex64))
    geo = fixed_geometry(tables, grid)
    m, n = geo["m"], geo["n"]
    g2r, g2i, s1r, s1i = resample_two_pass(sr, si, geo, range_sinc, az_sinc, range_mode, az_mode)
    wr, wi = window_q15(g2r, g2i, m, n)
    tw = twiddles_q15(grid)
    y1r, y1i, e1 = fft_pass(wr, wi, tw)
    if detect_order == "fused":
        y2r, y2i, e2 = fft_pass_raw(np.ascontiguousarray(y1r.T), np.ascontiguousarray(y1i.T), tw)
        img = np.ascontiguousarray(detect_fused(y2r, y2i, e2).T)
    else:
        y2r, y2i, e2 = fft_pass(np.ascontiguousarray(y1r.T), np.ascontiguousarray(y1i.T), tw)
        img = detect_q(y2r.T, y2i.T)
    diag = dict(q0_exp=q0e, e_range=e1, e_az=e2, geo=geo)
    if keep:
        diag.update(q_re=sr, q_im=si, s1=(s1r, s1i), g2=(g2r, g2i), win=(wr, wi), y1=(y1r, y1i),
                    y2=(y2r, y2i))
    return img, diag
