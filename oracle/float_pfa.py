"""ORACLE (test infrastructure, never shipped or measured as the product).

CPU restatement of the reference's float PFA focuser ``src/form_image_pfa.py``:

* ``resample_kspace``  form_image_pfa.py:165-222  (two-pass keystone resample with np.interp,
  Hamming window as a float32 outer product)
* ``focus``            form_image_pfa.py:225-240  (zero pad at the top-left to pow2, centred 2-D FFT
  ``fftshift(fft2(ifftshift(.)))`` for SGN<0, :144-147)
* ``detect``           mpfs/host/accel.py:43       (``np.abs(img).astype(float32)``)

``precision="ref"`` reproduces the reference's dtypes (complex64 intermediates, NumPy 2 single
precision FFT).  ``precision="f64"`` runs the same algorithm entirely in float64/complex128 and is the
FP64 oracle that float-mode errors are stated against.

The reference has no float sinc resampler (its 32-tap sinc exists only in fixed point).  The float
sinc variant defined here (``interp="sinc"``) uses the fixed-point table divided by 32768, the phase
``round(frac * 32768) >> 7`` and the interior/edge rule of the fixed-point gather
(mpfs/fpga/tb/gen_resample_vectors.py:257-295, silicon_emulator.py:88-122), with the np.interp
bracket; it is parity-unpinned by the reference beyond that restatement.
"""
from __future__ import annotations

import math

import numpy as np

from . import fixed_emulator as fe

C_LIGHT = 299_792_458.0


def to_pow2(v: int) -> int:
    return 1 << int(math.ceil(math.log2(v)))


def geometry(freq, ax, ay):
    """Shared geometry of resample_kspace (form_image_pfa.py:177-211): kr (m,n), KR, KC, tan_phi, order."""
    m, n = freq.shape
    kmag = 2.0 * freq / C_LIGHT
    dx, dy = ax.mean(), ay.mean()
    dn = math.hypot(dx, dy)
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
    order = np.argsort(tan_phi)
    return dict(m=m, n=n, kr=kr, KR=KR, KC=KC, tan_phi=tan_phi, order=order, pr=pr,
                geo={"dc": 1.0 / (KC[-1] - KC[0]), "dr": 1.0 / (KR[-1] - KR[0]),
                     "dhat": (dx, dy), "chat": (cx, cy)})


def _interp_sinc(x, xp, fp):
    """Float sinc resample of complex fp (ascending xp) at x, zero outside [xp[0], xp[-1]]."""
    tab = fe._tab().astype(np.float64) / 32768.0
    n = xp.size
    k = np.searchsorted(xp, x, side="right") - 1
    live = (x >= xp[0]) & (x <= xp[-1])
    k = np.clip(k, 0, n - 2)
    frac = (x - xp[k]) / (xp[k + 1] - xp[k])
    lin = fp[k] + frac * (fp[k + 1] - fp[k])
    interior = (k >= 15) & (k <= n - 17)
    ph = np.clip(np.round(np.where(live, frac, 0.0) * 32768.0), 0, 32767).astype(np.int64) >> 7
    base = np.where(interior, k - 15, 0)
    cols = base[:, None] + np.arange(32)[None, :]
    acc = (tab[ph] * fp[cols]).sum(axis=1)
    out = np.where(interior, acc, lin)
    return np.where(live, out, 0)


def _interp(x, xp, fp, interp):
    if interp == "sinc":
        return _interp_sinc(x, xp, fp)
    return np.interp(x, xp, fp.real, left=0, right=0) + 1j * np.interp(x, xp, fp.imag, left=0, right=0)


def resample_kspace(sig, freq, ax, ay, precision="ref", interp="lerp", window=True, threads=1):
    """form_image_pfa.resample_kspace restated; returns (g2 (m, n) [cross][range], geom).

    ``threads`` > 1 spreads the per-line loops over a thread pool (the vectorised sinc gather releases
    the GIL); the arithmetic of every line is unchanged."""
    cdt = np.complex64 if precision == "ref" else np.complex128
    g = geometry(freq, ax, ay)
    m, n, kr, KR, KC = g["m"], g["n"], g["kr"], g["KR"], g["KC"]
    sig = np.asarray(sig)
    g1 = np.empty((m, n), cdt)

    def pass1(rows):
        for i in rows:
            xp = kr[i]
            row = sig[i].astype(np.complex128)
            if xp[0] > xp[-1]:
                xp, row = xp[::-1], row[::-1]
            g1[i] = _interp(KR, xp, row, interp)

    order = g["order"]
    tan_s = g["tan_phi"][order]
    g2 = np.empty((m, n), cdt)

    def pass2(cols, g1s):
        for j in cols:
            src = KR[j] * tan_s
            g2[:, j] = _interp(KC, src, g1s[:, j].astype(np.complex128), interp)

    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(pass1, np.array_split(np.arange(m), 4 * threads)))
            g1s = g1[order]
            list(ex.map(lambda c: pass2(c, g1s), np.array_split(np.arange(n), 4 * threads)))
    else:
        pass1(range(m))
        pass2(range(n), g1[order])
    if window:
        if precision == "ref":
            g2 = g2 * np.outer(np.hamming(m), np.hamming(n)).astype(np.float32)
        else:
            g2 = g2 * np.outer(np.hamming(m), np.hamming(n))
    return g2, g


def focus(g2, sgn, precision="ref"):
    """form_image_pfa.focus: top-left zero pad to pow2 then centred 2-D transform (SGN<0 -> fft2)."""
    cdt = np.complex64 if precision == "ref" else np.complex128
    m, n = g2.shape
    m2, n2 = to_pow2(m), to_pow2(n)
    pad = np.zeros((m2, n2), cdt)
    pad[:m, :n] = g2
    fwd = np.fft.fft2 if sgn < 0 else np.fft.ifft2
    return np.fft.fftshift(fwd(np.fft.ifftshift(pad)))


def pfa_image(sig, freq, ax, ay, sgn, precision="ref", interp="lerp", threads=1):
    g2, _ = resample_kspace(sig, freq, ax, ay, precision, interp, threads=threads)
    return focus(g2, sgn, precision)


def detect(img):
    """accel.NumpyBackend.focus detection: |img| as float32 (mpfs/host/accel.py:43)."""
    return np.abs(img).astype(np.float32)


# ----------------------------------------------------------------------------- image metrics
def rel_l2(test, ref):
    test = np.asarray(test, np.complex128 if np.iscomplexobj(test) else np.float64)
    ref = np.asarray(ref, np.complex128 if np.iscomplexobj(ref) else np.float64)
    return float(np.linalg.norm((test - ref).ravel()) / max(np.linalg.norm(ref.ravel()), 1e-300))


def peak_islr(mag, peak_rc, main_half=3, side_half=20):
    """Peak power and integrated sidelobe ratio (dB) of the point response at ``peak_rc`` in |img|.

    Mainlobe: the (2*main_half+1)^2 box at the peak; sidelobes: the rest of the (2*side_half+1)^2 box.
    """
    p = np.asarray(mag, np.float64) ** 2
    r, c = peak_rc
    R, Cc = p.shape
    rows = np.arange(r - side_half, r + side_half + 1) % R
    cols = np.arange(c - side_half, c + side_half + 1) % Cc
    box = p[np.ix_(rows, cols)]
    ctr = side_half
    main = box[ctr - main_half:ctr + main_half + 1, ctr - main_half:ctr + main_half + 1].sum()
    side = box.sum() - main
    return float(p[r, c]), float(10.0 * np.log10(max(side, 1e-300) / max(main, 1e-300)))


def phase_rms(test, ref, mask=None):
    """RMS of the phase difference (rad) over pixels where |ref| is within 20 dB of its peak."""
    test = np.asarray(test)
    ref = np.asarray(ref)
    if mask is None:
        a = np.abs(ref)
        mask = a >= a.max() * 0.1
    d = np.angle(test[mask] * np.conj(ref[mask]))
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


def strongest_peaks(mag, k=64, guard=20):
    """(row, col) of the ``k`` strongest local maxima of ``mag`` (3x3 neighbourhood), at least ``guard``
    pixels from the border so that each one's ISLR box lies inside the image."""
    from scipy.ndimage import maximum_filter
    a = np.asarray(mag, np.float64)
    loc = (a == maximum_filter(a, size=3, mode="nearest")) & (a > 0)
    loc[:guard, :] = loc[-guard:, :] = False
    loc[:, :guard] = loc[:, -guard:] = False
    r, c = np.nonzero(loc)
    top = np.argsort(a[r, c])[::-1][:k]
    return list(zip(r[top].tolist(), c[top].tolist()))


def error_report(test, ref, k=64, main_half=3, side_half=20):
    """Errors of a complex image ``test`` against the FP64 image ``ref`` (same layout):

    * ``rel_l2_complex`` / ``rel_l2_detected``: relative L2 of the complex image and of |img|;
    * ``phase_rms_rad``: RMS phase difference over the pixels within 20 dB of the peak (``phase_rms``);
    * over the ``k`` strongest point responses of |ref| (``strongest_peaks``): the fraction whose peak
      pixel is the same in |test| (3x3 neighbourhood argmax), the largest relative peak-power error and
      the largest ISLR difference in dB (``peak_islr`` with the same boxes).
    """
    test = np.asarray(test)
    ref = np.asarray(ref)
    mt, mr = np.abs(test).astype(np.float64), np.abs(ref).astype(np.float64)
    peaks = strongest_peaks(mr, k=k, guard=side_half)
    same, dp, di = 0, 0.0, 0.0
    for r, c in peaks:
        win = mt[r - 1:r + 2, c - 1:c + 2]
        same += int(np.unravel_index(np.argmax(win), win.shape) == (1, 1))
        p0, i0 = peak_islr(mr, (r, c), main_half, side_half)
        p1, i1 = peak_islr(mt, (r, c), main_half, side_half)
        dp = max(dp, abs(p1 / p0 - 1.0))
        di = max(di, abs(i1 - i0))
    return {"rel_l2_complex": rel_l2(test, ref), "rel_l2_detected": rel_l2(mt, mr),
            "phase_rms_rad": phase_rms(test, ref), "peaks": len(peaks),
            "peak_pos_match": same / max(len(peaks), 1), "peak_power_rel_err_max": dp, "islr_err_db_max": di}
