"""Constant tables of the PFA engine.

``sinc_table_q15`` builds the 256-phase x 32-tap polyphase sinc table of the reference's resampler
(mpfs/fpga/tb/gen_resample_vectors.py:206-254; consumed by silicon_emulator.apply_sinc :88-122).  The
table must be bit-identical, so the recipe is the reference's: exact rational taps from the float64
``math.sin`` value and the float64 ``math.pi``, exact DC normalisation, round-half-up to Q15, then the
unity-gain residual spread over the int16-clamped taps, largest magnitude first.  The build writes it
into the library as a C array (``write_c_include``).
"""
from __future__ import annotations

import math
from fractions import Fraction
from pathlib import Path

import numpy as np

PHASES = 256
TAPS = 32


def sinc_table_q15(phases: int = PHASES, taps: int = TAPS) -> np.ndarray:
    first = -(taps // 2 - 1)
    pi_exact = Fraction(math.pi)
    out = np.zeros((phases, taps), np.int16)
    for ph in range(phases):
        mu = Fraction(ph, phases)
        offs = [mu - (first + t) for t in range(taps)]
        taps_q = [Fraction(1) if d == 0 else Fraction(math.sin(math.pi * float(d))) / (pi_exact * d) for d in offs]
        norm = sum(taps_q)
        q = []
        for c in taps_q:
            v = c * 32768 / norm + Fraction(1, 2)
            q.append(min(32767, max(-32768, v.numerator // v.denominator)))
        rest = 32768 - sum(q)
        for t in sorted(range(taps), key=lambda i: (-abs(q[i]), i)):
            if rest == 0:
                break
            head = (32767 - q[t]) if rest > 0 else (-32768 - q[t])
            step = rest if abs(rest) <= abs(head) else head
            q[t] += step
            rest -= step
        if rest:
            raise ValueError("sinc phase %d cannot reach unity gain within int16" % ph)
        out[ph] = q
    return out


def write_c_include(path: Path) -> None:
    tab = sinc_table_q15()
    rows = []
    for ph in range(tab.shape[0]):
        rows.append("    " + ", ".join(str(int(v)) for v in tab[ph]) + ",")
    text = ("// Generated by pfa_b200/tables.py (write_c_include): 256 x 32 Q15 polyphase sinc.\n"
            "static const int16_t kSincQ15[256 * 32] = {\n" + "\n".join(rows) + "\n};\n")
    path.parent.mkdir(parents=True, exist_ok=True)
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
