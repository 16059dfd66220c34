"""ORACLE (test infrastructure): the reference's CoreFFT known-answer vectors, restated.

``mpfs/host/corefft_vectors/`` holds 8 stimuli (N=8192, 16-bit data, 18-bit twiddles) produced by
``mpfs/host/fft_golden.py:103-126`` (stimuli) and :129-160 (codes) with the model
``src/fixedpoint.py:49-75`` (``fft1d_bfp``: radix-2 DIT on bit-reversed input, twiddles floored to
18 bits, whole-line block-floating-point requantise after every stage).  This module restates the
stimuli, the code conversion and that FFT so ``tests/test_oracle_pins.py`` can check them against the
CRC digests in ``tests/golden/fft_kat.json`` without the reference checkout.  It pins the building
blocks the emulator's per-row FFT shares with it (bit reversal, floored twiddles, butterfly).
"""
from __future__ import annotations

import math

import numpy as np

from .fixed_emulator import bitrev_perm


def stimuli(n: int = 8192) -> dict:
    """The eight named stimuli of fft_golden._cases (fft_golden.py:103-126)."""
    k = np.arange(n)
    rng = np.random.default_rng(1234)
    a = 2000.0
    k_imp = 37 % n
    return {
        "impulse": np.where(k == 0, a, 0).astype(np.complex128),
        "dc": np.full(n, a, dtype=np.complex128),
        "tone": a * np.exp(2j * np.pi * (n // 8) * k / n),
        "twotone": a * (np.exp(2j * np.pi * 5 * k / n) + 0.5 * np.exp(2j * np.pi * (n // 3) * k / n)),
        "random": (a * (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)).astype(np.complex128),
        "impulse_k": np.where(k == k_imp, a, 0).astype(np.complex128),
        "twotone_hidr": a * (np.exp(2j * np.pi * 11 * k / n) + 1e-3 * np.exp(2j * np.pi * (n // 3) * k / n)),
        "dc_smalltone": (a * np.ones(n) + 1e-3 * a * np.exp(2j * np.pi * (n // 5) * k / n)).astype(np.complex128),
    }


def block_exp(x, nbits):
    """fixedpoint.fit_scale (fixedpoint.py:19-26): (lsb, exp) so |x| fits signed nbits."""
    big = max(float(np.abs(x.real).max()), float(np.abs(x.imag).max()))
    if big == 0.0:
        return 1.0, 0
    e = math.ceil(math.log2(big / (2 ** (nbits - 1) - 1)))
    return 2.0 ** e, e


def requant(x, lsb, nbits):
    """fixedpoint.quant(mode='trunc') (fixedpoint.py:29-41): floor to the lsb grid, saturate."""
    top = 2 ** (nbits - 1) - 1
    return (np.clip(np.floor(x.real / lsb), -top - 1, top) + 1j * np.clip(np.floor(x.imag / lsb), -top - 1, top)) * lsb


def fft_bfp_line(x, nbits=16, nbits_tw=18):
    """fixedpoint.fft1d_bfp on one line; returns (values, per-stage exponents)."""
    n = x.size
    x = x[bitrev_perm(n)]
    lsb, e = block_exp(x, nbits)
    x = requant(x, lsb, nbits)
    exps = [e]
    lsb_tw = 2.0 ** -(nbits_tw - 1)
    for s in range(1, n.bit_length()):
        blk = 1 << s
        half = blk >> 1
        w = requant(np.exp(-2j * np.pi * np.arange(half) / blk), lsb_tw, nbits_tw)
        v = x.reshape(n // blk, blk)
        a, b = v[:, :half], v[:, half:]
        t = w * b
        x = np.concatenate([a + t, a - t], axis=1).reshape(n)
        lsb, e = block_exp(x, nbits)
        x = requant(x, lsb, nbits)
        exps.append(e)
    return x, exps


def codes(x, lsb, exact=False):
    """Integer codes of fft_golden._to_codes (floor, sat16) / _round_codes (exact multiples)."""
    if exact:
        return np.rint(x.real / lsb).astype(np.int64), np.rint(x.imag / lsb).astype(np.int64)
    top = 2 ** 15 - 1
    return (np.clip(np.floor(x.real / lsb), -top - 1, top).astype(np.int64),
            np.clip(np.floor(x.imag / lsb), -top - 1, top).astype(np.int64))
