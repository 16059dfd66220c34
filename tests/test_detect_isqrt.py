"""CPU: the integer square root of the fixed-point detect (k_fx_detect, detect_one).

The reference detects with floor(sqrt(re^2 + im^2)) in float64 (mpfs/host/silicon_emulator.py:208-213),
the integer square root of p = re^2 + im^2 <= 2^31.  The kernel takes an estimate from the hardware
square-root approximation of float(p) and applies one exact integer correction each way.  This checks the
argument it relies on: for any estimate within a relative error of 2^-21 (the hardware's is far smaller)
of sqrt(float(p)), truncation plus the two corrections give the exact integer square root, around every
perfect square of the range and at random points.
"""
import math

import numpy as np
import pytest


def _corrected(est, p):
    q = est.astype(np.int64)                      # truncation of the float estimate
    q = q - ((q * q) > p)
    q = q + (((q + 1) * (q + 1)) <= p)
    return q


@pytest.mark.parametrize("rel", [-2.0 ** -21, 0.0, 2.0 ** -21])
def test_one_step_corrections_give_the_integer_square_root(rel):
    k = np.arange(0, 46342, dtype=np.int64)
    p = np.concatenate([k * k + d for d in (-2, -1, 0, 1, 2)])
    p = np.concatenate([p[(p >= 0) & (p <= 2 ** 31)],
                        np.random.default_rng(7).integers(0, 2 ** 31 + 1, 500_000)])
    est = (np.sqrt(p.astype(np.float32).astype(np.float64)) * (1.0 + rel)).astype(np.float32)
    ref = np.fromiter((math.isqrt(int(x)) for x in p), dtype=np.int64, count=len(p))
    assert np.array_equal(_corrected(est, p), ref)
    # the reference's float64 floor(sqrt(.)) is the same integer on this range
    assert np.array_equal(np.floor(np.sqrt(p.astype(np.float64))).astype(np.int64), ref)
