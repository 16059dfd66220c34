"""The O(m + n) table preparation (geometry.prepare_tables_fast) gives bit-identical tables and job
vectors to the literal restatement of sar_pipeline.prepare_tables (itself pinned to the reference in
test_oracle_pins.py), including decimation, cropping and a descending frequency axis."""
import dataclasses

import numpy as np
import pytest

from pfa_b200 import geometry, synth
from pfa_b200.synth import FakeReader


def _both(sc, deci=1, crop=0):
    rd = FakeReader(sc)
    a = geometry.prepare_tables(rd, rd.cphd_meta, deci, deci, crop)
    b = geometry.prepare_tables_fast(rd, rd.cphd_meta, deci, deci, crop)
    return a, b


def _assert_identical(a, b):
    for k in ("ax", "ay", "KR", "KC", "tan_phi", "sgn", "dims", "samp0"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    assert np.array_equal(a["freq"], np.asarray(b["freq"]))
    assert b["freq"].shape == a["freq"].shape
    for c in (0, 1, -1):
        assert np.array_equal(a["freq"][:, c], b["freq"][:, c])
    fa, fb = geometry.float_job(a), geometry.float_job(b)
    for k, v in fa.items():
        assert np.array_equal(np.asarray(v), np.asarray(fb[k])), k
    g = geometry.pow2(max(a["freq"].shape))
    xa, xb = geometry.fixed_job(a, g), geometry.fixed_job(b, g)
    for k, v in xa.items():
        assert np.array_equal(np.asarray(v), np.asarray(xb[k])), k


@pytest.mark.parametrize("m,n,jit,seed", [(300, 257, 0.4, 5), (1024, 1000, 0.0, 6), (777, 1531, 0.3, 7)])
def test_fast_tables_identical(m, n, jit, seed):
    sc = synth.make_scene(m, n, with_signal=False, n_targets=4, seed=seed, jitter=jit)
    _assert_identical(*_both(sc))


def test_fast_tables_decimated_and_cropped():
    sc = synth.make_scene(640, 700, with_signal=False, n_targets=4, seed=8, jitter=0.2)
    _assert_identical(*_both(sc, deci=2))
    _assert_identical(*_both(sc, deci=1, crop=512))
    _assert_identical(*_both(sc, deci=3, crop=200))


def test_fast_tables_descending_frequency():
    sc = synth.make_scene(400, 333, with_signal=False, n_targets=4, seed=9, jitter=0.3)
    n = 333
    sc = dataclasses.replace(sc, sc0=sc.sc0 + (n - 1) * sc.scss, scss=-sc.scss)
    _assert_identical(*_both(sc))
