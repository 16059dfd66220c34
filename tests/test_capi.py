"""CPU: the C-ABI library loads, exports every function include/pfa_b200.h declares, and the host-side
tables the product builds equal the oracle's."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from pfa_b200 import _lib, geometry, tables
from oracle import fixed_emulator as fe

HEADER = Path(__file__).resolve().parents[1] / "include" / "pfa_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pfa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert set(names) <= set(_lib.SIGNATURES), sorted(set(names) - set(_lib.SIGNATURES))


def test_status_strings_and_version():
    lib = _lib.load()
    assert lib.pfa_version().startswith(b"pfa_b200")
    strings = [lib.pfa_status_string(st) for st in range(10)]
    assert all(strings) and len(set(strings)) == 10
    assert b"1024" in strings[_lib.TOO_LARGE]
    assert lib.pfa_status_string(99) == b"unknown status"


def test_plan_create_rejects_bad_args_without_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.pfa_plan_create(None, ctypes.byref(h)) == _lib.BAD_ARG
    cfg = _lib.Config(mode=_lib.MODE_FIXED, m=1, n=100, grid=256)
    assert lib.pfa_plan_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.BAD_DIMS
    cfg = _lib.Config(mode=_lib.MODE_FIXED, m=100, n=100, grid=256, range_interp=7)
    assert lib.pfa_plan_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.BAD_CONFIG
    assert lib.pfa_plan_destroy(None) == _lib.BAD_ARG
    assert lib.pfa_set_fixed_job(None, None) == _lib.BAD_ARG
    assert lib.pfa_form_fixed(None, None, None, None) == _lib.BAD_ARG


def test_variant_configs_validated_without_gpu():
    """The cubic resampler and the fused detect order are fixed-mode variants: float plans asking for
    them, and unknown values, are refused before any device is touched."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    for kw in (dict(mode=_lib.MODE_FLOAT32, range_interp=_lib.CUBIC), dict(mode=_lib.MODE_MIXED, az_interp=_lib.CUBIC),
               dict(mode=_lib.MODE_FLOAT32, detect_order=_lib.DETECT_ORDER_FUSED),
               dict(mode=_lib.MODE_FIXED, grid=256, range_interp=3), dict(mode=_lib.MODE_FIXED, grid=256, detect_order=2)):
        cfg = _lib.Config(m=200, n=200, **kw)
        assert lib.pfa_plan_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.BAD_CONFIG, kw


def test_product_sinc_table_equals_oracle():
    assert np.array_equal(tables.sinc_table_q15().astype(np.int64), fe.sinc_table_q15())


@pytest.mark.parametrize("G", [64, 256, 1024, 8192, 16384])
def test_product_twiddles_and_tapers_equal_oracle(G):
    wr, wi = fe.twiddles_q15(G)
    tw = geometry.twiddles_q15(G)
    assert np.array_equal(tw[:, 0], wr) and np.array_equal(tw[:, 1], wi)
    for length in (G // 2 + 1, G - 3, G):
        assert np.array_equal(geometry.hamming_q15_floor(length, G), fe.hamming_q15(length, G))


def test_fixed_job_matches_oracle_geometry():
    from pfa_b200 import synth
    sc = synth.make_scene(300, 280, n_targets=4, seed=3, jitter=0.4)
    tb = geometry.prepare_tables_from_scene(sc)
    job = geometry.fixed_job(tb, 512)
    geo = fe.fixed_geometry(tb, 512)
    for a, b in [("f0", "f0"), ("df", "df"), ("pr", "pr"), ("tan_s", "tan_s"), ("krp", "KRp"), ("kcp", "KCp")]:
        assert np.array_equal(job[a], geo[b]), a
    assert np.array_equal(job["order"], geo["order"])
    with pytest.raises(ValueError):
        geometry.fixed_job(tb, 256)


def test_noalloc_validates_before_touching_a_device():
    """The allocation-free entry point refuses a non-permutation inv_order (PFA_ERR_BAD_ARG), a grid above
    its static scratch (PFA_ERR_TOO_LARGE) and dims above the grid (PFA_ERR_BAD_DIMS) on the host, before
    any device call; the signal and image pointers are never dereferenced on these paths."""
    from pfa_b200 import synth
    lib = _lib.load()
    sc = synth.make_scene(120, 100, n_targets=2, seed=5, with_signal=False)
    tb = geometry.prepare_tables_from_scene(sc)
    j = geometry.fixed_job(tb, 256)
    inv = np.empty(j["m"], np.int32)
    inv[j["order"]] = np.arange(j["m"], dtype=np.int32)
    inv[1] = inv[0]                               # duplicate slot: not a permutation
    keep = [j["f0"], j["df"], j["pr"], j["tan_s"], inv, j["krp"], j["kcp"],
            np.ascontiguousarray(j["hamr"], np.int32), np.ascontiguousarray(j["hamc"], np.int32),
            np.ascontiguousarray(j["twiddle"], np.int16)]
    job = _lib.FixedJob(*[ctypes.c_void_p(a.ctypes.data) for a in keep], None)
    fake_sig, fake_img = ctypes.c_void_p(1 << 20), ctypes.c_void_p(2 << 20)    # aligned, never read
    cfg = _lib.Config(mode=_lib.MODE_FIXED, m=120, n=100, grid=256, range_interp=_lib.SINC, az_interp=_lib.SINC)
    assert lib.pfa_form_fixed_noalloc(ctypes.byref(cfg), ctypes.byref(job), fake_sig, fake_img, None) == _lib.BAD_ARG
    cfg.grid = 2048
    assert lib.pfa_form_fixed_noalloc(ctypes.byref(cfg), ctypes.byref(job), fake_sig, fake_img, None) == _lib.TOO_LARGE
    cfg.grid, cfg.m = 64, 120
    assert lib.pfa_form_fixed_noalloc(ctypes.byref(cfg), ctypes.byref(job), fake_sig, fake_img, None) == _lib.BAD_DIMS
    assert lib.pfa_form_fixed_noalloc(ctypes.byref(cfg), ctypes.byref(job), None, fake_img, None) == _lib.BAD_ARG
