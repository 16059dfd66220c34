"""CPU: pin the oracle against the reference's golden vectors and against the reference itself.

* FFT building blocks vs the reference's CoreFFT known-answer vectors (digests in golden/fft_kat.json).
* Whole fixed-point frames vs the reference emulator's CRC (golden/fixed_frames.json, produced by
  golden/make_golden.py running ``silicon_emulator.form_image`` unmodified).
* Float frames vs the reference ``pfa()`` digests (golden/float_frames.json).
* Where the reference checkout is present: stage-by-stage equality with the reference functions.
"""
import json
import zlib

import numpy as np
import pytest

from oracle import fft_kat, fixed_emulator as fe, float_pfa as fp
from pfa_b200 import synth, geometry


def _crc(a):
    return zlib.crc32(np.ascontiguousarray(a).tobytes()) & 0xFFFFFFFF


def test_fft_kat_vectors(golden_dir):
    g = json.loads((golden_dir / "fft_kat.json").read_text())
    for name, x in fft_kat.stimuli(g["n"]).items():
        c = g["cases"][name]
        lsb, e_in = fft_kat.block_exp(x, g["nbits"])
        ir, ii = fft_kat.codes(x, lsb)
        assert _crc(np.stack([ir, ii], 1).astype("<i2")) == c["in_crc"], name
        y, ex = fft_kat.fft_bfp_line(x, g["nbits"], g["nbits_tw"])
        orr, oi = fft_kat.codes(y, 2.0 ** ex[-1], exact=True)
        assert _crc(np.stack([orr, oi], 1).astype("<i2")) == c["out_crc"], name
        assert ex == c["stage_exps"], name


FIXED = json.loads((__import__("pathlib").Path(__file__).parent / "golden" / "fixed_frames.json").read_text())["cases"]


@pytest.mark.parametrize("name", sorted(FIXED))
def test_fixed_oracle_matches_reference_crc(name):
    c = FIXED[name]
    sc = synth.make_scene(**c["scene"])
    if _crc(sc.signal) != c["input_crc"]:
        pytest.skip("synthetic input not bit-identical on this host")
    tb = geometry.prepare_tables_from_scene(sc)
    img, _ = fe.form_image(sc.signal, tb, c["grid"], c["range_sinc"], c["az_sinc"])
    assert fe.frame_crc(img) == c["image_crc"]


FLOAT = json.loads((__import__("pathlib").Path(__file__).parent / "golden" / "float_frames.json").read_text())["cases"]


@pytest.mark.parametrize("name", sorted(FLOAT))
def test_float_oracle_matches_reference(name):
    c = FLOAT[name]
    sc = synth.make_scene(**c["scene"])
    if _crc(sc.signal) != c["input_crc"]:
        pytest.skip("synthetic input not bit-identical on this host")
    tb = geometry.prepare_tables_from_scene(sc)
    det = fp.detect(fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"]))
    assert _crc(det) == c["detect_crc"]


def test_sinc_table_matches_reference(ref_modules):
    ref = np.asarray(ref_modules.grv.sinc_table_q15(256, 32), np.int64)
    assert np.array_equal(fe.sinc_table_q15(), ref)


def test_stages_match_reference(ref_modules):
    """Each restated stage equals the reference function on the same operands."""
    emu, ser, fx = ref_modules.emu, ref_modules.ser, ref_modules.fx
    rng = np.random.default_rng(5)
    # bracket + Q15 weight, ascending and descending source axes, out-of-span queries included
    for asc in (True, False):
        xp = np.sort(rng.uniform(-3, 3, 300))
        xp = xp if asc else xp[::-1]
        q = rng.uniform(-3.5, 3.5, 700)
        i0, w0 = ser.interp_coeffs(q, xp)
        i1, w1 = fe.bracket_q15(q, xp)
        assert np.array_equal(i0, i1) and np.array_equal(w0, w1)
    # sinc / lerp gathers on adversarial int16 extremes
    sn = 96
    src = rng.choice([-32768, 32767, -1, 0, 1, 12345, -23456], size=sn) + 1j * rng.choice(
        [-32768, 32767, -1, 0, 1, 777, -999], size=sn)
    idx = rng.integers(-1, sn - 1, 500).astype(np.int32)
    wq = rng.integers(0, 32768, 500).astype(np.int16)
    wq[idx < 0] = 0
    r0 = emu.apply_sinc(src, idx, wq, sn)
    rr, ri = fe.gather_sinc(src.real.astype(np.int64), src.imag.astype(np.int64), idx.astype(np.int64),
                            wq.astype(np.int64), sn)
    assert np.array_equal(r0.real, rr) and np.array_equal(r0.imag, ri)
    r0 = emu.apply_fixed(src.astype(np.complex64), idx, wq)
    rr, ri = fe.gather_lerp(src.real.astype(np.int64), src.imag.astype(np.int64), idx.astype(np.int64),
                            wq.astype(np.int64), f32_product=True)
    assert np.array_equal(r0.real, rr) and np.array_equal(r0.imag, ri)
    # window with odd lengths (the 32768 centre tap wraps to -32768)
    g = rng.integers(-32768, 32768, (64, 64)) + 1j * rng.integers(-32768, 32768, (64, 64))
    w0 = emu.window_fixed(g, 63, 61)
    wr, wi = fe.window_q15(g.real.astype(np.int64), g.imag.astype(np.int64), 63, 61)
    assert np.array_equal(w0.real, wr) and np.array_equal(w0.imag, wi)
    # BFP FFT pass
    x = rng.integers(-32768, 32768, (16, 256)) + 1j * rng.integers(-32768, 32768, (16, 256))
    y0, e0 = emu.fft_pass_bfp(x.astype(np.complex128))
    yr, yi, e1 = fe.fft_pass(x.real.astype(np.int64), x.imag.astype(np.int64))
    assert np.array_equal(y0.real, yr) and np.array_equal(y0.imag, yi) and np.array_equal(e0, e1)
    # detect
    z = x[:, :64]
    assert np.array_equal(emu.detect_fixed(z), fe.detect_q(z.real.astype(np.int64), z.imag.astype(np.int64)))


def test_prepare_tables_matches_reference(ref_modules):
    sc = synth.make_scene(300, 280, n_targets=4, seed=3, jitter=0.4)
    from oracle import refshim
    t0 = refshim.reference_tables(sc)
    t1 = geometry.prepare_tables_from_scene(sc)
    for k in ("ax", "ay", "freq", "KR", "KC", "tan_phi", "window"):
        assert np.array_equal(np.asarray(t0[k]), np.asarray(t1[k])), k
    assert t0["sgn"] == t1["sgn"] and tuple(t0["dims"]) == tuple(t1["dims"])


# ----------------------------------------------------------------------------- silicon A/B variants
def _variant_inputs():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    import make_golden
    return make_golden.variant_inputs()


def test_cubic_taps_and_gather_match_reference_vectors(golden_dir):
    g = json.loads((golden_dir / "variants.json").read_text())
    taps = fe.lagrange_taps_q15(np.arange(32768))
    assert _crc(taps.astype("<i4")) == g["lagrange_taps_crc"]
    assert list(taps[16384]) == g["lagrange_taps_w16384"]
    v = _variant_inputs()
    rr, ri = fe.gather_cubic(v["src_re"], v["src_im"], v["idx"], v["wq"], v["sn"])
    words = ((ri.astype(np.int64) & 0xFFFF) << 16) | (rr.astype(np.int64) & 0xFFFF)
    assert _crc(words.astype("<u4")) == g["gather_cubic_crc"]


def test_fused_detect_matches_reference_vectors(golden_dir):
    g = json.loads((golden_dir / "variants.json").read_text())
    v = _variant_inputs()
    img = fe.detect_fused(v["y_re"], v["y_im"], v["e"])
    assert _crc(img.astype("<u2")) == g["detect_fused_crc"]


def test_variant_frames_are_consistent():
    """Frame level: the cubic variant differs from lerp only inside the cubic's interior, and the fused
    detect stays within a few counts of the emulator order."""
    sc = synth.make_scene(96, 80, n_targets=6, snr_db=20.0, seed=31)
    tb = geometry.prepare_tables_from_scene(sc)
    lerp, _ = fe.form_image(sc.signal, tb, 128, range_mode="lerp", az_mode="lerp")
    cub, _ = fe.form_image(sc.signal, tb, 128, range_mode="cubic", az_mode="cubic")
    assert (lerp > 0).sum() > 0 and not np.array_equal(lerp, cub)
    emu, _ = fe.form_image(sc.signal, tb, 128, True, True)
    fused, _ = fe.form_image(sc.signal, tb, 128, True, True, detect_order="fused")
    d = np.abs(emu.astype(np.int64) - fused.astype(np.int64))
    assert d.max() <= 2 and (d > 0).any()


def test_synth_phase_error_matches_autofocus_oracle():
    """The bench's injected autofocus phase error (pfa_b200.synth) is the oracle's (autofocus_ref)."""
    from oracle import autofocus_ref
    for m, seed in ((4096, 4), (256, 7)):
        assert np.array_equal(synth.phase_error(m, seed=seed), autofocus_ref.phase_error(m, seed=seed))


def test_c_restatement_matches_numpy_oracle():
    """The C restatement of the fixed datapath (oracle/fixed_frame.c, timed by bench.py's reference arm)
    gives the NumPy oracle's image and exponents on every interpolator pair and a descending axis."""
    from oracle import cpu_sample
    from pfa_b200 import geometry, synth
    for m, n, grid, rs, az, seed in [(300, 250, 512, False, True, 42), (240, 256, 256, True, False, 3),
                                     (120, 110, 128, True, True, 7), (200, 180, 256, False, False, 11)]:
        sc = synth.make_scene(m, n, n_targets=12, clutter_db=-10.0, seed=seed, jitter=0.3)
        tb = geometry.prepare_tables_from_scene(sc)
        ref, d = fe.form_image(sc.signal, tb, grid, rs, az)
        img, dc = cpu_sample.c_fixed_frame(sc.signal, tb, grid, rs, az, threads=2)
        assert np.array_equal(img, ref), (m, n, grid, rs, az)
        assert dc["q0_exp"] == d["q0_exp"]
        assert np.array_equal(dc["e_range"], d["e_range"]) and np.array_equal(dc["e_az"], d["e_az"])


def test_c_restatement_reproduces_reference_crc_of_full_frame():
    r"""The whole Centerfield-shaped 5634x4319 -> 8192^2 sinc/sinc frame: the C restatement's image has the
    CRC the unmodified reference emulator produced (tests/golden/big_frames.json)."""
    import json
    from oracle import cpu_sample
    from pfa_b200 import geometry, synth
    from pathlib import Path
    case = json.loads((Path(__file__).parent / "golden" / "big_frames.json").read_text())["cases"]["centerfield_5634x4319_sinc"]
    sc = synth.workload_scene("centerfield_5634x4319")
    assert _crc(sc.signal) == case["input_crc"]
    tb = geometry.prepare_tables_from_scene(sc)
    img, _ = cpu_sample.c_fixed_frame(sc.signal, tb, 8192, True, True)
    assert fe.frame_crc(img) == case["image_crc"]
