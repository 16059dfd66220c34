"""GPU parity of the float path (FP32) against the oracle: the reference-precision restatement of
form_image_pfa.pfa (bit-identical to the reference, tests/test_oracle_pins.py) and the FP64 version.

Tolerances (FP32 arithmetic throughout, FP64 coordinates):
  * relative L2 of the detected image and of the complex image vs FP64:          <= 1e-6
  * relative L2 vs the reference-precision oracle (complex64 intermediates):     <= 1e-6
  * point-target peak location identical, ISLR within 0.01 dB of FP64
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import float_pfa as fp
from pfa_b200 import _lib, engine, geometry, synth

pytestmark = pytest.mark.gpu
TOL = 1e-6
FLOAT = json.loads((Path(__file__).resolve().parent / "golden" / "float_frames.json").read_text())["cases"]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(sig, tables, detect="mag", rs=False, az=False, centred=True, window=True):
    m, n = sig.shape
    with engine.FloatPlan(m, n, rs, az) as plan:
        plan.set_tables(tables, window=window, centred=centred)
        return plan.form(sig, detect=detect)


@pytest.mark.parametrize("m,n,jit", [(256, 240, 0.3), (1024, 1024, 0.0), (600, 900, 0.3), (512, 700, 0.5), (130, 70, 0.0)])
def test_lerp_frames(torch_cuda, m, n, jit):
    sc = synth.make_scene(m, n, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=m + n, jitter=jit)
    tb = geometry.prepare_tables_from_scene(sc)
    det = _run(sc.signal, tb)
    cz = _run(sc.signal, tb, detect="complex")
    ref = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="ref")
    r64 = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64")
    assert det.shape == ref.shape == (geometry.pow2(m), geometry.pow2(n))
    assert fp.rel_l2(det, fp.detect(ref)) <= TOL
    assert fp.rel_l2(det, np.abs(r64)) <= TOL
    assert fp.rel_l2(cz, r64) <= TOL


@pytest.mark.parametrize("rs,az", [(True, True), (True, False), (False, True)])
def test_sinc_frames_vs_fp64(torch_cuda, rs, az):
    sc = synth.make_scene(512, 512, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=1024)
    tb = geometry.prepare_tables_from_scene(sc)
    cz = _run(sc.signal, tb, detect="complex", rs=rs, az=az)
    g2 = _f64_mixed(sc.signal, tb, rs, az)
    assert fp.rel_l2(cz, g2) <= TOL


def _f64_mixed(sig, tb, rs, az):
    """FP64 oracle with a per-pass interpolator choice."""
    g = fp.geometry(tb["freq"], tb["ax"], tb["ay"])
    m, n = sig.shape
    g1 = np.empty((m, n), np.complex128)
    for i in range(m):
        xp, row = g["kr"][i], sig[i].astype(np.complex128)
        if xp[0] > xp[-1]:
            xp, row = xp[::-1], row[::-1]
        g1[i] = fp._interp(g["KR"], xp, row, "sinc" if rs else "lerp")
    g1s = g1[g["order"]]
    tan_s = g["tan_phi"][g["order"]]
    g2 = np.empty((m, n), np.complex128)
    for j in range(n):
        g2[:, j] = fp._interp(g["KC"], g["KR"][j] * tan_s, g1s[:, j], "sinc" if az else "lerp")
    g2 = g2 * np.outer(np.hamming(m), np.hamming(n))
    return fp.focus(g2, tb["sgn"], precision="f64")


def test_descending_axes_sinc(torch_cuda):
    sc = synth.make_scene(300, 280, n_targets=8, snr_db=20.0, seed=51, jitter=0.4)
    tb = dict(geometry.prepare_tables_from_scene(sc))
    tb["freq"] = tb["freq"][:, ::-1].copy()     # descending frequency axis: pass-1 source reversed
    tb.pop("KR"), tb.pop("KC")
    cz = _run(sc.signal, tb, detect="complex", rs=True, az=True)
    assert fp.rel_l2(cz, _f64_mixed(sc.signal, tb, True, True)) <= TOL


def test_layouts_signs_and_power(torch_cuda):
    sc = synth.make_scene(256, 256, n_targets=8, snr_db=20.0, seed=52)
    tb = dict(geometry.prepare_tables_from_scene(sc))
    g2, _ = fp.resample_kspace(sc.signal, tb["freq"], tb["ax"], tb["ay"], precision="f64")
    nat = _run(sc.signal, tb, detect="complex", centred=False)
    assert fp.rel_l2(nat, np.fft.fft2(g2)) <= TOL
    tb["sgn"] = 1
    inv = _run(sc.signal, tb, detect="complex")
    assert fp.rel_l2(inv, np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(g2)))) <= TOL
    tb["sgn"] = -1
    mag = _run(sc.signal, tb)
    pw = _run(sc.signal, tb, detect="power")
    assert np.allclose(pw, mag.astype(np.float64) ** 2, rtol=1e-5, atol=0)
    raw = _run(sc.signal, tb, detect="complex", window=False)
    g2w, _ = fp.resample_kspace(sc.signal, tb["freq"], tb["ax"], tb["ay"], precision="f64", window=False)
    assert fp.rel_l2(raw, fp.focus(g2w, -1, precision="f64")) <= TOL


def test_point_target_quality(torch_cuda):
    sc = synth.make_scene(1024, 1024, n_targets=1, scene_half=60.0, snr_db=None, seed=53)
    tb = geometry.prepare_tables_from_scene(sc)
    det = _run(sc.signal, tb)
    r64 = np.abs(fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64"))
    pk = np.unravel_index(np.argmax(r64), r64.shape)
    assert np.unravel_index(np.argmax(det), det.shape) == pk
    p0, i0 = fp.peak_islr(r64, pk)
    p1, i1 = fp.peak_islr(det, pk)
    assert abs(i1 - i0) < 0.01 and abs(p1 / p0 - 1) < 1e-5


@pytest.mark.parametrize("name", sorted(FLOAT))
def test_golden_float_frames(torch_cuda, name):
    c = FLOAT[name]
    sc = synth.make_scene(**c["scene"])
    tb = geometry.prepare_tables_from_scene(sc)
    det = _run(sc.signal, tb).ravel()
    assert list(det.shape) == [int(np.prod(c["shape"]))]
    got_top = np.argsort(det)[::-1][:8]
    assert set(got_top[:4]) == set(c["top_index"][:4])
    np.testing.assert_allclose(det[c["top_index"]], c["top_value"], rtol=1e-5)
    assert abs((det.astype(np.float64) ** 2).sum() / c["energy"] - 1) < 1e-6


def test_host_entry_point_and_errors(torch_cuda):
    sc = synth.make_scene(200, 190, n_targets=4, seed=54)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(200, 190) as plan:
        with pytest.raises(_lib.PfaError) as ei:
            plan.form(sc.signal)
        assert ei.value.status == _lib.NOT_READY
        plan.set_tables(tb)
        a = plan.form_host(sc.signal)
        b = plan.form(sc.signal)
        assert np.array_equal(a, b)
        st = plan._lib.pfa_form_float(plan.handle, None, None, 0, None)
        assert st == _lib.BAD_ARG


@pytest.mark.parametrize("m,n,rs", [(9000, 300, False), (300, 9000, True)])
def test_16384_point_lines(torch_cuda, m, n, rs):
    """Lines of 16384 points on either axis (the reference's NDSU scene, 8167 x 8999, pads its range
    axis to 16384): FP32 against FP64."""
    sc = synth.make_scene(m, n, n_targets=8, clutter_db=-10.0, snr_db=20.0, seed=m + n, jitter=0.2)
    tb = geometry.prepare_tables_from_scene(sc)
    cz = _run(sc.signal, tb, detect="complex", rs=rs, az=rs)
    assert cz.shape == (geometry.pow2(m), geometry.pow2(n))
    assert fp.rel_l2(cz, _f64_mixed(sc.signal, tb, rs, rs)) <= TOL


@pytest.mark.parametrize("rs,az", [(False, False), (False, True)])
@pytest.mark.parametrize("m", [255, 256, 257, 4099])
def test_tma_row_boxes_cover_every_row_length(torch_cuda, m, rs, az):
    """Pass 2 reads each range-bin row as 256-sample TMA boxes (the last one partly past the row, zero
    filled): row lengths just below, at and above a box boundary and a long odd one match FP64."""
    sc = synth.make_scene(m, 300, n_targets=12, clutter_db=-10.0, snr_db=20.0, seed=m, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    cz = _run(sc.signal, tb, detect="complex", rs=rs, az=az)
    assert fp.rel_l2(cz, _f64_mixed(sc.signal, tb, rs, az)) <= TOL


@pytest.mark.parametrize("az", [False, True])
def test_row_load_bounded_wait_runs_out_and_the_context_recovers(torch_cuda, az):
    """The TMA row load of pass 2 waits on an mbarrier with a poll limit.  A plan whose pass 2 first waits
    on a barrier nothing arrives on (the test hook pfa_config.test_wait_polls) gives up, uses no row, waits
    for its copies before it exits, and the synchronous entry point returns PFA_ERR_TIMEOUT; the context
    stays usable and a normal plan right after forms the correct frame."""
    sc = synth.make_scene(300, 260, n_targets=8, clutter_db=-10.0, snr_db=20.0, seed=67)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(300, 260, False, az, test_wait_polls=500) as p:
        p.set_tables(tb)
        with pytest.raises(_lib.PfaError) as ei:
            p.form_host(sc.signal)
        assert ei.value.status == _lib.TIMEOUT
        assert "timed out" in str(ei.value)
        # the flag is cleared once reported: the next frame times out again rather than inheriting it
        with pytest.raises(_lib.PfaError):
            p.form_host(sc.signal)
    cz = _run(sc.signal, tb, detect="complex", az=az)
    assert fp.rel_l2(cz, _f64_mixed(sc.signal, tb, False, az)) <= TOL
