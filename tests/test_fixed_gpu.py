"""GPU parity of the fixed-point path (bit-exact): the CUDA library vs the oracle and vs the reference's
golden CRCs, through the C ABI."""
import json
import zlib
from pathlib import Path

import numpy as np
import pytest

from oracle import fixed_emulator as fe
from pfa_b200 import _lib, engine, geometry, synth

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
FIXED = json.loads((GOLD / "fixed_frames.json").read_text())["cases"]
BIG = json.loads((GOLD / "big_frames.json").read_text())["cases"]


def _crc(a):
    return zlib.crc32(np.ascontiguousarray(a).tobytes()) & 0xFFFFFFFF


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _form(torch, sig, tables, grid, rs, az):
    m, n = sig.shape
    with engine.FixedPlan(m, n, grid, rs, az) as plan:
        plan.set_tables(tables)
        img = plan.form(torch.from_numpy(np.ascontiguousarray(sig)).cuda()).cpu().numpy()
        er, ea, q0 = plan.exponents()
    return img, er, ea, q0


@pytest.mark.parametrize("name", sorted(k for k, v in FIXED.items() if v["grid"] >= 64))
def test_golden_frames(torch_cuda, name):
    c = FIXED[name]
    sc = synth.make_scene(**c["scene"])
    tb = geometry.prepare_tables_from_scene(sc)
    img, er, ea, q0 = _form(torch_cuda, sc.signal, tb, c["grid"], c["range_sinc"], c["az_sinc"])
    ref, d = fe.form_image(sc.signal, tb, c["grid"], c["range_sinc"], c["az_sinc"])
    assert np.array_equal(img, ref), f"{(img != ref).sum()} pixels differ from the oracle"
    assert np.array_equal(er, d["e_range"][: sc.signal.shape[1]])
    assert np.array_equal(ea, d["e_az"])
    assert q0 == d["q0_exp"]
    if _crc(sc.signal) == c["input_crc"]:
        assert fe.frame_crc(img) == c["image_crc"]


def test_full_centerfield_frame_matches_reference_crc(torch_cuda):
    c = BIG["centerfield_5634x4319_sinc"]
    sc = synth.workload_scene(c["workload"])
    if _crc(sc.signal) != c["input_crc"]:
        pytest.skip("synthetic input not bit-identical on this host")
    tb = geometry.prepare_tables_from_scene(sc)
    img, *_ = _form(torch_cuda, sc.signal, tb, c["grid"], c["range_sinc"], c["az_sinc"])
    assert fe.frame_crc(img) == c["image_crc"]


@pytest.mark.parametrize("rs,az", [(True, True), (False, False), (True, False), (False, True)])
def test_uneven_dims_and_knobs(torch_cuda, rs, az):
    sc = synth.make_scene(300, 470, n_targets=12, clutter_db=-10.0, snr_db=20.0, seed=31, jitter=0.5)
    tb = geometry.prepare_tables_from_scene(sc)
    img, er, ea, _ = _form(torch_cuda, sc.signal, tb, 512, rs, az)
    ref, d = fe.form_image(sc.signal, tb, 512, rs, az)
    assert np.array_equal(img, ref)


def test_scene_filling_the_grid(torch_cuda):
    sc = synth.make_scene(256, 256, n_targets=6, snr_db=10.0, seed=32)
    tb = geometry.prepare_tables_from_scene(sc)
    img, *_ = _form(torch_cuda, sc.signal, tb, 256, True, True)
    ref, _ = fe.form_image(sc.signal, tb, 256, True, True)
    assert np.array_equal(img, ref)


def test_zero_signal(torch_cuda):
    sc = synth.make_scene(120, 100, n_targets=2, seed=33)
    tb = geometry.prepare_tables_from_scene(sc)
    z = np.zeros_like(sc.signal)
    img, er, ea, q0 = _form(torch_cuda, z, tb, 128, True, True)
    assert not img.any() and not er.any() and not ea.any() and q0 == 0


def test_saturating_nyquist_input(torch_cuda):
    """Alternating full-scale samples make the 32-tap sinc overshoot int16: exercises every saturation."""
    sc = synth.make_scene(160, 150, n_targets=2, seed=34)
    tb = geometry.prepare_tables_from_scene(sc)
    k = np.arange(150)
    i = np.arange(160)[:, None]
    s = (np.where((k + i) % 2 == 0, 3.0e4, -3.0e4) + 1j * np.where(k % 3 == 0, -3.0e4, 3.0e4)).astype(np.complex64)
    for rs, az in [(True, True), (False, False)]:
        img, *_ = _form(torch_cuda, s, tb, 256, rs, az)
        ref, _ = fe.form_image(s, tb, 256, rs, az)
        assert np.array_equal(img, ref)


def test_descending_axes(torch_cuda):
    """Negated frequency table and grids: both pass-1 and pass-2 brackets take the descending branch."""
    sc = synth.make_scene(140, 130, n_targets=5, snr_db=20.0, seed=35, jitter=0.4)
    tb = dict(geometry.prepare_tables_from_scene(sc))
    tb["freq"] = -tb["freq"]
    tb["KR"] = -tb["KR"][::-1]
    for rs, az in [(True, True), (False, False)]:
        img, *_ = _form(torch_cuda, sc.signal, tb, 256, rs, az)
        ref, _ = fe.form_image(sc.signal, tb, 256, rs, az)
        assert np.array_equal(img, ref)


def test_iq16_and_host_entry_points(torch_cuda):
    torch = torch_cuda
    sc = synth.make_scene(200, 190, n_targets=6, snr_db=20.0, seed=36)
    tb = geometry.prepare_tables_from_scene(sc)
    ref, _ = fe.form_image(sc.signal, tb, 256, True, True)
    with engine.FixedPlan(200, 190, 256, True, True) as plan:
        plan.set_tables(tb)
        a = plan.form_host(sc.signal)
        b = plan.form_host(sc.signal)          # plan reuse: identical second call
        qr, qi, _ = fe.quantize_q0(sc.signal)
        iq = torch.from_numpy(np.stack([qr, qi], -1).astype(np.int16)).cuda().contiguous()
        c = plan.form_iq16(iq).cpu().numpy()
    assert np.array_equal(a, ref) and np.array_equal(b, ref) and np.array_equal(c, ref)


def test_two_plans_on_two_streams(torch_cuda):
    torch = torch_cuda
    s1 = synth.make_scene(128, 120, n_targets=4, seed=37)
    s2 = synth.make_scene(100, 128, n_targets=4, seed=38, jitter=0.5)
    t1, t2 = geometry.prepare_tables_from_scene(s1), geometry.prepare_tables_from_scene(s2)
    st1, st2 = torch.cuda.Stream(), torch.cuda.Stream()
    with engine.FixedPlan(128, 120, 128, True, True) as p1, engine.FixedPlan(100, 128, 128, False, True) as p2:
        p1.set_tables(t1)
        p2.set_tables(t2)
        x1 = torch.from_numpy(s1.signal).cuda()
        x2 = torch.from_numpy(s2.signal).cuda()
        torch.cuda.synchronize()
        with torch.cuda.stream(st1):
            o1 = p1.form(x1, stream=st1)
        with torch.cuda.stream(st2):
            o2 = p2.form(x2, stream=st2)
        torch.cuda.synchronize()
    assert np.array_equal(o1.cpu().numpy(), fe.form_image(s1.signal, t1, 128, True, True)[0])
    assert np.array_equal(o2.cpu().numpy(), fe.form_image(s2.signal, t2, 128, False, True)[0])


def test_errors_are_status_codes(torch_cuda):
    torch = torch_cuda
    with pytest.raises(_lib.PfaError) as ei:
        engine.FixedPlan(300, 200, 256)
    assert ei.value.status == _lib.BAD_DIMS
    with pytest.raises(_lib.PfaError) as ei:
        engine.FixedPlan(100, 100, 100)
    assert ei.value.status == _lib.BAD_CONFIG
    with engine.FixedPlan(100, 100, 128) as plan:
        x = torch.zeros((100, 100), dtype=torch.complex64, device="cuda")
        with pytest.raises(_lib.PfaError) as ei:
            plan.form(x)
        assert ei.value.status == _lib.NOT_READY
        sc = synth.make_scene(100, 100, n_targets=2, seed=39)
        plan.set_tables(geometry.prepare_tables_from_scene(sc))
        flat = torch.zeros(100 * 100 * 2 + 1, dtype=torch.float32, device="cuda")
        img = torch.empty((128, 128), dtype=torch.uint16, device="cuda")
        st = plan._lib.pfa_form_fixed(plan.handle, flat.data_ptr() + 4, img.data_ptr(), None)
        assert st == _lib.BAD_ARG


def test_caller_sinc_table(torch_cuda):
    """A caller-supplied Q15 table: the reference's own table gives the same image; a table whose taps
    could overflow the int32 half sums (sum |tap| > 65535 over 16 taps) is refused."""
    from pfa_b200 import tables
    sc = synth.make_scene(128, 120, n_targets=4, seed=40)
    tb = geometry.prepare_tables_from_scene(sc)
    job = geometry.fixed_job(tb, 128)
    ref, _ = fe.form_image(sc.signal, tb, 128, True, True)
    with engine.FixedPlan(128, 120, 128, True, True) as plan:
        job["sinc_q15"] = np.asarray(tables.sinc_table_q15(), np.int16).reshape(256, 32)
        plan.set_job(job)
        assert np.array_equal(plan.form(sc.signal), ref)
        job["sinc_q15"] = np.full((256, 32), 32767, np.int16)
        with pytest.raises(_lib.PfaError) as ei:
            plan.set_job(job)
        assert ei.value.status == _lib.BAD_ARG


@pytest.mark.parametrize("rmode,amode,order", [("cubic", "cubic", "emulator"), ("cubic", "sinc", "fused"),
                                               ("lerp", "cubic", "fused"), ("sinc", "sinc", "fused")])
def test_silicon_variants_bit_exact(torch_cuda, rmode, amode, order):
    """The A/B variants (cubic Lagrange resampler, silicon detect order) against the oracle restating
    gen_resample_vectors.gather_cubic and model_detect_fusion.order_B_fused, bit for bit."""
    sc = synth.make_scene(230, 210, n_targets=8, snr_db=20.0, seed=41, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    ref, _ = fe.form_image(sc.signal, tb, 256, range_mode=rmode, az_mode=amode, detect_order=order)
    with engine.FixedPlan(230, 210, 256, range_interp=rmode, az_interp=amode, detect_order=order) as plan:
        plan.set_tables(tb)
        img = plan.form(sc.signal)
    assert np.array_equal(img, ref), f"{(img != ref).sum()} pixels differ"



def test_largest_grid_matches_reference_crc(torch_cuda):
    """The largest grid (16384^2: 14-stage BFP FFTs of 1024-thread CTAs) against the reference
    emulator's CRC on a tiny scene (too large for the oracle in a test)."""
    c = BIG.get("tiny40x48_g16384_sinc")
    if c is None:
        pytest.skip("golden not generated")
    sc = synth.make_scene(**c["scene"])
    if _crc(sc.signal) != c["input_crc"]:
        pytest.skip("synthetic input not bit-identical on this host")
    tb = geometry.prepare_tables_from_scene(sc)
    img, *_ = _form(torch_cuda, sc.signal, tb, c["grid"], c["range_sinc"], c["az_sinc"])
    assert fe.frame_crc(img) == c["image_crc"]
