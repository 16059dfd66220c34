"""GPU parity of the split-precision (mixed) float mode: FFTs as fp16 hi/lo DFT-matrix products on the
tensor cores with fp32 accumulation, against the FP64 oracle of form_image_pfa.pfa.

Stated tolerance (the mixed mode's error budget): relative L2 of the complex and the detected image
against FP64 <= 1e-4; point-target peak position identical, ISLR within 0.01 dB of FP64.  At the full
8192^2 size (too large for the FP64 oracle in a test) the mixed image is checked against the FP32 image,
itself pinned to FP64 at 1e-6.
"""
import numpy as np
import pytest

from oracle import float_pfa as fp
from pfa_b200 import engine, geometry, synth

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(sig, tables, mixed, detect="mag", rs=False, az=False, centred=True, window=True):
    m, n = sig.shape
    with engine.FloatPlan(m, n, rs, az, mixed=mixed) as plan:
        plan.set_tables(tables, window=window, centred=centred)
        return plan.form(sig, detect=detect)


# (m, n): both axes on the tensor cores (2048, 4096 points), and one axis each
@pytest.mark.parametrize("m,n", [(2000, 1900), (3000, 2500), (1500, 700), (700, 3500)])
def test_mixed_lerp_vs_fp64(torch_cuda, m, n):
    sc = synth.make_scene(m, n, n_targets=32, clutter_db=-10.0, snr_db=15.0, seed=m + 7 * n, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    cz = _run(sc.signal, tb, True, detect="complex")
    det = _run(sc.signal, tb, True)
    r64 = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64")
    e_c, e_d = fp.rel_l2(cz, r64), fp.rel_l2(det, np.abs(r64))
    assert e_c <= TOL and e_d <= TOL, (e_c, e_d)


def test_mixed_sinc_power_inverse_natural(torch_cuda):
    sc = synth.make_scene(2048, 2048, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=61)
    tb = dict(geometry.prepare_tables_from_scene(sc))
    f32 = _run(sc.signal, tb, False, detect="complex", rs=True, az=True)
    mx = _run(sc.signal, tb, True, detect="complex", rs=True, az=True)
    assert fp.rel_l2(mx, f32) <= TOL
    pw32 = _run(sc.signal, tb, False, detect="power")
    pwmx = _run(sc.signal, tb, True, detect="power")
    assert fp.rel_l2(pwmx, pw32) <= 2 * TOL
    nat32 = _run(sc.signal, tb, False, detect="complex", centred=False)
    natmx = _run(sc.signal, tb, True, detect="complex", centred=False)
    assert fp.rel_l2(natmx, nat32) <= TOL
    tb["sgn"] = 1
    inv32 = _run(sc.signal, tb, False, detect="complex")
    invmx = _run(sc.signal, tb, True, detect="complex")
    assert fp.rel_l2(invmx, inv32) <= TOL


def test_mixed_point_target_quality(torch_cuda):
    sc = synth.make_scene(2048, 2048, n_targets=1, scene_half=60.0, snr_db=None, seed=62)
    tb = geometry.prepare_tables_from_scene(sc)
    det = _run(sc.signal, tb, True)
    r64 = np.abs(fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64"))
    pk = np.unravel_index(np.argmax(r64), r64.shape)
    assert np.unravel_index(np.argmax(det), det.shape) == pk
    p0, i0 = fp.peak_islr(r64, pk)
    p1, i1 = fp.peak_islr(det, pk)
    assert abs(i1 - i0) < 0.01 and abs(p1 / p0 - 1) < 1e-4


def test_mixed_full_size_vs_fp32(torch_cuda):
    torch = torch_cuda
    sc, sig = synth.make_scene_device(8167, 8192, n_targets=256, clutter_db=-10.0, snr_db=15.0, seed=3)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(8167, 8192) as p32, engine.FloatPlan(8167, 8192, mixed=True) as pmx:
        p32.set_tables(tb)
        pmx.set_tables(tb)
        a = p32.form(sig, detect="complex")
        b = pmx.form(sig, detect="complex")
        err = float(torch.linalg.vector_norm(b - a) / torch.linalg.vector_norm(a))
    assert err <= TOL, err


def test_bounded_wait_runs_out_and_the_context_recovers(torch_cuda):
    """Every tensor-core completion wait is bounded.  A plan whose range FFT first waits on a barrier that
    nothing arrives on (the test hook pfa_config.test_wait_polls) gives up, issues no MMA, and the
    synchronous entry point returns PFA_ERR_TIMEOUT; the context stays usable and a normal plan right
    after forms the correct frame."""
    from pfa_b200 import _lib
    sc = synth.make_scene(600, 2000, n_targets=8, clutter_db=-10.0, snr_db=20.0, seed=66)   # range: 2048 points
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(600, 2000, mixed=True, test_wait_polls=2000) as p:
        p.set_tables(tb)
        with pytest.raises(_lib.PfaError) as ei:
            p.form_host(sc.signal)
        assert ei.value.status == _lib.TIMEOUT
        assert "timed out" in str(ei.value)
    mx = _run(sc.signal, tb, True, detect="complex")
    f32 = _run(sc.signal, tb, False, detect="complex")
    assert fp.rel_l2(mx, f32) <= TOL
