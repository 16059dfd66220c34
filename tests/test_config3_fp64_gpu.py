"""GPU: the production-shape float frame and 8192-point tensor-core lines against the FP64 oracle.

The float mode's stated tolerances, against the FP64 restatement of form_image_pfa.pfa
(src/form_image_pfa.py:165-246 in float64/complex128, ``oracle.float_pfa`` with ``precision="f64"``):

* FP32 path: relative L2 of the complex and of the detected image <= 1e-6; phase RMS <= 1e-5 rad;
* split-precision tensor-core path (mixed): relative L2 <= 1e-4; phase RMS <= 1e-4 rad;
* both: the peak pixel of each of the 64 strongest point responses unchanged, peak power within the
  relative L2 tolerance x 10 and ISLR within 0.01 dB of FP64.

The full frame is the 8167 x 8192 scene of 1024 point targets plus Rayleigh clutter at 15 dB SNR (seed 3)
onto the 8192^2 raster; its FP64 image takes the oracle about 15 s (lerp) or a minute (sinc) on the host.
The line tests put 8192-point lines on the tensor cores along each axis in turn (8192 x 300 and 300 x 8192).
"""
import numpy as np
import pytest

from oracle import float_pfa as fp
from pfa_b200 import engine, geometry, synth

pytestmark = pytest.mark.gpu
TOL = {False: 1e-6, True: 1e-4}          # relative L2 by mode (mixed = True)
PHASE_TOL = {False: 1e-5, True: 1e-4}    # phase RMS (rad) by mode


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _form(sig, tables, mixed, sinc):
    m, n = sig.shape
    with engine.FloatPlan(m, n, sinc, sinc, mixed=mixed) as plan:
        plan.set_tables(tables)
        out = plan.form(sig, detect="complex")
    return out.cpu().numpy() if not isinstance(out, np.ndarray) else out


def _check(rep, mixed, what):
    tol = TOL[mixed]
    assert rep["rel_l2_complex"] <= tol and rep["rel_l2_detected"] <= tol, (what, rep)
    assert rep["phase_rms_rad"] <= PHASE_TOL[mixed], (what, rep)
    assert rep["peak_pos_match"] == 1.0, (what, rep)
    assert rep["peak_power_rel_err_max"] <= 10 * tol and rep["islr_err_db_max"] <= 0.01, (what, rep)


@pytest.mark.parametrize("sinc", [False, True], ids=["lerp", "sinc"])
@pytest.mark.parametrize("m,n", [(8192, 300), (300, 8192)], ids=["cross8192", "range8192"])
def test_8192_point_tensor_core_lines_vs_fp64(torch_cuda, m, n, sinc):
    sc = synth.make_scene(m, n, n_targets=48, clutter_db=-10.0, snr_db=15.0, seed=m + 3 * n + sinc, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    r64 = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64",
                       interp="sinc" if sinc else "lerp")
    for mixed in (False, True):
        img = _form(sc.signal, tb, mixed, sinc)
        _check(fp.error_report(img, r64, k=16), mixed, ("mixed" if mixed else "fp32", m, n, sinc))


@pytest.fixture(scope="module")
def ndsu(torch_cuda):
    """The production-shape scene (device synthesis), its host copy and tables."""
    wl = {k: v for k, v in synth.WORKLOADS["ndsu_8167x8192"].items() if k not in ("m", "n")}
    sc, sig = synth.make_scene_device(8167, 8192, **wl)
    tb = geometry.prepare_tables_from_scene(sc)
    return sig, sig.cpu().numpy(), tb


@pytest.mark.parametrize("sinc", [False, True], ids=["lerp", "sinc"])
def test_production_frame_vs_fp64(ndsu, sinc):
    sig, sig_h, tb = ndsu
    r64 = fp.pfa_image(sig_h, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64",
                       interp="sinc" if sinc else "lerp")
    for mixed in (False, True):
        img = _form(sig, tb, mixed, sinc)
        _check(fp.error_report(img, r64, k=64), mixed, ("mixed" if mixed else "fp32", "8167x8192", sinc))
        del img
