"""GPU: the device display scaling of save_detected_geotiff (pfa_display_u8, src/form_image_pfa.py:287-292)
against the reference arithmetic (np.percentile(amp, 99.7), clip, uint8), bit for bit: random magnitudes
of many sizes (vector tails, a single element, heavy ties, constant images, a range of scales), other
percentiles, and the detected image of a focused scene; plus the whole GeoTIFF path on that image."""
import numpy as np
import pytest

from oracle import geotiff_ref
from pfa_b200 import engine, geocode, geometry, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _check(torch, amp, pct=99.7):
    x = torch.from_numpy(amp).cuda()
    out, hi = geocode.display_u8(x, pct)
    ref_amp = amp.astype(np.float32)
    ref_hi = np.percentile(ref_amp, pct)
    ref = np.clip(ref_amp / (ref_hi + 1e-12) * 255.0, 0, 255).astype(np.uint8)
    assert float(hi) == float(ref_hi), (float(hi), float(ref_hi), amp.size)
    got = out.cpu().numpy()
    assert np.array_equal(got, ref), (amp.size, int((got != ref).sum()))


@pytest.mark.parametrize("n", [1, 2, 5, 1023, 4096, 100003, 1 << 20, 3_000_001])
def test_random_sizes(torch_cuda, n):
    rng = np.random.default_rng(n)
    _check(torch_cuda, (rng.random(n) * rng.choice([1e-3, 1.0, 7.5, 3e4])).astype(np.float32))


def test_ties_constants_and_percentiles(torch_cuda):
    rng = np.random.default_rng(3)
    ties = rng.integers(0, 40, 500000).astype(np.float32) * 0.25
    _check(torch_cuda, ties)
    _check(torch_cuda, np.full(77777, 3.5, np.float32))
    _check(torch_cuda, np.zeros(1000, np.float32) + np.float32(1e-30))
    ray = rng.rayleigh(1.0, 2_000_000).astype(np.float32)
    for pct in (0.0, 50.0, 99.0, 99.7, 99.99, 100.0):
        _check(torch_cuda, ray, pct)


def test_focused_image_and_geotiff(torch_cuda, tmp_path):
    torch = torch_cuda
    sc = synth.make_scene(1500, 1300, n_targets=32, clutter_db=-10.0, snr_db=20.0, seed=31)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(1500, 1300) as plan:
        plan.set_tables(tb)
        mag = plan.form(torch.from_numpy(sc.signal).cuda())
    cz = None
    ref, ref_hi = geotiff_ref.display_u8(mag.cpu().numpy())
    got, hi = geocode.display_u8(mag)
    assert float(hi) == float(ref_hi) and np.array_equal(got.cpu().numpy(), ref)
    # the file: the synthetic scene sits at the Earth's centre, so give it a real place for the projection
    tbg = dict(tb)
    tbg["center_ecef"] = geocode.geodetic_to_ecef(-96.8, 46.9, 270.0)
    tbg["uiax"], tbg["uiay"] = np.array([0.11, 0.99, 0.0]), np.array([-0.73, 0.08, 0.68])
    path, epsg, aff = geocode.save_detected_geotiff(mag, tbg, tmp_path / "img.tif")
    Image = pytest.importorskip("PIL.Image")
    assert np.array_equal(np.array(Image.open(path)), ref) and epsg == 32614
    del cz
