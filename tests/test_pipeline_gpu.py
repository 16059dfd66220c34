"""GPU: the scene pipeline over the engine (sar_pipeline.process_scene / watch,
mpfs/host/sar_pipeline.py:118-163): CPHD file -> tables -> pinned signal -> device frame -> display
scaling -> GeoTIFF, checked against the same steps taken one by one (the float image against the FP64
oracle, the display bytes against the reference arithmetic); the watch loop skips a broken file."""
import numpy as np
import pytest

from oracle import float_pfa as fp, geotiff_ref
from pfa_b200 import cphd, geocode, geometry, pipeline, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _placed_scene(seed):
    """A synthetic scene moved to a place on the Earth (a common ECEF offset leaves every look vector,
    hence the tables and the image, unchanged) so that the UTM affine is meaningful."""
    sc = synth.make_scene(700, 650, n_targets=12, clutter_db=-10.0, snr_db=20.0, seed=seed, jitter=0.2)
    off = geocode.geodetic_to_ecef(-96.8, 46.9, 270.0)
    sc.tx, sc.rcv, sc.srp = sc.tx + off, sc.rcv + off, sc.srp + off
    return sc


def test_process_scene_matches_the_steps(torch_cuda, tmp_path):
    Image = pytest.importorskip("PIL.Image")
    sc = _placed_scene(51)
    src = cphd.write_scene(tmp_path / "a_CPHD.cphd", sc)
    be = pipeline.B200Backend()
    out = pipeline.process_scene(src, tmp_path / "out", be)
    assert out.name == "a_detected.tif"
    tb = geometry.prepare_tables_from_scene(sc)
    det = be.focus(sc.signal, tb)
    r64 = np.abs(fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64"))
    assert fp.rel_l2(det, r64) <= 1e-6
    want, _ = geotiff_ref.display_u8(det)
    assert np.array_equal(np.array(Image.open(out)), want)
    im = Image.open(out)
    epsg, aff = geocode.geotransform(det.shape, tb["geo"], tb["center_ecef"], tb["uiax"], tb["uiay"])
    assert im.tag_v2[34735][-1] == epsg == 32614
    assert np.allclose(im.tag_v2[34264][:8], (aff[0], aff[1], 0.0, aff[2], aff[3], aff[4], 0.0, aff[5]))
    be.close()


def test_watch_processes_every_scene_once_and_skips_a_broken_file(torch_cuda, tmp_path):
    inp = tmp_path / "in"
    inp.mkdir()
    for k in range(2):
        cphd.write_scene(inp / f"s{k}_CPHD.cphd", _placed_scene(60 + k))
    (inp / "broken_CPHD.cphd").write_bytes(b"CPHD/1.0.1\nXML_BLOCK_SIZE := 5\n")
    outs = pipeline.watch(inp, tmp_path / "out", once=True)
    assert sorted(p.name for p in outs) == ["s0_detected.tif", "s1_detected.tif"]
