"""CPU: the sarpy-free CPHD reader (pfa_b200.cphd) on files written by its writer: PVP vectors, signal
(full, decimated, into a caller buffer), the metadata the focusing path reads, tables identical to those of
the in-memory scene, and -- where the reference checkout is present -- the reference's own prepare_tables
(mpfs/host/sar_pipeline.py:36-115) running unchanged on the reader."""
import numpy as np
import pytest

from oracle import refshim
from pfa_b200 import cphd, geometry, synth


@pytest.fixture(scope="module")
def scene_file(tmp_path_factory):
    sc = synth.make_scene(300, 260, n_targets=6, clutter_db=-10.0, snr_db=20.0, seed=17, jitter=0.3)
    path = tmp_path_factory.mktemp("cphd") / "scene_CPHD.cphd"
    cphd.write_scene(path, sc)
    return sc, path


def test_reader_returns_what_was_written(scene_file):
    sc, path = scene_file
    with cphd.open_phase_history(path) as rd:
        assert rd.get_data_size_as_tuple() == ((300, 260),)
        for name, want in (("TxPos", sc.tx), ("RcvPos", sc.rcv), ("SRPPos", sc.srp), ("SC0", sc.sc0),
                           ("SCSS", sc.scss)):
            assert np.array_equal(rd.read_pvp_variable(name, 0), want), name
        meta = rd.cphd_meta
        assert meta.Global.DomainType == "FX" and meta.Global.SGN == -1
        p = meta.SceneCoordinates.ReferenceSurface.Planar
        assert (p.uIAX.X, p.uIAX.Y, p.uIAX.Z) == tuple(sc.uiax) and (p.uIAY.X, p.uIAY.Y, p.uIAY.Z) == tuple(sc.uiay)
        assert np.array_equal(rd.read_chip((0, 300, 1), (0, 260, 1)), sc.signal)
        assert np.array_equal(rd.read_chip((1, 300, 2), (0, 260, 3)), sc.signal[1::2, ::3])
        buf = np.empty((150, 87), np.complex64)
        rd.read_signal_into(buf, rows=(0, 300, 2), cols=(0, 260, 3))
        assert np.array_equal(buf, sc.signal[::2, ::3])


def test_tables_from_file_equal_tables_from_scene(scene_file):
    sc, path = scene_file
    with cphd.open_phase_history(path) as rd:
        a = geometry.prepare_tables_fast(rd, rd.cphd_meta, 1, 1)
    b = geometry.prepare_tables_from_scene_fast(sc)
    for k in ("ax", "ay", "KR", "KC", "tan_phi"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(np.asarray(a["freq"]), np.asarray(b["freq"]))


def test_integer_signal_format(tmp_path):
    sc = synth.make_scene(64, 80, n_targets=2, seed=3)
    sig = (sc.signal / np.abs(sc.signal).max() * 20000.0).astype(np.complex64)
    path = cphd.write_cphd(tmp_path / "i_CPHD.cphd", sig, sc.tx, sc.rcv, sc.srp, sc.sc0, sc.scss, sc.uiax, sc.uiay,
                           fmt="CI4")
    with cphd.open_phase_history(path) as rd:
        assert rd.signal_format == "CI4"
        got = rd.read_chip((0, 64, 1), (0, 80, 1))
    assert np.array_equal(got, (np.rint(sig.real) + 1j * np.rint(sig.imag)).astype(np.complex64))


def test_reference_prepare_tables_runs_on_the_reader(scene_file):
    if not refshim.available():
        pytest.skip("reference checkout not present")
    sc, path = scene_file
    mods = refshim.modules()
    with cphd.open_phase_history(path) as rd:
        ref = mods.pipe.prepare_tables(rd, rd.cphd_meta, 1, 1)
        own = geometry.prepare_tables(rd, rd.cphd_meta, 1, 1)
    for k in ("ax", "ay", "KR", "KC", "tan_phi", "freq"):
        assert np.array_equal(np.asarray(ref[k]), np.asarray(own[k])), k


def test_rejects_non_cphd(tmp_path):
    p = tmp_path / "x.cphd"
    p.write_bytes(b"NITF02.10 not a phase history\f\n")
    with pytest.raises(ValueError):
        cphd.open_phase_history(p)
