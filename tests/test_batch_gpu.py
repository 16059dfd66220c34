"""GPU: FFT tile variants (the autotuner's knob), the autotuner, and batched uneven scenes in one
CUDA graph against the one-scene-at-a-time path."""
import numpy as np
import pytest

from oracle import float_pfa as fp
from pfa_b200 import autotune, batch, engine, geometry, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("tile", [(8, 8), (8, 16), (16, 8)])
def test_tile_variants_match_fp64(torch_cuda, tile):
    sc = synth.make_scene(600, 900, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=61, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(600, 900, tile=tile) as plan:
        plan.set_tables(tb)
        cz = plan.form(sc.signal, detect="complex")
    r64 = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64")
    assert fp.rel_l2(cz, r64) <= 1e-6


# the 32-value tile (radix-32 passes) exists for lines of 8192 and 16384 points: cross lines of 8192
# (4500 pulses), range lines of 8192 (4500 samples) and cross lines of 16384 (8200 pulses)
@pytest.mark.parametrize("m,n,tile", [(4500, 600, (32, 16)), (700, 4500, (16, 32)), (8200, 500, (32, 32))])
def test_tile32_matches_fp64(torch_cuda, m, n, tile):
    sc = synth.make_scene(m, n, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=63, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(m, n, tile=tile) as plan:
        plan.set_tables(tb)
        cz = plan.form(sc.signal, detect="complex")
    r64 = fp.pfa_image(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64")
    assert fp.rel_l2(cz, r64) <= 1e-6


def test_tile_values_checked(torch_cuda):
    """Tiles other than 0 (automatic), 8, 16 and 32 are a configuration error; 32 on lines it does not
    apply to (here 1024 points) runs the 16-value tile."""
    from pfa_b200 import _lib
    for bad in ((24, 16), (16, 4), (64, 64)):
        with pytest.raises(_lib.PfaError) as ei:
            engine.FloatPlan(600, 900, tile=bad)
        assert ei.value.status == _lib.BAD_CONFIG
    sc = synth.make_scene(600, 900, n_targets=8, seed=64)
    tb = geometry.prepare_tables_from_scene(sc)
    out = []
    for tile in ((32, 32), (16, 16)):
        with engine.FloatPlan(600, 900, tile=tile) as plan:
            plan.set_tables(tb)
            out.append(np.asarray(plan.form(sc.signal, detect="complex")))
    assert np.array_equal(out[0], out[1])


def test_autotuner_picks_a_candidate(torch_cuda, tmp_path, monkeypatch):
    torch = torch_cuda
    monkeypatch.setenv("PFA_TUNE_CACHE", str(tmp_path / "tune.json"))
    autotune._MEM.clear()
    sc = synth.make_scene(512, 1000, n_targets=8, seed=62)
    tb = geometry.prepare_tables_from_scene(sc)
    x = torch.from_numpy(sc.signal).cuda()
    tile, times = autotune.tune_float(tb, x, reps=3)
    assert tile in autotune.CANDIDATES and set(times) == set(autotune.CANDIDATES)
    assert (tmp_path / "tune.json").is_file()
    tile2, _ = autotune.tune_float(tb, x)           # cached
    assert tile2 == tile


def _scenes(torch, shapes, seed0):
    out = []
    for k, (m, n) in enumerate(shapes):
        sc = synth.make_scene(m, n, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=seed0 + k)
        out.append((geometry.prepare_tables_from_scene(sc), torch.from_numpy(sc.signal).cuda()))
    return out


def test_batch_graph_equals_one_at_a_time(torch_cuda):
    torch = torch_cuda
    scenes = _scenes(torch, [(300, 500), (700, 400), (1000, 900), (256, 256), (512, 700)], 70)
    bf = batch.BatchFormer(scenes, streams=3, tiles=[(16, 16), (8, 16), (16, 8), (16, 16), (8, 8)])
    bf.run_eager()
    torch.cuda.synchronize()
    eager = [im.clone() for im in bf.images]
    for im in bf.images:
        im.zero_()
    bf.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, bf.images):
        assert torch.equal(a, b)
    # and each equals a stand-alone plan
    for (tb, x), im in zip(scenes, bf.images):
        with engine.FloatPlan(*x.shape) as p:
            p.set_tables(tb)
            ref = p.form(x)
        assert fp.rel_l2(im.cpu().numpy(), ref.cpu().numpy()) <= 1e-6
    bf.close()


def test_batch_with_autofocus_iterations(torch_cuda):
    torch = torch_cuda
    scenes = _scenes(torch, [(256, 300), (400, 256), (300, 300)], 80)
    bf = batch.BatchFormer(scenes, streams=2, af_iters=3)
    bf.run_eager()
    torch.cuda.synchronize()
    eager = [im.clone() for im in bf.images]
    th_eager = [t.clone() for t in bf.theta]
    bf.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, bf.images):
        assert fp.rel_l2(b.cpu().numpy(), a.cpu().numpy()) <= 1e-4
    for a, b in zip(th_eager, bf.theta):
        assert torch.allclose(a, b, atol=1e-4)
    bf.close()


def test_mixed_batch_graph(torch_cuda):
    """Mixed-precision images in the multi-stream graph (scenes with 2048/4096-point lines on the tensor
    cores next to FP32 ones): the graph replay equals the eager run and each image is within the mixed
    error budget of the FP32 image."""
    torch = torch_cuda
    scenes = _scenes(torch, [(2000, 1500), (700, 3000), (1200, 600)], 90)
    bf = batch.BatchFormer(scenes, streams=3, mixed=True, af_iters=2)
    bf.run_eager()
    torch.cuda.synchronize()
    eager = [im.clone() for im in bf.images]
    bf.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, bf.images):
        assert fp.rel_l2(b.cpu().numpy(), a.cpu().numpy()) <= 1e-4
    ref = batch.BatchFormer(scenes, streams=1, af_iters=2)
    ref.run_eager()
    torch.cuda.synchronize()
    for a, b in zip(ref.images, bf.images):
        assert fp.rel_l2(b.cpu().numpy(), a.cpu().numpy()) <= 1e-4
    ref.close()
    bf.close()


def test_batch_images_against_the_oracle_per_scene(torch_cuda):
    """After the batch's autofocus iterations (device steps in the graph), every scene's image equals the
    FP64 oracle's image of the signal corrected by the batch's own final phase (FP32 images: 1e-6;
    split-precision images: 1e-4)."""
    torch = torch_cuda
    shapes = [(300, 400), (520, 260), (2100, 700)]
    scenes = _scenes(torch, shapes, 95)
    for mixed, tol in ((False, 1e-6), (True, 1e-4)):
        bf = batch.BatchFormer(scenes, streams=2, af_iters=3, mixed=mixed)
        bf.replay()
        torch.cuda.synchronize()
        for (tb, x), im, th in zip(scenes, bf.images, bf.theta):
            t = th.double().cpu().numpy()
            corr = (x.cpu().numpy() * np.exp(-1j * t)[:, None]).astype(np.complex64)
            r64 = np.abs(fp.pfa_image(corr, tb["freq"], tb["ax"], tb["ay"], tb["sgn"], precision="f64"))
            assert fp.rel_l2(im.cpu().numpy(), r64) <= tol, (mixed, tuple(x.shape))
            assert np.abs(t).max() > 0          # the phase did move
        bf.close()
