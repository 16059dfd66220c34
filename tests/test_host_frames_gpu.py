"""Pipelined host frames (pfa_form_fixed_host_frames / pfa_form_float_host_frames): every frame of a
double-buffered upload/compute/download pipeline equals the same frame formed alone; fixed frames are
bit-exact against the oracle."""
import numpy as np
import pytest

from oracle import fixed_emulator as fe
from pfa_b200 import _lib, engine, geometry, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _frames(torch, sc, count, seed):
    """``count`` different signals on one acquisition geometry, in pinned host memory."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        noise = (rng.standard_normal(sc.signal.shape) + 1j * rng.standard_normal(sc.signal.shape)) * 0.05
        x = (sc.signal * (0.5 + 0.25 * k) + noise).astype(np.complex64)
        buf = torch.empty(x.shape, dtype=torch.complex64).pin_memory().numpy()
        buf[...] = x
        out.append(buf)
    return out


@pytest.mark.parametrize("count", [1, 2, 5])
def test_fixed_frames_match_oracle(torch_cuda, count):
    sc = synth.make_scene(200, 190, n_targets=5, snr_db=20.0, seed=71)
    tb = geometry.prepare_tables_from_scene(sc)
    sigs = _frames(torch_cuda, sc, count, 72)
    with engine.FixedPlan(200, 190, 256, True, True) as plan:
        plan.set_tables(tb)
        imgs = plan.form_host_frames(sigs)
        again = plan.form_host_frames(sigs)            # staging reuse
        single = [plan.form_host(s) for s in sigs]
    for k, s in enumerate(sigs):
        ref, _ = fe.form_image(s, tb, 256, True, True)
        assert np.array_equal(imgs[k], ref), f"frame {k}: {(imgs[k] != ref).sum()} pixels differ"
        assert np.array_equal(again[k], ref) and np.array_equal(single[k], ref)


@pytest.mark.parametrize("detect", ["mag", "complex"])
def test_float_frames_match_single_frames(torch_cuda, detect):
    sc = synth.make_scene(300, 260, n_targets=5, seed=73, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    sigs = _frames(torch_cuda, sc, 4, 74)
    with engine.FloatPlan(300, 260) as plan:
        plan.set_tables(tb)
        imgs = plan.form_host_frames(sigs, detect=detect)
        single = [plan.form_host(s, detect=detect) for s in sigs]
    for k in range(len(sigs)):
        assert np.array_equal(imgs[k], single[k]), f"frame {k} differs from the single-frame result"


def test_frames_errors(torch_cuda):
    sc = synth.make_scene(128, 120, n_targets=3, seed=75)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FixedPlan(128, 120, 128) as plan:
        plan.set_tables(tb)
        assert plan.form_host_frames([]) == []
        with pytest.raises(ValueError):
            plan.form_host_frames([sc.signal.astype(np.complex128)])
        with pytest.raises(ValueError):
            plan.form_host_frames([sc.signal], outs=[])
        st = plan._lib.pfa_form_fixed_host_frames(plan.handle, None, None, 1)
        assert st == _lib.BAD_ARG
    with engine.FloatPlan(128, 120) as fplan:
        fplan.set_tables(tb)
        sig = np.ascontiguousarray(sc.signal, np.complex64)
        out = np.empty((128, 128), np.float32)
        st = fplan._lib.pfa_form_float_host_frames(fplan.handle, engine._frame_ptrs([sig]),
                                                   engine._frame_ptrs([out]), 7, 1)
        assert st == _lib.BAD_ARG
        st = fplan._lib.pfa_form_fixed_host_frames(fplan.handle, engine._frame_ptrs([sig]),
                                                   engine._frame_ptrs([out]), 1)
        assert st == _lib.BAD_CONFIG


def test_mixed_host_frames(torch_cuda):
    """Split-precision plans through the host entry points (both axes on the tensor cores): pipelined
    frames equal single frames, and the completion-wait status reads clean."""
    sc = synth.make_scene(2000, 1800, n_targets=8, seed=76, jitter=0.3)
    tb = geometry.prepare_tables_from_scene(sc)
    sigs = _frames(torch_cuda, sc, 3, 77)
    with engine.FloatPlan(2000, 1800, mixed=True) as plan:
        plan.set_tables(tb)
        imgs = plan.form_host_frames(sigs)
        single = [plan.form_host(s) for s in sigs]
    for k in range(len(sigs)):
        assert np.array_equal(imgs[k], single[k])


def test_scene_queue_new_geometry_each_frame(torch_cuda):
    """engine.form_host_scenes: scenes of different geometries (same shape) with the next scene's tables
    prepared on a host thread during the current frame; fixed images bit-exact against the oracle per
    scene (a job left over from the previous scene would change the image), float images equal to the
    same scene formed alone."""
    scenes = [synth.make_scene(200, 190, n_targets=5, snr_db=20.0, seed=80 + k, jitter=0.2 * k,
                              aperture_deg=2.5 + 0.5 * k) for k in range(4)]
    prep = lambda sc: (geometry.prepare_tables_from_scene_fast(sc), sc.signal)
    with engine.FixedPlan(200, 190, 256, True, True) as plan:
        imgs = engine.form_host_scenes(plan, scenes, prep)
        reused = engine.form_host_scenes(plan, scenes[:2], prep, outs=[np.empty((256, 256), np.uint16)])
    for k, sc in enumerate(scenes):
        ref, _ = fe.form_image(sc.signal, geometry.prepare_tables_from_scene(sc), 256, True, True)
        assert np.array_equal(imgs[k], ref), f"scene {k}: {(imgs[k] != ref).sum()} pixels differ"
    assert np.array_equal(reused[1], imgs[1])
    with engine.FloatPlan(200, 190) as plan:
        fimgs = engine.form_host_scenes(plan, scenes, prep, detect="complex")
        for k, sc in enumerate(scenes):
            plan.set_tables(geometry.prepare_tables_from_scene(sc))
            assert np.array_equal(fimgs[k], plan.form_host(sc.signal, detect="complex")), k
