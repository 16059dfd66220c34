"""Seeded random sweep over shapes and knobs, GPU against the oracle: fixed-point frames bit for bit
(sizes 17..480 on grids 64..512, every interpolator pair including the cubic variant, both detect
orders, descending frequency axes), float frames within 1e-6 of FP64."""
import dataclasses

import numpy as np
import pytest

from oracle import fixed_emulator as fe, float_pfa as fp
from pfa_b200 import engine, geometry, synth

pytestmark = pytest.mark.gpu
MODES = ("lerp", "sinc", "cubic")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scene(rng, m, n, seed):
    sc = synth.make_scene(m, n, n_targets=int(rng.integers(1, 12)), snr_db=float(rng.choice([10.0, 20.0, 40.0])),
                          seed=seed, jitter=float(rng.choice([0.0, 0.3, 0.5])))
    if rng.random() < 0.25:                       # descending frequency axis
        sc = dataclasses.replace(sc, sc0=sc.sc0 + (n - 1) * sc.scss, scss=-sc.scss)
    return sc


@pytest.mark.parametrize("case", range(12))
def test_fixed_random(torch_cuda, case):
    rng = np.random.default_rng(1000 + case)
    G = int(rng.choice([64, 128, 256, 512]))
    m = int(rng.integers(max(4, G // 8), G + 1))
    n = int(rng.integers(max(4, G // 8), G + 1))
    rmode, amode = (str(x) for x in rng.choice(MODES, 2))
    order = "fused" if rng.random() < 0.3 else "emulator"
    sc = _scene(rng, m, n, 2000 + case)
    tb = geometry.prepare_tables_from_scene(sc)
    ref, _ = fe.form_image(sc.signal, tb, G, range_mode=rmode, az_mode=amode, detect_order=order)
    with engine.FixedPlan(m, n, G, range_interp=rmode, az_interp=amode, detect_order=order) as plan:
        plan.set_tables(tb)
        img = plan.form(sc.signal)
    assert np.array_equal(img, ref), (m, n, G, rmode, amode, order, int((img != ref).sum()))


@pytest.mark.parametrize("case", range(8))
def test_float_random(torch_cuda, case):
    rng = np.random.default_rng(3000 + case)
    m = int(rng.integers(40, 700))
    n = int(rng.integers(40, 700))
    sinc = bool(rng.random() < 0.5)
    sc = _scene(rng, m, n, 4000 + case)
    tb = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(m, n, sinc, sinc) as plan:
        plan.set_tables(tb)
        cz = plan.form(sc.signal, detect="complex")
    g2, _ = fp.resample_kspace(sc.signal, tb["freq"], tb["ax"], tb["ay"], precision="f64",
                               interp="sinc" if sinc else "lerp")
    ref = fp.focus(g2, tb["sgn"], precision="f64")
    assert fp.rel_l2(cz, ref) <= 1e-6, (m, n, sinc)
