"""GPU: the autofocus adjoint against an FP64 torch-autograd reference and central finite differences
of the FP64 objective (tolerance 1e-3 relative, per the stated target), plus a focusing run.  Covered:
the lerp passes, the float 32-tap sinc in either or both passes (its transposed resample is the
segmented reduction of the cross adjoint), and descending pass-1 and pass-2 source axes."""
import numpy as np
import pytest

from oracle import autofocus_ref as afr
from pfa_b200 import autofocus, engine, geometry, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scene(m, n, seed):
    sc = synth.make_scene(m, n, n_targets=8, clutter_db=-10.0, snr_db=20.0, seed=seed)
    tb = geometry.prepare_tables_from_scene(sc)
    phi = afr.phase_error(m, seed=seed)
    sig = (sc.signal * np.exp(1j * phi)[:, None]).astype(np.complex64)
    return sig, tb, phi


@pytest.mark.parametrize("m,n,seed", [(128, 128, 4), (256, 256, 5), (200, 240, 6)])
def test_gradient_matches_fp64_autograd(torch_cuda, m, n, seed):
    torch = torch_cuda
    sig, tb, phi = _scene(m, n, seed)
    theta = np.random.default_rng(seed).normal(0.0, 0.3, m)
    e64, g64 = afr.entropy_and_grad(sig, tb, theta)
    with engine.FloatPlan(m, n) as plan:
        plan.set_tables(tb)
        ent, g = autofocus.entropy_grad(plan, torch.from_numpy(sig).cuda(),
                                        torch.from_numpy(theta.astype(np.float32)).cuda())
    g = g.cpu().numpy().astype(np.float64)
    assert abs(float(ent) - e64) / abs(e64) < 1e-5
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 1e-3
    idx = [1, m // 3, m // 2, m - 2]
    fd = afr.fd_grad(sig, tb, theta, idx)
    assert np.abs(g[idx] - fd).max() / np.abs(fd).max() < 1e-3


def _check_grad(torch, sig, tb, theta, rs, az):
    m, n = sig.shape
    ri, ai = ("sinc" if rs else "lerp"), ("sinc" if az else "lerp")
    e64, g64 = afr.entropy_and_grad(sig, tb, theta, ri, ai)
    with engine.FloatPlan(m, n, rs, az) as plan:
        plan.set_tables(tb)
        ent, g = autofocus.entropy_grad(plan, torch.from_numpy(sig).cuda(),
                                        torch.from_numpy(theta.astype(np.float32)).cuda())
    g = g.cpu().numpy().astype(np.float64)
    assert abs(float(ent) - e64) / abs(e64) < 1e-5, (float(ent), e64)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 1e-3, np.linalg.norm(g - g64) / np.linalg.norm(g64)
    idx = [1, m // 3, m // 2, m - 2]
    fd = afr.fd_grad(sig, tb, theta, idx, range_interp=ri, az_interp=ai)
    assert np.abs(g[idx] - fd).max() / np.abs(fd).max() < 1e-3


@pytest.mark.parametrize("rs,az,m,n,seed", [(True, True, 128, 128, 8), (False, True, 256, 256, 9),
                                            (True, False, 200, 240, 10), (True, True, 300, 160, 11)])
def test_sinc_gradient_matches_fp64_autograd(torch_cuda, rs, az, m, n, seed):
    sig, tb, phi = _scene(m, n, seed)
    theta = np.random.default_rng(seed).normal(0.0, 0.3, m)
    _check_grad(torch_cuda, sig, tb, theta, rs, az)


@pytest.mark.parametrize("rs,az", [(False, False), (True, True)])
def test_gradient_with_descending_source_axes(torch_cuda, rs, az):
    """Negative frequencies make every pulse's wavenumbers and KR negative: both passes resample from
    descending source axes (the forward mirrors its brackets, the adjoint maps slots back)."""
    sig, tb, phi = _scene(128, 144, 12)
    tb = {k: v for k, v in tb.items() if k not in ("KR", "KC")}     # recomputed from the negated frequencies
    tb["freq"] = -np.asarray(tb["freq"])
    theta = np.random.default_rng(12).normal(0.0, 0.3, 128)
    _check_grad(torch_cuda, sig, tb, theta, rs, az)


def test_autograd_function_and_focusing(torch_cuda):
    torch = torch_cuda
    sig, tb, phi = _scene(256, 256, 7)
    x = torch.from_numpy(sig).cuda()
    with engine.FloatPlan(256, 256) as plan:
        plan.set_tables(tb)
        th = torch.zeros(256, device="cuda", requires_grad=True)
        e = autofocus.image_entropy(th, plan, x)
        e.backward()
        _, g = autofocus.entropy_grad(plan, x, torch.zeros(256, device="cuda"))
        assert torch.allclose(th.grad, g)
        theta, hist = autofocus.autofocus(plan, x, steps=50, step=0.3, history=True)
    assert hist[-1] < hist[0]
    e_true = afr.entropy(sig, tb, phi)
    assert hist[-1] <= e_true + 0.1 * (hist[0] - e_true)


def test_device_step_and_corrected_form(torch_cuda):
    """pfa_autofocus_step equals the gradient plus the host-side update; pfa_form_float_phase equals the
    frame of the corrected signal."""
    torch = torch_cuda
    sig, tb, phi = _scene(256, 240, 13)
    x = torch.from_numpy(sig).cuda()
    with engine.FloatPlan(256, 240) as plan:
        plan.set_tables(tb)
        th0 = torch.from_numpy(np.random.default_rng(13).normal(0.0, 0.2, 256).astype(np.float32)).cuda()
        _, g = autofocus.entropy_grad(plan, x, th0)
        g = g - g.mean()
        want = th0 - 0.3 * g / g.abs().max()
        got = th0.clone()
        autofocus.descent_step(plan, x, got, 0.3)
        assert torch.allclose(got, want, atol=1e-6)
        img = autofocus.form_corrected(plan, x, got, detect="complex")
        corr = x * torch.polar(torch.ones_like(got), -got)[:, None]
        ref = plan.form(corr.contiguous(), detect="complex")
        assert float(torch.linalg.vector_norm(img - ref) / torch.linalg.vector_norm(ref)) <= 1e-6
        # the device loop of autofocus() follows the same path as the one with history
        t_dev, _ = autofocus.autofocus(plan, x, steps=5, step=0.3)
        t_host, h = autofocus.autofocus(plan, x, steps=5, step=0.3, history=True)
        assert torch.allclose(t_dev, t_host, atol=1e-4) and len(h) == 5
