"""GPU: the allocation-free entry point pfa_form_fixed_noalloc.

It exists for callers that cannot allocate device memory (a host that owns all device memory through
its own pool, a real-time loop that must not touch the allocator, a process whose allocator is
exhausted).  It keeps its scratch in one static device array, so this test calls it through the C ABI
twice in a row on different frames (the second call must not see the first call's leftovers) and checks
each image against the planned entry point pfa_form_fixed and against the CPU oracle of the emulator's
datapath, bit for bit (the fixed-point tolerance is 0).  One of the calls passes its own copy of the sinc
table (the caller-supplied table branch).  It also checks that a frame above the array's limit (grid 1024)
is rejected with PFA_ERR_TOO_LARGE.
This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import fixed_emulator as fe
from pfa_b200 import _lib, engine, geometry, synth

pytestmark = pytest.mark.gpu


def _job(tables, grid, sinc=None):
    j = geometry.fixed_job(tables, grid)
    inv = np.empty(j["m"], np.int32)
    inv[j["order"]] = np.arange(j["m"], dtype=np.int32)
    keep = [j["f0"], j["df"], j["pr"], j["tan_s"], inv, j["krp"], j["kcp"],
            np.ascontiguousarray(j["hamr"], np.int32), np.ascontiguousarray(j["hamc"], np.int32),
            np.ascontiguousarray(j["twiddle"], np.int16)]
    if sinc is not None:
        keep.append(np.ascontiguousarray(sinc, np.int16))
    ptrs = [C.c_void_p(a.ctypes.data) for a in keep] + ([] if sinc is not None else [None])
    return _lib.FixedJob(*ptrs), keep


def _noalloc(torch, sig, tables, grid, rs, az, sinc=None):
    lib = _lib.load()
    m, n = sig.shape
    cfg = _lib.Config(mode=_lib.MODE_FIXED, m=m, n=n, grid=grid, range_interp=int(rs), az_interp=int(az), device=0)
    job, keep = _job(tables, grid, sinc)
    x = torch.from_numpy(np.ascontiguousarray(sig)).cuda()
    img = torch.empty((grid, grid), dtype=torch.uint16, device="cuda")
    st = lib.pfa_form_fixed_noalloc(C.byref(cfg), C.byref(job), C.c_void_p(x.data_ptr()), C.c_void_p(img.data_ptr()),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.OK, lib.pfa_status_string(st)
    torch.cuda.synchronize()
    return img.cpu().numpy()


def _planned(torch, sig, tables, grid, rs, az):
    m, n = sig.shape
    with engine.FixedPlan(m, n, grid, rs, az) as plan:
        plan.set_tables(tables)
        return plan.form(torch.from_numpy(np.ascontiguousarray(sig)).cuda()).cpu().numpy()


def test_noalloc_matches_planned_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # the reference's own table, passed explicitly in the second call ([phase][tap] int16, host memory)
    own_sinc = np.array(fe._tab(), dtype=np.int16).reshape(256, 32)
    cases = [
        (synth.make_scene(900, 1000, n_targets=16, clutter_db=-10.0, snr_db=20.0, seed=41, jitter=0.3), 1024, True, True,
         None),
        (synth.make_scene(300, 250, n_targets=8, snr_db=20.0, seed=42), 512, False, True, own_sinc),
    ]
    for sc, grid, rs, az, sinc in cases:
        tables = geometry.prepare_tables_from_scene(sc)
        got = _noalloc(torch, sc.signal, tables, grid, rs, az, sinc)
        want = _planned(torch, sc.signal, tables, grid, rs, az)
        assert got.shape == want.shape
        assert np.array_equal(got, want), f"{(got != want).sum()} pixels differ"
        ref, _ = fe.form_image(sc.signal, tables, grid, range_sinc=rs, az_sinc=az)
        assert np.array_equal(got, ref), f"{(got != ref).sum()} pixels differ from the oracle"
        assert got.any()


def test_noalloc_rejects_frames_above_its_limit():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    sc = synth.make_scene(1500, 1200, n_targets=4, seed=43, with_signal=False)
    sc.signal = np.zeros((1500, 1200), np.complex64)
    tables = geometry.prepare_tables_from_scene(sc)
    job, keep = _job(tables, 2048)
    cfg = _lib.Config(mode=_lib.MODE_FIXED, m=1500, n=1200, grid=2048, range_interp=1, az_interp=1, device=0)
    x = torch.zeros((1500, 1200), dtype=torch.complex64, device="cuda")
    img = torch.empty((2048, 2048), dtype=torch.uint16, device="cuda")
    st = lib.pfa_form_fixed_noalloc(C.byref(cfg), C.byref(job), C.c_void_p(x.data_ptr()), C.c_void_p(img.data_ptr()), None)
    assert st == _lib.TOO_LARGE
    assert b"1024" in lib.pfa_status_string(st)
