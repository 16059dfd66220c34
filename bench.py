"""Benchmark of the B200 PFA focusing engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one PFA frame of the workload over its synthetic phase history.  Default workload: the
Centerfield-shaped fixed-point frame (5634 x 4319 complex64 -> 8192^2, --range-sinc --az-sinc,
256 point targets + Rayleigh clutter at -10 dB, seed 2), bit-exact to the reference emulator.

Metric: ms per 8192^2 frame (lower is better).  `value` is the device-timed whole-job ms per frame
with inputs resident in HBM (CUDA events on the launching stream, max over ranks); `e2e` is the same
metric through the pipelined host-buffer C-ABI entry point (pinned host signals in, images out, all
copies inside the timed region; uploads and downloads overlap neighbouring frames).  Frames are independent, so N GPUs run N replicas (weak scaling, no
collective on the data path).  Inputs (195 MB signal, 268 MB FFT-2 buffer) exceed the 126 MB L2, so
no explicit flush is done between frames.

--impl reference times the CPU restatement of the reference's emulator (the oracle port in C; the
reference itself is Python and does not travel): one whole frame per step on every host core, its
image CRC checked against the reference emulator's; it prints the same JSON line with
"impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "mpfs250t-sar-ifp_b200"))

METRIC = "ms per 8192^2 PFA frame (mixed vs FP32 at stated err vs FP64); autofocus grads/s"
FPGA_FRAME_MS = {"centerfield_5634x4319": 14170.0, "ndsu_8167x8192": 15738.0}   # published MPFS250T fabric frame times

WORKLOADS = {
    "centerfield_5634x4319": dict(mode="fixed", grid=8192, range_sinc=True, az_sinc=True, scene="centerfield_5634x4319",
                                  desc="Centerfield-shaped 5634x4319 c64 -> 8192^2, fixed point, "
                                       "--deci 1 --grid 8192 --range-sinc --az-sinc, 256 targets + "
                                       "Rayleigh clutter -10 dB, seed 2",
                                  # CRC-32 of the unmodified reference emulator's image of this frame
                                  ref_crc=0x7A44896A, ref_emulator_s=176.7),
    "ndsu_8167x8192_fp32": dict(mode="float", mixed=False, range_sinc=False, az_sinc=False, scene="ndsu_8167x8192",
                                desc="NDSU-shaped 8167x8192 c64 -> 8192^2, float FP32 (lerp, form_image_pfa), "
                                     "1024 targets + Rayleigh clutter -10 dB, 15 dB SNR, seed 3"),
    "ndsu_8167x8192_fp32_sinc": dict(mode="float", mixed=False, range_sinc=True, az_sinc=True, scene="ndsu_8167x8192",
                                     desc="NDSU-shaped 8167x8192 c64 -> 8192^2, float FP32, 32-tap sinc both passes, "
                                          "1024 targets + Rayleigh clutter -10 dB, 15 dB SNR, seed 3"),
}


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.gettempdir()) / f"pfa_bench_clocks_dev{device}_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.is_file():
            return None
        rows = [ln.split(",") for ln in self.path.read_text().splitlines() if ln.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _profile_value(kernel: str, workload: str, key: str):
    """A `key: value` line of the committed ncu summary profiles/<kernel>__<workload>.md (or None)."""
    p = ROOT / "profiles" / f"{kernel}__{workload}.md"
    if not p.is_file():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith(key + ":"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def _traffic(kernel: str, workload: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from the ncu summary."""
    return _profile_value(kernel, workload, "dram_bytes_per_launch")


def stage_bytes(stage: str, m: int, n: int, G: int, mode: str = "fixed") -> float:
    """Algorithmic (compulsory) HBM bytes per launch of each kernel (G = pow2 raster side)."""
    mpad = (m + 31) // 32 * 32
    if mode == "float":
        return {
            "pass1": 8.0 * m * n + 8.0 * n * mpad,          # read c64 signal, write c64 range-bin rows
            "pass2_win_fft1": 8.0 * n * mpad + 8.0 * n * G,  # read rows, write cross-FFT rows
            "fft2_detect": 8.0 * n * G + 4.0 * G * G,        # read cross-FFT columns, write f32 |img|
        }[stage]
    return {
        "q0max": 8.0 * m * n,                              # read the complex64 signal
        "pass1": 8.0 * m * n + 4.0 * n * mpad,             # read signal, write int16x2 range-bin rows
        "pass2_win_fft1": 4.0 * n * mpad + 4.0 * n * G,     # read rows, write FFT-1 rows
        "fft2": 4.0 * n * G + 4.0 * G * G,                  # read FFT-1 columns (rows < n), write FFT-2 rows
        "renorm_detect": 4.0 * G * G + 2.0 * G * G,         # read FFT-2, write uint16 image
    }[stage]


def _device_ms(fn, steps, warmup):
    """Mean device time (ms) of fn() over `steps` calls after `warmup`, CUDA events on the current stream."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def cpu_float_small(sc, tables):
    """CPU baseline of the small float scene: the oracle's restatement of form_image_pfa (np.interp
    passes, float32 window, NumPy 2 single-precision FFT, |z|), lerp, whole frame, one core, best of 3."""
    from oracle import float_pfa as fp
    best = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        fp.detect(fp.pfa_image(sc.signal, tables["freq"], tables["ax"], tables["ay"], tables["sgn"], precision="ref"))
        best = min(best, time.perf_counter() - t0)
    return {"value": round(best * 1000.0, 1), "unit": "ms/frame", "cores": 1, "kind": "port",
            "sample": "whole 1024x1024 frame, form_image_pfa restated (lerp), best of 3"}


def _float_e2e(sig, tables, local):
    """FP32 lerp frames end to end through the pipelined host-buffer entry point (pinned host in/out)."""
    import torch
    from pfa_b200 import engine
    sig_h = torch.empty(tuple(sig.shape), dtype=torch.complex64).pin_memory()
    sig_h.copy_(sig)
    outs_h = [torch.empty((8192, 8192), dtype=torch.float32).pin_memory() for _ in range(2)]
    with engine.FloatPlan(8167, 8192, device=local) as hp:
        hp.set_tables(tables)
        frames = [sig_h.numpy()] * 4
        outs = [outs_h[k & 1].numpy() for k in range(4)]
        hp.form_host_frames(frames[:2], outs[:2])
        t0 = time.perf_counter()
        hp.form_host_frames(frames, outs)
        ms = round((time.perf_counter() - t0) * 1000.0 / 4, 4)
    return ms, {"h2d": int(sig_h.numel() * 8), "d2h": 8192 * 8192 * 4}


def float_cpu_leg(sig_np, tables, interp, imgs):
    """CPU baseline and FP64 checker of the production-shape float frame (8167x8192 -> 8192^2).

    lerp: the reference-precision restatement of form_image_pfa.resample_kspace + focus + |.| (complex64,
    np.interp, NumPy FFT) over the whole frame on one core is the cpu_baseline; the FP64 restatement of the
    same algorithm is the checker.  sinc: the reference has no float sinc, so the FP64 restatement of the
    float sinc (over all host cores) is both.  Returns (cpu_baseline dict, {mixed: errors vs FP64})."""
    from oracle import cpu_sample, float_pfa as fp
    cores = cpu_sample.available_cores()
    t0 = time.perf_counter()
    r64 = fp.pfa_image(sig_np, tables["freq"], tables["ax"], tables["ay"], tables["sgn"], precision="f64",
                       interp=interp, threads=cores if interp == "sinc" else 1)
    t64 = time.perf_counter() - t0
    if interp == "lerp":
        t0 = time.perf_counter()
        fp.detect(fp.pfa_image(sig_np, tables["freq"], tables["ax"], tables["ay"], tables["sgn"], precision="ref"))
        cpu = {"value": round((time.perf_counter() - t0) * 1000.0, 1), "unit": "ms/frame", "cores": 1, "kind": "port",
               "sample": "whole 8167x8192 frame, form_image_pfa restated at its own precision (np.interp passes, "
                         "complex64, NumPy FFT, |z|)"}
    else:
        cpu = {"value": round(t64 * 1000.0, 1), "unit": "ms/frame", "cores": cores, "kind": "port",
               "sample": "whole 8167x8192 frame, FP64 restatement of the float 32-tap sinc PFA (the reference "
                         "has no float sinc), sinc lines over a thread pool"}
    errs = {mixed: fp.error_report(img, r64, k=64) for mixed, img in imgs.items()}
    return cpu, errs


def measure_modes(a, local):
    """The other configurations of the metric, device-timed at N=1: the NDSU-shaped float frame
    (8167x8192 -> 8192^2; FP32 lerp as form_image_pfa, FP32 32-tap sinc, and both in the split-precision
    tensor-core FFT mode), each with its errors against the FP64 oracle image (relative L2 of the complex
    and detected image, phase RMS, peak position / power and ISLR of the 64 strongest point responses)
    and a CPU baseline, the image-entropy autofocus gradient on the 4096^2 scene (grads/s) and the
    16-scene batch."""
    import numpy as np
    import torch
    from pfa_b200 import autofocus, engine, geometry, synth
    steps = max(3, min(a.steps, 10))
    out = {}
    # the small float scene (1024x1024, 64 targets, 20 dB SNR): lerp as form_image_pfa and the float sinc,
    # inputs (8 MB) L2 resident, with the CPU restatement of form_image_pfa timed beside it
    sc1 = synth.workload_scene("small_1024")
    tb1 = geometry.prepare_tables_from_scene(sc1)
    sig1 = torch.from_numpy(np.ascontiguousarray(sc1.signal, np.complex64)).to(f"cuda:{local}")
    small = {"workload": "small_1024: 1024x1024 c64 -> 1024^2, 64 targets, 20 dB SNR (inputs L2 resident)"}
    for nm, rs in (("lerp", False), ("sinc", True)):
        with engine.FloatPlan(1024, 1024, rs, rs, device=local) as plan:
            plan.set_tables(tb1)
            img = torch.empty((1024, 1024), dtype=torch.float32, device=sig1.device)
            small[f"ms_per_frame_{nm}"] = round(_device_ms(lambda: plan.form(sig1, out=img), 20, 5), 4)
    if not a.no_cpu_baseline:
        small["cpu_baseline"] = cpu_float_small(sc1, tb1)
    out["small_1024"] = small
    del sig1
    sc, sig = synth.make_scene_device(8167, 8192, device=f"cuda:{local}", **{k: v for k, v in synth.WORKLOADS["ndsu_8167x8192"].items() if k not in ("m", "n")})
    tables = geometry.prepare_tables_from_scene(sc)
    sig_np = sig.cpu().numpy() if not a.no_cpu_baseline else None
    for interp, rs in (("lerp", False), ("sinc", True)):
        imgs = {}
        for mixed in (False, True):
            name = f"float_{'mixed' if mixed else 'fp32'}_{interp}"
            with engine.FloatPlan(8167, 8192, rs, rs, mixed=mixed, device=local) as plan:
                plan.set_tables(tables)
                img = torch.empty((8192, 8192), dtype=torch.float32, device=sig.device)
                ms = _device_ms(lambda: plan.form(sig, out=img), steps, 3)
                plan.set_profiling(True)
                plan.form(sig, out=img)
                st = plan.stage_times()
                plan.set_profiling(False)
                cz = plan.form(sig, detect="complex")
            fb = sum(stage_bytes(s_, 8167, 8192, 8192, "float") for s_ in st)
            out[name] = {"workload": "ndsu_8167x8192 -> 8192^2", "ms_per_frame": round(ms, 4),
                         "stages_ms": {k: round(v, 4) for k, v in st.items()},
                         "frame_bytes": fb, "frame_frac_of_hbm": round(fb / (ms * 1e-3) / 1e9 / _peaks()[0], 4)}
            if name == "float_fp32_lerp":
                out[name]["e2e_ms_per_frame"], out[name]["e2e_bytes_per_frame"] = _float_e2e(sig, tables, local)
            if mixed:
                r, ms32 = imgs[False]
                out[name]["rel_l2_vs_fp32_complex"] = float(torch.linalg.vector_norm(cz - r) / torch.linalg.vector_norm(r))
                out[name]["speed_vs_fp32"] = round(ms32 / ms, 3)
            imgs[mixed] = (cz, ms)
        if not a.no_cpu_baseline:
            # the cpu_baseline leg: the oracle's restatement of form_image_pfa over the whole frame on the
            # host, timed; its FP64 image is also the checker of both device images' errors
            host = {k: v[0].cpu().numpy() for k, v in imgs.items()}
            imgs.clear()
            cpu, errs = float_cpu_leg(sig_np, tables, interp, host)
            for mixed, e in errs.items():
                nm = f"float_{'mixed' if mixed else 'fp32'}_{interp}"
                out[nm]["vs_fp64"] = e
                out[nm]["cpu_baseline"] = cpu
            del host
        imgs.clear()
    del sig
    wl = synth.WORKLOADS["autofocus_4096"]
    sc, sig = synth.make_scene_device(4096, 4096, device=f"cuda:{local}", **{k: v for k, v in wl.items() if k not in ("m", "n")})
    phi = torch.as_tensor(synth.phase_error(4096, seed=4), device=sig.device)
    sig = (sig * torch.polar(torch.ones_like(phi), phi)[:, None].to(torch.complex64)).contiguous()
    tables = geometry.prepare_tables_from_scene(sc)
    with engine.FloatPlan(4096, 4096, device=local) as plan:
        plan.set_tables(tables)
        theta = torch.zeros(4096, dtype=torch.float32, device=sig.device)
        dth = torch.empty_like(theta)
        ent = torch.empty((), dtype=torch.float64, device=sig.device)
        ms = _device_ms(lambda: autofocus.entropy_grad(plan, sig, theta, dth, ent), steps, 3)
        plan.set_profiling(True)
        autofocus.entropy_grad(plan, sig, theta, dth, ent)
        st = plan.stage_times()
        plan.set_profiling(False)
        th50, hist = autofocus.autofocus(plan, sig, steps=50, step=0.3, history=True)
        # focus quality: the entropy of the image with the injected error removed exactly (theta = phi)
        # and the residual phase error after 50 steps, without the constant and linear terms (a constant
        # phase leaves the image unchanged, a linear one only shifts it)
        e_true, _ = autofocus.entropy_grad(plan, sig, phi.float())
        res = (th50.double() - phi).cpu().numpy()
        u = np.arange(4096, dtype=np.float64)
        res = res - np.polyval(np.polyfit(u, res, 1), u)
        res0 = phi.cpu().numpy() - np.polyval(np.polyfit(u, phi.cpu().numpy(), 1), u)
    out["autofocus_4096"] = {"workload": "4096x4096 c64, 128 targets + clutter, quadratic 3 rad + random walk "
                                         "0.05 rad/pulse phase error; entropy gradient w.r.t. 4096 phases",
                             "ms_per_grad": round(ms, 4), "grads_per_s": round(1000.0 / ms, 1),
                             "stages_ms": {k: round(v, 4) for k, v in st.items()},
                             "entropy_first_last_of_50_steps": [round(hist[0], 5), round(hist[-1], 5)],
                             "entropy_true_phase": round(float(e_true), 5),
                             "phase_rms_rad_before_after_50_steps": [round(float(np.sqrt(np.mean(res0 ** 2))), 4),
                                                                     round(float(np.sqrt(np.mean(res ** 2))), 4)]}
    # the same gradient through the float 32-tap sinc passes (transposed sinc resample in the adjoint)
    with engine.FloatPlan(4096, 4096, True, True, device=local) as plan:
        plan.set_tables(tables)
        theta = torch.zeros(4096, dtype=torch.float32, device=sig.device)
        ms_s = _device_ms(lambda: autofocus.entropy_grad(plan, sig, theta, dth, ent), steps, 3)
        plan.set_profiling(True)
        autofocus.entropy_grad(plan, sig, theta, dth, ent)
        st_s = plan.stage_times()
        plan.set_profiling(False)
    out["autofocus_4096"]["sinc"] = {"ms_per_grad": round(ms_s, 4), "grads_per_s": round(1000.0 / ms_s, 1),
                                     "stages_ms": {k: round(v, 4) for k, v in st_s.items()}}
    del sig
    out["batch_16_uneven"] = measure_batch(a, local)
    return out


def measure_batch(a, local, nscene=16, af_iters=5, streams=4):
    """16 scenes with pulses and samples uniform in [2048, 8192] (seed 5), 64-512 targets + clutter, each
    formed on its own pow2 raster after `af_iters` autofocus steps on the device (pfa_autofocus_step; the
    image applies the phase in pass 1), autotuned FFT tiles; one CUDA graph launch for the batch vs one
    scene at a time on one stream.  Aggregate frames/s."""
    import numpy as np
    import torch
    from pfa_b200 import autotune, batch, geometry, synth
    rng = np.random.default_rng(5)
    scenes, tiles = [], []
    for k in range(nscene):
        m, n = (int(v) for v in rng.integers(2048, 8193, 2))
        sc, x = synth.make_scene_device(m, n, device=f"cuda:{local}", n_targets=int(rng.integers(64, 513)),
                                        clutter_db=-10.0, snr_db=20.0, seed=500 + k)
        tb = geometry.prepare_tables_from_scene(sc)
        tile, _ = autotune.tune_float(tb, x, reps=3)
        scenes.append((tb, x))
        tiles.append(tile)
    reps = max(2, min(a.steps, 5))
    shapes = [list(map(int, s.shape)) for _, s in scenes]
    out = {"workload": f"{nscene} scenes, M,N uniform in [2048, 8192] (seed 5), 64-512 targets + clutter, "
                       f"pow2 rasters, {af_iters} autofocus iterations each on the device (FP32 gradients)",
           "shapes": shapes, "tiles": [list(t) for t in tiles], "streams": streams}
    for tag, mixed in (("fp32", False), ("mixed", True)):
        bf = batch.BatchFormer(scenes, streams=streams, tiles=tiles, af_iters=af_iters, device=local, mixed=mixed)
        bf.capture()
        eager_ms = _device_ms(bf.run_eager, reps, 1)
        graph_ms = _device_ms(bf.replay, reps, 1)
        bf.close()
        out[tag] = {"images": "FP32 FFTs" if not mixed else "split-precision tensor-core FFTs (2048..8192-point lines)",
                    "graph_ms_per_batch": round(graph_ms, 3), "eager_ms_per_batch": round(eager_ms, 3),
                    "frames_per_s_graph": round(nscene * 1000.0 / graph_ms, 1),
                    "frames_per_s_one_at_a_time": round(nscene * 1000.0 / eager_ms, 1),
                    "speedup": round(eager_ms / graph_ms, 3)}
    return out


def run_ours(a, ws, rank, local):
    import numpy as np
    import torch
    from pfa_b200 import engine, geometry, synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    wl = WORKLOADS[a.workload]
    mode = wl["mode"]
    sc = synth.workload_scene(wl["scene"])
    m, n = sc.signal.shape
    tables = geometry.prepare_tables_from_scene(sc)
    sig_host = torch.from_numpy(sc.signal).pin_memory()
    sig = sig_host.to(dev)
    if mode == "fixed":
        G = wl["grid"]
        plan = engine.FixedPlan(m, n, G, wl["range_sinc"], wl["az_sinc"], device=local)
        img = torch.empty((G, G), dtype=torch.uint16, device=dev)
        out_bytes = G * G * 2
        launches_per_frame = 6
    else:
        G = geometry.pow2(max(m, n))
        plan = engine.FloatPlan(m, n, wl["range_sinc"], wl["az_sinc"], wl.get("mixed", False), device=local)
        img = torch.empty((plan.m2, plan.n2), dtype=torch.float32, device=dev)
        out_bytes = plan.m2 * plan.n2 * 4
        launches_per_frame = 3
    plan.set_tables(tables)
    stream = torch.cuda.current_stream()

    from pfa_b200 import replicas
    barrier = replicas.barrier
    max_over_ranks = replicas.max_over_ranks

    for _ in range(a.warmup):
        plan.form(sig, out=img)
    torch.cuda.synchronize()
    # ---- timed region: device-resident inputs
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(a.steps):
            plan.form(sig, out=img)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    dev_ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_per_frame = dev_ms / (a.steps * ws)
    clocks = clk.summary()

    # ---- per-stage device times (CUDA events between the library's kernels, same stream)
    plan.set_profiling(True)
    acc = {}
    for _ in range(max(3, min(a.steps, 10))):
        plan.form(sig, out=img)
        for k, v in plan.stage_times().items():
            acc.setdefault(k, []).append(v)
    plan.set_profiling(False)
    stages = {k: statistics.mean(v) for k, v in acc.items()}
    top = max(stages, key=stages.get)
    hbm, peak_kind = _peaks()
    ach = stage_bytes(top, m, n, G, mode) / (stages[top] * 1e-3) / 1e9
    kname = ({"pass1": "k_fx_pass1", "pass2_win_fft1": "k_fx_pass2_fft", "fft2": "k_fx_fft2",
              "renorm_detect": "k_fx_detect", "q0max": "k_q0max"} if mode == "fixed" else
             {"pass1": "k_fl_pass1", "pass2_win_fft1": "k_fl_pass2_fft", "fft2_detect": "k_fl_fft2"})[top]
    traffic = _traffic(kname, a.workload)
    frame_bytes = sum(stage_bytes(s, m, n, G, mode) for s in stages)

    # ---- end to end through the host-buffer C-ABI entry points (pinned host in/out).  The headline
    # e2e is the pipelined one (pfa_form_*_host_frames: uploads, frames and downloads of consecutive
    # frames overlap on three streams); the single-frame entry point (copy in, form, copy out, sync)
    # is reported beside it.
    outs_host = [torch.empty(tuple(img.shape), dtype=img.dtype).pin_memory() for _ in range(2)]
    sig_np = sig_host.numpy()
    outs_np = [o.numpy() for o in outs_host]
    ne2e = max(4, min(a.steps, 16))
    frames_in = [sig_np] * ne2e
    frames_out = [outs_np[k & 1] for k in range(ne2e)]
    for _ in range(2):
        plan.form_host(sig_np, outs_np[0])
    plan.form_host_frames(frames_in[:2], frames_out[:2])
    barrier()
    t0 = time.perf_counter()
    plan.form_host_frames(frames_in, frames_out)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0) / (ne2e * ws)
    barrier()
    t0 = time.perf_counter()
    for _ in range(ne2e):
        plan.form_host(sig_np, outs_np[0])
    e2e_single_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0) / (ne2e * ws)
    # a new geometry every frame, as in the reference's scene loop: O(m + n) table preparation from the
    # per-vector parameters, job upload, then the frame through the host-buffer entry point; serially,
    # and as the engine's scene queue (next scene's tables on a host thread during the current frame)
    barrier()
    t0 = time.perf_counter()
    for _ in range(ne2e):
        plan.set_tables(geometry.prepare_tables_from_scene_fast(sc))
        plan.form_host(sig_np, outs_np[0])
    e2e_geom_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0) / (ne2e * ws)
    barrier()
    t0 = time.perf_counter()
    engine.form_host_scenes(plan, [sc] * ne2e, lambda s: (geometry.prepare_tables_from_scene_fast(s), sig_np),
                            outs=outs_np[:1])
    e2e_queue_ms = max_over_ranks((time.perf_counter() - t0) * 1000.0) / (ne2e * ws)

    # ---- CPU baseline: the oracle port on a bounded sample, rank 0 at N=1
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        from oracle import cpu_sample
        if mode == "fixed":
            # the C restatement of the emulator's datapath, one whole frame on one core
            t0 = time.perf_counter()
            ref_img, _ = cpu_sample.c_fixed_frame(sc.signal, tables, G, wl["range_sinc"], wl["az_sinc"], threads=1)
            cpu = {"value": round((time.perf_counter() - t0) * 1000.0, 1), "unit": "ms/frame", "cores": 1,
                   "kind": "port", "sample": "one whole frame of the C restatement of the emulator datapath "
                                             "(oracle/fixed_frame.c), 1 thread",
                   "image_equal_to_gpu": bool(np.array_equal(ref_img, img.cpu().numpy()))}
        else:
            est = cpu_sample.float_frame_estimate(sc.signal, tables, sample=a.cpu_sample, workers=1)
            cpu = {"value": round(est["ms_per_frame"], 1), "unit": "ms/frame", "cores": 1, "kind": "port",
                   "sample": est["sample"], "stage_seconds": est["stage_seconds"]}

    line = {
        "metric": METRIC, "value": round(ms_per_frame, 4), "unit": "ms/frame", "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(dev_ms / a.steps, 4),
        "higher_is_better": False, "scaling": "weak",
        "vs_baseline": round(ms_per_frame / FPGA_FRAME_MS[a.workload], 8) if a.workload in FPGA_FRAME_MS else None,
        "dtype": ("int16 fixed point (int32/int64 accumulate; fp64 coordinates)" if mode == "fixed"
                  else "fp32 (fp64 coordinates)"), "data": "synthetic",
        "config": {"workload": a.workload, "desc": wl["desc"], "m": m, "n": n, "grid": G,
                   "parallelism": f"replicas x{ws}",
                   "l2": f"inputs larger than L2 ({sc.signal.nbytes / 1e6:.0f} MB signal, "
                         f"{G * G * 4 / 1e6:.0f}+ MB intermediates); no flush",
                   "frames_per_s": round(1000.0 / ms_per_frame, 2)},
        "stages_ms": {k: round(v, 4) for k, v in stages.items()},
        "roofline": {"kernel": kname, "stage": top, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                     "unit": "GB/s", "frac": round(ach / hbm, 4), "peak_kind": f"of {peak_kind}",
                     "traffic": traffic, "algorithmic_bytes": stage_bytes(top, m, n, G, mode),
                     "frame_bytes": frame_bytes,
                     "frame_frac": round(frame_bytes / (ms_per_frame * 1e-3) / 1e9 / hbm, 4),
                     # what bounds it instead: pipe utilisation of the same kernel from the ncu summary
                     "compute": {"pipe": "integer ALU" if mode == "fixed" else "FP32/LSU",
                                 "alu_pipe_active_pct": _profile_value(kname, a.workload, "alu_pipe_active_pct"),
                                 "issue_active_pct": _profile_value(kname, a.workload, "issue_active_pct")}},
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/frame", "h2d_bytes_per_step": int(sc.signal.nbytes),
                "d2h_bytes_per_step": int(out_bytes), "frames": ne2e, "api": "pfa_form_*_host_frames (pipelined)",
                "single_frame_ms": round(e2e_single_ms, 4),
                "per_scene_geometry_ms": round(e2e_geom_ms, 4),
                "per_scene_geometry_queued_ms": round(e2e_queue_ms, 4)},
        "gpu_launches": launches_per_frame * a.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    plan.close()
    if ws == 1 and not a.no_modes:
        line["modes"] = measure_modes(a, local)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(a, ws, rank):
    """The reference arm: the CPU restatement of the reference's path on every host core, rank 0 only.

    Fixed workload: every step (warm-up and timed) forms one WHOLE frame with the C restatement of the
    emulator's datapath (oracle/fixed_frame.c, OpenMP over all host threads); the first frame's CRC is
    checked against the unmodified reference emulator's CRC of the same frame.  Float workloads: the
    sampled estimate of form_image_pfa's restatement (spawned workers)."""
    if rank != 0:
        return
    import numpy as np
    from pfa_b200 import geometry, synth
    from oracle import cpu_sample
    from oracle import fixed_emulator as fe
    wl = WORKLOADS[a.workload]
    sc = synth.workload_scene(wl["scene"])
    m, n = sc.signal.shape
    G = wl.get("grid", geometry.pow2(max(m, n)))
    tables = geometry.prepare_tables_from_scene(sc)
    cores = cpu_sample.available_cores()
    per = []
    extra = {}
    if wl["mode"] == "fixed":
        for i in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            img, _ = cpu_sample.c_fixed_frame(sc.signal, tables, G, wl["range_sinc"], wl["az_sinc"], threads=cores)
            dt = (time.perf_counter() - t0) * 1000.0
            if i == 0 and "ref_crc" in wl:
                crc = fe.frame_crc(img)
                extra["image_crc"] = f"0x{crc:08x}"
                extra["crc_equals_reference_emulator"] = crc == wl["ref_crc"]
            if i >= a.warmup:
                per.append(dt)
        sample = (f"whole frame per step: C restatement of the emulator datapath (oracle/fixed_frame.c), "
                  f"OpenMP, {cores} threads")
        dtype = "int16 fixed point (int32/int64 C)"
        if "ref_emulator_s" in wl:
            extra["context"] = {"reference_emulator_whole_frame_ms_1_core": wl["ref_emulator_s"] * 1000.0,
                                "note": "the unmodified NumPy emulator, measured once on this frame"}
    else:
        pool = cpu_sample.make_pool(cores) if cores > 1 else None
        try:
            for i in range(a.warmup + a.steps):
                est = cpu_sample.float_frame_estimate(sc.signal, tables, sample=a.ref_sample, workers=cores,
                                                      seed=i, pool=pool)
                if i >= a.warmup:
                    per.append(est["ms_per_frame"])
        finally:
            if pool is not None:
                pool.shutdown()
        sample = est["sample"] + f"; {cores} spawned worker processes"
        dtype = "complex64/float64 numpy"
    v = statistics.mean(per)
    line = {
        "metric": METRIC, "value": round(v, 1), "unit": "ms/frame", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(v, 1), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": round(v / FPGA_FRAME_MS[a.workload], 6) if a.workload in FPGA_FRAME_MS else None,
        "dtype": dtype, "data": "synthetic", "impl": "reference",
        "config": {"workload": a.workload, "desc": wl["desc"], "m": m, "n": n, "grid": G},
        "cpu_baseline": {"value": round(v, 1), "unit": "ms/frame", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": round(v, 1), "unit": "ms/frame", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line.update(extra)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="centerfield_5634x4319", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=512)
    ap.add_argument("--ref-sample", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-modes", action="store_true", help="skip the float and autofocus configurations")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    ws, rank, local = _dist()
    if a.impl == "reference":
        run_reference(a, ws, rank)
    else:
        run_ours(a, ws, rank, local)


if __name__ == "__main__":
    main()
