"""Form PFA frames from the command line (the counterpart of the reference's drivers
``silicon_emulator.py --grid --range-sinc --az-sinc`` and ``form_image_pfa.py``).

    PYTHONPATH=mpfs250t-sar-ifp_b200 python -m pfa_b200.cli --mode fixed --m 5634 --n 4319 --grid 8192 \\
        --range-sinc --az-sinc --frames 3

The input is a seeded synthetic scene of the given shape (or ``--input`` a complex64 .npy phase history
with ``--tables`` an .npz of ``prepare_tables`` output).  Prints the device time of every frame; ``--out``
saves the last image.  Modes: ``fixed`` (bit-exact emulator datapath), ``float`` (FP32), ``mixed``
(split-precision tensor-core FFTs) and ``autofocus`` (the image-entropy gradient w.r.t. the per-pulse
phase of a scene with the injected quadratic + random-walk phase error; one gradient per frame, through
the float-sinc passes with ``--range-sinc`` / ``--az-sinc``).
``--display`` adds the device display scaling of save_detected_geotiff to each float frame.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--mode", choices=("fixed", "float", "mixed", "autofocus"), default="float")
    ap.add_argument("--m", type=int, default=2048, help="pulses")
    ap.add_argument("--n", type=int, default=2048, help="samples per pulse")
    ap.add_argument("--grid", type=int, default=0, help="fixed mode: square output raster (default pow2)")
    ap.add_argument("--range-sinc", action="store_true")
    ap.add_argument("--az-sinc", action="store_true")
    ap.add_argument("--detect", choices=("mag", "power", "complex"), default="mag")
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--targets", type=int, default=64)
    ap.add_argument("--input", help="complex64 .npy phase history (m, n)")
    ap.add_argument("--tables", help=".npz of prepare_tables output (with --input)")
    ap.add_argument("--out", help="save the last image (.npy)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--display", action="store_true",
                    help="float/mixed: also scale each |img| to the uint8 display image on the device")
    a = ap.parse_args(argv)

    import torch

    from . import engine, geometry, synth

    dev = torch.device("cuda", a.device)
    if a.input:
        sig = torch.from_numpy(np.ascontiguousarray(np.load(a.input), np.complex64)).to(dev)
        tb = dict(np.load(a.tables))
        tb["sgn"] = int(tb.get("sgn", -1))
    else:
        sc, sig = synth.make_scene_device(a.m, a.n, device=str(dev), n_targets=a.targets, clutter_db=-10.0,
                                          snr_db=15.0, seed=a.seed)
        tb = geometry.prepare_tables_from_scene(sc)
    m, n = sig.shape
    if a.mode == "autofocus":
        from . import autofocus
        phi = torch.as_tensor(synth.phase_error(m, seed=a.seed), device=dev)
        sig = (sig * torch.polar(torch.ones_like(phi), phi)[:, None].to(torch.complex64)).contiguous()
        theta = torch.zeros(m, dtype=torch.float32, device=dev)
        with engine.FloatPlan(m, n, a.range_sinc, a.az_sinc, device=a.device) as plan:
            plan.set_tables(tb)
            for k in range(a.frames):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                ent, dth = autofocus.entropy_grad(plan, sig, theta)
                e1.record()
                torch.cuda.synchronize()
                print(f"gradient {k}: {e0.elapsed_time(e1):.3f} ms  (entropy {float(ent):.5f}, {m}x{n}"
                      f"{', sinc' if a.range_sinc or a.az_sinc else ''})")
        return 0
    if a.mode == "fixed":
        grid = a.grid or geometry.pow2(max(m, n))
        plan = engine.FixedPlan(m, n, grid, a.range_sinc, a.az_sinc, device=a.device)
        form = lambda: plan.form(sig)                                            # noqa: E731
    else:
        plan = engine.FloatPlan(m, n, a.range_sinc, a.az_sinc, mixed=a.mode == "mixed", device=a.device)
        form = lambda: plan.form(sig, detect=a.detect)                           # noqa: E731
    with plan:
        plan.set_tables(tb)
        img = None
        for k in range(a.frames):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            img = form()
            e1.record()
            torch.cuda.synchronize()
            msg = f"frame {k}: {e0.elapsed_time(e1):.3f} ms  ({a.mode}, {m}x{n} -> {tuple(img.shape)})"
            if a.display and a.mode != "fixed" and a.detect == "mag":
                from . import geocode
                e0.record()
                disp, hi = geocode.display_u8(img)
                e1.record()
                torch.cuda.synchronize()
                msg += f"; display {e0.elapsed_time(e1):.3f} ms (hi {float(hi):.6g})"
            print(msg)
        if a.out:
            np.save(a.out, img.cpu().numpy())
    return 0


if __name__ == "__main__":
    sys.exit(main())
