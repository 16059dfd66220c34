"""Generate the golden fixtures in this folder by running the UNMODIFIED reference.

Run where the reference checkout exists (a ``reference`` checkout beside this repository, or PFA_REFERENCE_ROOT):

    python tests/golden/make_golden.py            # small fixed/float cases + FFT KAT digests
    python tests/golden/make_golden.py --big      # also the 5634x4319 -> 8192^2 sinc/sinc frame

Outputs (JSON, a few KB):
  fixed_frames.json  per case: scene parameters, CRC-32 of the complex64 input bytes, CRC-32 of the
                     reference emulator's uint16 image (``silicon_emulator.form_image``), exponent
                     spreads.  A test first regenerates the input and checks its CRC, so the output
                     golden only applies to a bit-identical input.
  float_frames.json  per case: input CRC and the reference ``pfa()`` image digest (|img| at the 8
                     strongest pixels, total energy).
  fft_kat.json       CRC-32 of the reference's CoreFFT BFP golden vectors (mpfs/host/corefft_vectors,
                     model ``fixedpoint.fft1d_bfp``, 16-bit data, 18-bit twiddles) per stimulus, plus
                     the manifest's exponents; the oracle's restated BFP FFT is pinned against them.
  variants.json      CRC-32 of gen_resample_vectors.lagrange_taps_q15 over every Q15 weight, of
                     gen_resample_vectors.gather_cubic and of model_detect_fusion.order_B_fused on
                     seeded operands (``variant_inputs``): the cubic interpolator and the
                     silicon-order detect the engine offers as variants.
  big_frames.json    (--big) the Centerfield-shaped full frame and a tiny scene on the largest grid
                     (16384^2, about 15 minutes of the reference emulator).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "mpfs250t-sar-ifp_b200"))

from oracle import refshim                     # noqa: E402
from pfa_b200 import synth                     # noqa: E402

# (name, scene kwargs, grid, range_sinc, az_sinc)
FIXED_CASES = [
    ("sq256_sinc", dict(m=256, n=256, n_targets=16, scene_half=40.0, snr_db=20.0, seed=11), 256, True, True),
    ("sq256_lerp", dict(m=256, n=256, n_targets=16, scene_half=40.0, snr_db=20.0, seed=12, jitter=0.5), 256, False, False),
    ("r200x180_mixed", dict(m=200, n=180, n_targets=8, snr_db=20.0, seed=13, jitter=0.3), 256, True, False),
    ("r180x200_mixed", dict(m=180, n=200, n_targets=8, snr_db=20.0, seed=14), 256, False, True),
    ("sq1024_sinc", dict(m=1024, n=1024, n_targets=32, clutter_db=-10.0, snr_db=20.0, seed=15), 1024, True, True),
    ("r1000x700_lerp", dict(m=1000, n=700, n_targets=32, clutter_db=-10.0, snr_db=20.0, seed=16, jitter=0.5), 1024, False, False),
    ("r700x1000_sinc_g2048", dict(m=700, n=1000, n_targets=32, snr_db=20.0, seed=17, jitter=0.2), 2048, True, True),
    ("tiny33x40", dict(m=33, n=40, n_targets=4, snr_db=20.0, seed=18), 64, True, True),
    ("tiny17x20", dict(m=17, n=20, n_targets=4, snr_db=20.0, seed=19), 32, False, True),
]

FLOAT_CASES = [
    ("small_1024", dict(m=1024, n=1024, n_targets=64, scene_half=100.0, snr_db=20.0, seed=1)),
    ("r600x900", dict(m=600, n=900, n_targets=32, clutter_db=-10.0, snr_db=20.0, seed=21, jitter=0.3)),
]

BIG_CASES = [
    ("centerfield_5634x4319_sinc", "centerfield_5634x4319", 8192, True, True),
]

# the largest grid the engine accepts (16384^2), on a tiny scene so the reference emulator finishes
MAX_GRID_CASES = [
    ("tiny40x48_g16384_sinc", dict(m=40, n=48, n_targets=4, snr_db=20.0, seed=23), 16384, True, True),
]


def crc(a: np.ndarray) -> int:
    return zlib.crc32(np.ascontiguousarray(a).tobytes()) & 0xFFFFFFFF


def fixed_cases():
    out = {}
    for name, kw, grid, rs, az in FIXED_CASES:
        sc = synth.make_scene(**kw)
        t = time.time()
        img = refshim.emulator_form_image(sc, grid, rs, az)
        out[name] = dict(scene=kw, grid=grid, range_sinc=rs, az_sinc=az,
                         input_crc=crc(sc.signal), image_crc=crc(img.astype("<u2")),
                         image_max=int(img.max()), seconds=round(time.time() - t, 2))
        print(name, hex(out[name]["image_crc"]), out[name]["seconds"], "s", flush=True)
    return out


def float_cases():
    m = refshim.modules()
    out = {}
    for name, kw in FLOAT_CASES:
        sc = synth.make_scene(**kw)
        tb = refshim.reference_tables(sc)
        img, _ = m.ref.pfa(sc.signal, tb["freq"], tb["ax"], tb["ay"], tb["sgn"])
        det = np.abs(img).astype(np.float32)
        top = np.argsort(det.ravel())[::-1][:8]
        out[name] = dict(scene=kw, input_crc=crc(sc.signal), shape=list(det.shape),
                         top_index=[int(i) for i in top], top_value=[float(det.ravel()[i]) for i in top],
                         energy=float((det.astype(np.float64) ** 2).sum()),
                         detect_crc=crc(det))
        print(name, out[name]["top_index"][:3], flush=True)
    return out


def fft_kat():
    vec = refshim.REF_ROOT / "mpfs" / "host" / "corefft_vectors"
    man = json.loads((vec / "manifest.json").read_text())
    out = {"n": man["n"], "nbits": man["nbits"], "nbits_tw": man["nbits_tw"], "cases": {}}
    for name, c in man["cases"].items():
        codes = {}
        for kind in ("in", "out"):
            rows = [ln.split(",") for ln in (vec / f"{name}_{kind}.csv").read_text().splitlines()
                    if ln and not ln.startswith("#")]
            arr = np.asarray(rows, np.int64)
            codes[kind] = crc(arr.astype("<i2"))
        out["cases"][name] = dict(in_crc=codes["in"], out_crc=codes["out"], e_in=c["e_in"],
                                  e_out=c["e_out"], stage_exps=c["stage_exps"])
    return out


def variant_inputs():
    """Seeded operands of the variant pins (regenerated identically by the tests)."""
    rng = np.random.default_rng(20261203)
    sn = 300
    src_re = rng.integers(-32768, 32768, sn)
    src_im = rng.integers(-32768, 32768, sn)
    idx = rng.integers(-3, sn - 1, 4000)
    idx = np.where(idx < 0, -1, np.minimum(idx, sn - 2))
    wq = rng.integers(0, 32768, 4000)
    y_re = rng.integers(-32768, 32768, (32, 128))
    y_im = rng.integers(-32768, 32768, (32, 128))
    e = rng.integers(0, 12, 32)
    return dict(sn=sn, src_re=src_re, src_im=src_im, idx=idx, wq=wq, y_re=y_re, y_im=y_im, e=e)


def variants():
    """The silicon A/B variants the engine also implements: gen_resample_vectors.lagrange_taps_q15 for
    every Q15 weight, gen_resample_vectors.gather_cubic and model_detect_fusion.order_B_fused."""
    m = refshim.modules()
    taps = np.asarray([m.grv.lagrange_taps_q15(w) for w in range(32768)], np.int64)
    v = variant_inputs()
    src = [((int(i) & 0xFFFF) << 16) | (int(r) & 0xFFFF) for r, i in zip(v["src_re"], v["src_im"])]
    words = m.grv.gather_cubic(src, [int(x) for x in v["idx"]], [int(x) for x in v["wq"]], v["sn"])
    fused = m.mdf.order_B_fused(v["y_re"] + 1j * v["y_im"], v["e"])
    return dict(lagrange_taps_crc=crc(taps.astype("<i4")),
                lagrange_taps_w16384=[int(t) for t in taps[16384]],
                gather_cubic_crc=crc(np.asarray(words, "<u4")),
                detect_fused_crc=crc(np.asarray(fused, "<u2")))


def big_cases():
    out = {}
    for name, wl, grid, rs, az in BIG_CASES:
        sc = synth.workload_scene(wl)
        t = time.time()
        img = refshim.emulator_form_image(sc, grid, rs, az)
        out[name] = dict(workload=wl, grid=grid, range_sinc=rs, az_sinc=az, input_crc=crc(sc.signal),
                         image_crc=crc(img.astype("<u2")), image_max=int(img.max()),
                         seconds=round(time.time() - t, 1))
        print(name, hex(out[name]["image_crc"]), out[name]["seconds"], "s", flush=True)
    return out


def max_grid_cases():
    out = {}
    for name, kw, grid, rs, az in MAX_GRID_CASES:
        sc = synth.make_scene(**kw)
        t = time.time()
        img = refshim.emulator_form_image(sc, grid, rs, az)
        out[name] = dict(scene=kw, grid=grid, range_sinc=rs, az_sinc=az, input_crc=crc(sc.signal),
                         image_crc=crc(img.astype("<u2")), image_max=int(img.max()),
                         seconds=round(time.time() - t, 1))
        print(name, hex(out[name]["image_crc"]), out[name]["seconds"], "s", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--only-big", action="store_true")
    a = ap.parse_args()
    env = dict(numpy=np.__version__)
    if not a.only_big:
        (HERE / "fixed_frames.json").write_text(json.dumps(dict(env=env, cases=fixed_cases()), indent=1))
        (HERE / "float_frames.json").write_text(json.dumps(dict(env=env, cases=float_cases()), indent=1))
        (HERE / "fft_kat.json").write_text(json.dumps(fft_kat(), indent=1))
        (HERE / "variants.json").write_text(json.dumps(variants(), indent=1))
    if a.big or a.only_big:
        cases = big_cases()
        cases.update(max_grid_cases())
        (HERE / "big_frames.json").write_text(json.dumps(dict(env=env, cases=cases), indent=1))


if __name__ == "__main__":
    main()
