"""Seeded synthetic spotlight phase history (FX domain) standing in for the Umbra CPHD scenes.

The reference focuses Umbra CPHD collects (Centerfield 5634x4319, NDSU 8167x8999, ship), which are not
available here.  This module builds phase history with the same shapes and the same per-vector
parameters (PVP) the reference reads through sarpy (``TxPos``, ``RcvPos``, ``SRPPos``, ``SC0``,
``SCSS``; ``src/form_image_pfa.py:323-327``, ``mpfs/host/sar_pipeline.py:62-66``):

* SRP at the origin, monostatic APC_i = R (cos th_i, sin th_i, h/R), th_i uniform over +/- half the
  aperture (optionally jittered so the tan(phi) sort is a non-trivial permutation);
* SC0 = fc - BW/2, SCSS = BW/N, image plane uIAX=(1,0,0), uIAY=(0,1,0), SGN=-1;
* signal s[i,k] = sum_p a_p exp(+j 4 pi f_ik/c (u_i . r_p)) + clutter + noise, where u_i is the
  in-plane unit look vector (ax_i, ay_i) that ``prepare_tables`` derives from the PVP.  With SGN=-1
  (forward FFT) each point focuses at its own (range, cross) position.
* the clutter field is homogeneous with Rayleigh amplitude and uniform phase; its phase history is
  complex white Gaussian over the support, so it is drawn directly in that domain at the stated level
  below the point-target power.  White complex noise is added at the stated SNR.

The point-target sum is evaluated as a blocked geometric series
``s[i, 64q+r] = sum_p (a_p z_ip^(64q) w_ip) z_ip^r`` (one small complex matmul per pulse block), which
keeps the 5634x4319x256 case to seconds on the host.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C = 299_792_458.0


@dataclass
class Scene:
    """Synthetic collect: PVP arrays plus the complex64 (M, N) phase history."""
    signal: np.ndarray            # (M, N) complex64
    tx: np.ndarray                # (M, 3) float64
    rcv: np.ndarray               # (M, 3)
    srp: np.ndarray               # (M, 3)
    sc0: np.ndarray               # (M,)
    scss: np.ndarray              # (M,)
    uiax: np.ndarray = field(default_factory=lambda: np.array([1.0, 0.0, 0.0]))
    uiay: np.ndarray = field(default_factory=lambda: np.array([0.0, 1.0, 0.0]))
    sgn: int = -1
    targets: np.ndarray | None = None    # (P, 2) x, y metres
    amps: np.ndarray | None = None       # (P,) complex
    mn: tuple | None = None              # (M, N), also when the signal lives elsewhere

    @property
    def dims(self):
        return self.mn if self.mn is not None else self.signal.shape


def _look_vectors(apc, srp, uiax, uiay):
    los = srp - apc
    u = los / np.linalg.norm(los, axis=1, keepdims=True)
    return u @ uiax, u @ uiay


def make_scene(m: int, n: int, *, fc: float = 9.6e9, bw: float = 600e6, aperture_deg: float = 3.0,
               n_targets: int = 64, scene_half: float | None = None, clutter_db: float | None = None,
               snr_db: float | None = 20.0, seed: int = 0, jitter: float = 0.0,
               range_m: float = 10_000.0, height_m: float = 3_000.0,
               with_signal: bool = True) -> Scene:
    """Build a seeded scene.

    ``scene_half``: half-width of the square the point targets are drawn in (metres); default is 40 %
    of the smaller unambiguous extent so every target lands inside the formed image.
    ``clutter_db``: clutter power relative to the total point-target power (None = no clutter).
    ``jitter``: fraction of the angular pulse spacing by which pulse angles are randomly displaced
    (non-zero values make ``argsort(tan_phi)`` a non-trivial permutation).
    """
    rng = np.random.default_rng(seed)
    half = math.radians(aperture_deg) / 2.0
    th = np.linspace(-half, half, m)
    if jitter:
        dth = (2 * half) / max(m - 1, 1)
        th = th + rng.uniform(-jitter, jitter, m) * dth
    apc = np.stack([range_m * np.cos(th), range_m * np.sin(th), np.full(m, height_m)], axis=1)
    srp = np.zeros((m, 3))
    sc0 = np.full(m, fc - bw / 2.0)
    scss = np.full(m, bw / n)
    uiax = np.array([1.0, 0.0, 0.0])
    uiay = np.array([0.0, 1.0, 0.0])
    ax, ay = _look_vectors(apc, srp, uiax, uiay)

    if scene_half is None:
        rng_ext = (n - 1) * C / (2.0 * bw)                     # image extent along range (m)
        cr_ext = (m - 1) * (C / fc) / (2.0 * (2 * half))        # image extent along cross (m)
        scene_half = 0.35 * min(rng_ext, cr_ext)
    tgt = rng.uniform(-scene_half, scene_half, (n_targets, 2))
    amp = (rng.standard_normal(n_targets) + 1j * rng.standard_normal(n_targets)) / math.sqrt(2.0)

    sig = None
    if with_signal:
        sig = _point_targets(ax, ay, sc0, scss, n, tgt, amp)
        p_t = float(np.mean(np.abs(sig) ** 2)) if n_targets else 1.0
        extra = 0.0
        if clutter_db is not None:
            extra += p_t * 10.0 ** (clutter_db / 10.0)
        if snr_db is not None:
            extra += (p_t + (p_t * 10.0 ** (clutter_db / 10.0) if clutter_db is not None else 0.0)) \
                * 10.0 ** (-snr_db / 10.0)
        if extra > 0.0:
            s = math.sqrt(extra / 2.0)
            sig = sig + s * (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))
        sig = sig.astype(np.complex64)
    return Scene(signal=sig, tx=apc.copy(), rcv=apc.copy(), srp=srp, sc0=sc0, scss=scss,
                 uiax=uiax, uiay=uiay, sgn=-1, targets=tgt, amps=amp, mn=(m, n))


def make_scene_device(m: int, n: int, device="cuda", **kw) -> tuple:
    """Same scene model as ``make_scene`` (PVP from NumPy, so the tables are identical), with the
    point-target sum, clutter and noise evaluated by torch on ``device`` in float64.  For benchmark
    inputs of production size; parity fixtures use ``make_scene``.  Returns (Scene without signal,
    complex64 device tensor)."""
    import torch
    sc = make_scene(m, n, with_signal=False, **kw)
    dev = torch.device(device)
    ax, ay = _look_vectors(sc.tx, sc.srp, sc.uiax, sc.uiay)
    g = torch.Generator(device=dev).manual_seed(int(kw.get("seed", 0)) + 7919)
    tgt = torch.as_tensor(sc.targets, device=dev)
    amp = torch.as_tensor(sc.amps, device=dev)
    out = torch.empty((m, n), dtype=torch.complex64, device=dev)
    axd = torch.as_tensor(ax, device=dev)
    ayd = torch.as_tensor(ay, device=dev)
    sc0 = torch.as_tensor(sc.sc0, device=dev)
    scss = torch.as_tensor(sc.scss, device=dev)
    blk = 64
    nq = (n + blk - 1) // blk
    qq = torch.arange(nq, device=dev, dtype=torch.float64) * blk
    rr = torch.arange(blk, device=dev, dtype=torch.float64)
    npt = max(tgt.shape[0], 1)
    chunk = max(1, (1 << 27) // (npt * (nq + blk)))
    p_t = 0.0
    for i0 in range(0, m, chunk):
        i1 = min(m, i0 + chunk)
        proj = axd[i0:i1, None] * tgt[None, :, 0] + ayd[i0:i1, None] * tgt[None, :, 1]        # (b, P)
        ph0 = (4.0 * math.pi / C) * sc0[i0:i1, None] * proj
        dph = (4.0 * math.pi / C) * scss[i0:i1, None] * proj
        # s[i, 64 q + r] = sum_p (a_p e^{j(ph0 + 64 q dph)}) e^{j r dph}: one batched matmul per chunk
        pa = ph0[:, None, :] + qq[None, :, None] * dph[:, None, :]                             # (b, Q, P)
        a = (torch.polar(torch.ones_like(pa), pa) * amp[None, None, :]).to(torch.complex64)
        pb = dph[:, :, None] * rr[None, None, :]                                               # (b, P, 64)
        b = torch.polar(torch.ones_like(pb), pb).to(torch.complex64)
        s = torch.bmm(a, b).reshape(i1 - i0, nq * blk)[:, :n]
        out[i0:i1] = s
        p_t += float((s.abs().double() ** 2).sum())
    p_t /= m * n
    clutter_db, snr_db = kw.get("clutter_db"), kw.get("snr_db", 20.0)
    extra = 0.0
    if clutter_db is not None:
        extra += p_t * 10.0 ** (clutter_db / 10.0)
    if snr_db is not None:
        extra += (p_t + (p_t * 10.0 ** (clutter_db / 10.0) if clutter_db is not None else 0.0)) * 10.0 ** (-snr_db / 10.0)
    if extra > 0.0:
        sd = math.sqrt(extra / 2.0)
        out += torch.complex(torch.randn((m, n), generator=g, device=dev) * sd,
                             torch.randn((m, n), generator=g, device=dev) * sd)
    return sc, out


def _point_targets(ax, ay, sc0, scss, n, tgt, amp, blk: int = 64, pulse_chunk: int = 128):
    """sum_p a_p exp(j 4 pi f_ik / c (u_i . r_p)) with f_ik = sc0_i + k scss_i, as a blocked series."""
    m = ax.shape[0]
    out = np.zeros((m, n), np.complex128)
    if tgt.shape[0] == 0:
        return out
    q = (n + blk - 1) // blk
    r = np.arange(blk)
    qq = np.arange(q) * blk
    for i0 in range(0, m, pulse_chunk):
        i1 = min(m, i0 + pulse_chunk)
        proj = ax[i0:i1, None] * tgt[None, :, 0] + ay[i0:i1, None] * tgt[None, :, 1]   # (b, P)
        ph0 = (4.0 * math.pi / C) * sc0[i0:i1, None] * proj                               # (b, P)
        dph = (4.0 * math.pi / C) * scss[i0:i1, None] * proj                              # (b, P)
        a = amp[None, :, None] * np.exp(1j * (ph0[:, :, None] + dph[:, :, None] * qq[None, None, :]))
        b = np.exp(1j * dph[:, :, None] * r[None, None, :])                               # (b, P, blk)
        blocks = np.matmul(np.transpose(a, (0, 2, 1)), b)                                 # (b, q, blk)
        out[i0:i1] = blocks.reshape(i1 - i0, q * blk)[:, :n]
    return out


# ----------------------------------------------------------------------------- named workloads
# Shapes follow the five benchmark configurations: 1024^2 float scene, the Centerfield-shaped
# 5634x4319 fixed-point scene, the NDSU-shaped 8167x8192 production scene, the 4096^2 autofocus
# scene and the uneven batch.
WORKLOADS = {
    "small_1024": dict(m=1024, n=1024, bw=600e6, n_targets=64, scene_half=100.0, clutter_db=None,
                       snr_db=20.0, seed=1),
    "centerfield_5634x4319": dict(m=5634, n=4319, bw=113.6e6, n_targets=256, clutter_db=-10.0,
                                  snr_db=None, seed=2),
    "ndsu_8167x8192": dict(m=8167, n=8192, bw=600e6, n_targets=1024, clutter_db=-10.0, snr_db=15.0,
                           seed=3),
    "autofocus_4096": dict(m=4096, n=4096, bw=600e6, n_targets=128, clutter_db=-10.0, snr_db=20.0,
                           seed=4),
}


def workload_scene(name: str, **over) -> Scene:
    kw = dict(WORKLOADS[name])
    kw.update(over)
    return make_scene(**kw)


class FakeReader:
    """Duck-typed stand-in for the sarpy CPHD reader interface the reference touches
    (``get_data_size_as_tuple``, ``read_pvp_variable``, ``read_chip``, ``cphd_meta``, ``close``)."""

    class _Vec:
        def __init__(self, v):
            self.X, self.Y, self.Z = (float(v[0]), float(v[1]), float(v[2]))

    def __init__(self, scene: Scene):
        self.scene = scene
        planar = type("Planar", (), {"uIAX": self._Vec(scene.uiax), "uIAY": self._Vec(scene.uiay)})()
        refsurf = type("RefSurf", (), {"Planar": planar})()
        scoords = type("SceneCoords", (), {"ReferenceSurface": refsurf})()
        glob = type("Global", (), {"SGN": scene.sgn, "DomainType": "FX"})()
        self.cphd_meta = type("Meta", (), {"Global": glob, "SceneCoordinates": scoords})()

    def get_data_size_as_tuple(self):
        return (tuple(self.scene.dims),)

    def read_pvp_variable(self, name, index=0):
        return {"TxPos": self.scene.tx, "RcvPos": self.scene.rcv, "SRPPos": self.scene.srp,
                "SC0": self.scene.sc0, "SCSS": self.scene.scss}[name].copy()

    def read_chip(self, rows, cols, index=0):
        r0, r1, rs = rows
        c0, c1, cs = cols
        return self.scene.signal[r0:r1:rs, c0:c1:cs].copy()

    def close(self):
        pass


def phase_error(m: int, seed: int = 4, quad_edge: float = 3.0, walk_std: float = 0.05) -> np.ndarray:
    """The autofocus workload's injected per-pulse phase error (float64, radians): quadratic with
    `quad_edge` rad at the aperture edges plus a random walk of `walk_std` rad/pulse (seeded)."""
    rng = np.random.default_rng(seed)
    u = np.linspace(-1.0, 1.0, m)
    return quad_edge * u * u + np.cumsum(rng.normal(0.0, walk_std, m))
