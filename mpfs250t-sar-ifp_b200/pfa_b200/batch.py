"""Batched uneven scenes: many PFA frames of different shapes in one graph-captured launch.

``BatchFormer`` owns one float plan per scene (each with its autotuned FFT tile), assigns the scenes
to ``streams`` CUDA streams largest-first (greedy on the estimated frame cost, so the streams finish
together), and captures the whole batch -- for every scene ``af_iters`` autofocus gradient steps on its
per-pulse phase, the phase-corrected signal and the final detected image -- into one CUDA graph.
``replay()`` then forms the whole batch with a single graph launch; kernels of different scenes
overlap across the streams.  Every node of the graph is a kernel of the engine: the autofocus update runs
on the device (``pfa_autofocus_step``) and the final image applies the phase correction in pass 1
(``pfa_form_float_phase``), so the batch has no eager tensor operations and no host round trip.
``run_eager()`` is the one-scene-at-a-time reference on a single stream.
"""
from __future__ import annotations

from . import autofocus as af
from .engine import FloatPlan


class BatchFormer:
    def __init__(self, scenes, range_sinc=False, az_sinc=False, streams=4, tiles=None, af_iters=0,
                 af_step=0.3, device=0, mixed=False):
        """scenes: list of (tables, signal) with signal an (m, n) complex64 CUDA tensor.  ``mixed``: form
        the final images with the split-precision tensor-core FFTs (the autofocus gradients stay FP32)."""
        import torch
        self.torch = torch
        self.n = len(scenes)
        self.af_iters, self.af_step = int(af_iters), float(af_step)
        self.signals = [s for _, s in scenes]
        self.plans = []
        for i, (tb, sig) in enumerate(scenes):
            m, n = tuple(sig.shape)
            tile = tiles[i] if tiles is not None else (0, 0)
            p = FloatPlan(m, n, range_sinc, az_sinc, mixed=mixed, device=device, tile=tile)
            p.set_tables(tb)
            self.plans.append(p)
        dev = self.signals[0].device
        self.images = [torch.empty((p.m2, p.n2), dtype=torch.float32, device=dev) for p in self.plans]
        self.theta = [torch.zeros(p.m, dtype=torch.float32, device=dev) for p in self.plans]
        self.zero = [torch.zeros_like(t) for t in self.theta]
        self.nstreams = max(1, min(int(streams), self.n))
        self.streams = [torch.cuda.Stream(device=dev) for _ in range(self.nstreams)]
        cost = [p.m2 * p.n2 for p in self.plans]
        load = [0] * self.nstreams
        self.assign = [0] * self.n
        for i in sorted(range(self.n), key=lambda k: -cost[k]):
            s = min(range(self.nstreams), key=lambda k: load[k])
            self.assign[i] = s
            load[s] += cost[i]
        self.graph = None

    def _scene(self, i, stream):
        p, sig = self.plans[i], self.signals[i]
        th = self.theta[i]
        th.copy_(self.zero[i])               # a memcpy node: theta starts at 0 on every replay
        for _ in range(self.af_iters):
            af.descent_step(p, sig, th, self.af_step, stream=stream)
        if self.af_iters:
            af.form_corrected(p, sig, th, out=self.images[i], stream=stream)
        else:
            p.form(sig, out=self.images[i], stream=stream)

    def run_eager(self):
        """One scene after another on the current stream (the baseline the graph is compared with)."""
        torch = self.torch
        st = torch.cuda.current_stream()
        for i in range(self.n):
            self._scene(i, st)

    def capture(self):
        torch = self.torch
        self.run_eager()                     # warm-up: lazy workspaces, kernel attributes
        torch.cuda.synchronize()
        cap = torch.cuda.Stream(device=self.signals[0].device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=cap):
            for s in self.streams:
                s.wait_stream(cap)
            for i in sorted(range(self.n), key=lambda k: self.assign[k]):
                st = self.streams[self.assign[i]]
                with torch.cuda.stream(st):
                    self._scene(i, st)
            for s in self.streams:
                cap.wait_stream(s)
        return self.graph

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def close(self):
        self.graph = None
        for p in self.plans:
            p.close()
