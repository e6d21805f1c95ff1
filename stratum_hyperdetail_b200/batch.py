"""Batched multi-view rendering over the C ABI.

A `Batch` holds a device table of stratum_view records for a set of `View`s
(any mix of resolution, pose and world seed), the batched renderer's scratch,
the chosen tune, and optionally a CUDA graph of the whole batched frame
(stepViews, refreshViews, buildViews, renderViews), replayed each frame.
"""
from __future__ import annotations

import ctypes as ct

import torch

from . import GROUP_CACHE_ENTRIES, Tune, ViewRecord, call, lib, ptr
from .views import View


def _s(stream):
    return (stream or torch.cuda.current_stream()).cuda_stream


class Batch:
    def __init__(self, views: list[View], tune: tuple[int, int, int] = (128, 1, 1), device="cuda",
                 group_cache: int = GROUP_CACHE_ENTRIES):
        """`group_cache`: entries of the group cache given to every view that has
        none yet (0: views without a cache stay without one)."""
        if not views:
            raise ValueError("a batch needs at least one view")
        self.views = list(views)
        self.n = len(self.views)
        rec = (ViewRecord * self.n)()
        for r, v in zip(rec, self.views):
            if group_cache > 0 and v.Groups is None:
                v.enable_group_cache(group_cache)
            for name in ("C", "Origin", "I", "World", "Tags", "Nodes", "Queue", "Hit", "Surface", "Linear",
                         "History", "Pixels", "Groups"):
                setattr(r, name, ptr(getattr(v, name)))
            r.width, r.height, r.dt = v.width, v.height, 0.0
        raw = bytes(rec)
        self.table = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)
        self.scratch_bytes = int(lib().stratum_batchScratchBytes(self.n))
        self.scratch = torch.zeros((self.scratch_bytes + 255) // 256 * 256, dtype=torch.uint8, device=device)
        self.tune = Tune(*tune)
        self.graph = None

    def set_dt(self, dt: float):
        """Time step of every view for the next frames (re-captures nothing)."""
        rec = (ViewRecord * self.n).from_buffer_copy(self.table.cpu().numpy().tobytes())
        for r in rec:
            r.dt = float(dt)
        self.table.copy_(torch.frombuffer(bytearray(bytes(rec)), dtype=torch.uint8))

    def _args(self):
        return ptr(self.table), self.n, ptr(self.scratch), self.scratch_bytes, ct.byref(self.tune)

    def frame(self, stream=None):
        """One batched frame: one sample of every view."""
        call("stratum_frameViews", *self._args(), _s(stream))

    def render(self, stream=None):
        call("stratum_renderViews", *self._args(), _s(stream))

    def trace(self, stream=None):
        call("stratum_traceViews", *self._args(), _s(stream))

    def render_no_alloc(self, stream=None):
        """renderViews through the allocation-free entry point: the library's
        own static scratch instead of this batch's scratch buffer (at most
        NOALLOC_MAX_VIEWS views; calls must not overlap on the GPU)."""
        call("stratum_renderViewsNoAlloc", ptr(self.table), self.n, ct.byref(self.tune), _s(stream))

    def shade(self, stream=None):
        call("stratum_shadeViews", *self._args(), _s(stream))

    def step(self, stream=None):
        call("stratum_stepViews", ptr(self.table), self.n, _s(stream))

    def refresh(self, stream=None):
        s = _s(stream)
        call("stratum_refreshViews", ptr(self.table), self.n, s)
        call("stratum_buildViews", ptr(self.table), self.n, s)

    def autotune(self, stream=None) -> float:
        best = Tune()
        ms = ct.c_float(0.0)
        call("stratum_autotune", ptr(self.table), self.n, ptr(self.scratch), self.scratch_bytes, ct.byref(best),
             ct.byref(ms), _s(stream))
        self.tune = best
        self.graph = None
        return ms.value

    @property
    def launches_per_frame(self) -> int:
        # stepViews, clearViews, refreshViews, buildViews, prologue, cacheReset, trace, shade, light, resolve
        return 10

    def capture(self):
        """Capture one batched frame as a CUDA graph (after one eager frame so
        every lazily initialised launch parameter exists)."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self.frame(side)
        torch.cuda.current_stream().wait_stream(side)
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            raise RuntimeError("no captured graph: call capture() first")
        self.graph.replay()
