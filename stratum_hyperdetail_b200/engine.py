"""Host engine: a mirror of the reference's src/engine.js over the C ABI.

Same buffers (src/engine.js:41-42,58), same per-frame order
(src/engine.js:67-83), same resize policy (width rounded up to a multiple of
64, height to a multiple of 8, src/engine.js:54) and the same errors
(`Renderer disposed`, `Invalid render dimensions`).  Device memory and
streams come from PyTorch; every kernel is a C-ABI call into libstratum.so.
Stage times use CUDA events in place of WebGPU timestamp queries.
"""
from __future__ import annotations

import math

import torch

from . import (BUILD_CHUNK, BUILD_CHUNKS, GROUP_NODES, LOT_FLOATS, WORLD_LOTS, call, ptr, stream_handle)

BUILD_ID = "infinite-shared-grammar-1"
STAGES = ["World descriptors", "Bounds refresh", "Exact visibility", "Materials + light", "Resolve"]
ROWS = 64


class Engine:
    def __init__(self, device: str | torch.device = "cuda"):
        self.device = torch.device(device)
        self.buffers: dict[str, torch.Tensor] = {}
        self.input = torch.zeros(32, dtype=torch.float32)
        self.frames = 0
        self.disposed = False
        self.width = self.height = 0
        self.resize_dirty = False
        self.timings = None
        self.stream = None
        self.use_drop_in_build = False  # True: 8 chunks x (build + 6 reduces) as src/engine.js:71

    # -- set-up ----------------------------------------------------------------
    def init(self, width=1600, height=900, seed=1788, warmup=True, exact_size=False, stream=None):
        if not torch.cuda.is_available():
            raise RuntimeError("STRATUM requires a CUDA device")
        self.stream = stream or torch.cuda.current_stream(self.device)
        f32, u32 = torch.float32, torch.int32  # u32 buffers are raw 32-bit words
        sizes = {"World": (WORLD_LOTS * LOT_FLOATS, f32), "Tags": (WORLD_LOTS * 4, u32),
                 "Nodes": (WORLD_LOTS * GROUP_NODES * 8, f32), "Origin": (4, u32), "C": (64, f32), "I": (32, f32),
                 "Queue": (WORLD_LOTS + 1, u32), "Args": (BUILD_CHUNKS * 21, u32), "Stats": (256, f32)}
        with torch.cuda.stream(self.stream):
            for name, (n, dt) in sizes.items():
                self.buffers[name] = torch.zeros(n, dtype=dt, device=self.device)
        self.exact_size = exact_size
        self.resize(width, height)
        b = self.buffers
        call("stratum_initCamera", ptr(b["C"]), ptr(b["Origin"]), int(seed), self._s())
        if warmup:
            self.prepare(0.0)
            self.refresh()
            self.stream.synchronize()
        return self

    def _s(self):
        return stream_handle(self.stream)

    def resize(self, width, height):
        if not (math.isfinite(width) and math.isfinite(height)):
            raise ValueError("Invalid render dimensions")
        if not self.exact_size:
            width = max(64, int(math.ceil(width / 64)) * 64)
            height = max(64, int(math.ceil(height / 8)) * 8)
        width, height = int(width), int(height)
        if width > 16384 or height > 16384:
            raise ValueError("Resolution exceeds this GPU buffer limit.")
        if width == self.width and height == self.height:
            return
        self.stream and self.stream.synchronize()
        self.width, self.height = width, height
        with torch.cuda.stream(self.stream):
            for n in ("Hit", "Surface", "Linear", "History"):
                self.buffers[n] = torch.zeros(width * height * 4, dtype=torch.float32, device=self.device)
            self.buffers["Pixels"] = torch.zeros(width * height, dtype=torch.int32, device=self.device)
        # A new resolution restarts the sampling sequence (src/engine.js:64).
        self.resize_dirty = True

    # -- per frame -------------------------------------------------------------
    def prepare(self, dt):
        self.input[23] = 1.0 if self.resize_dirty else 0.0
        self.resize_dirty = False
        b, s = self.buffers, self._s()
        b["I"].copy_(self.input, non_blocking=False)
        self.input[23] = 0.0
        dt = max(0.0, min(0.1, float(dt)))
        call("stratum_stepCamera", ptr(b["C"]), ptr(b["Origin"]), ptr(b["I"]), dt, self.width, self.height, s)
        call("stratum_clearQueue", ptr(b["Queue"]), s)
        call("stratum_prepareLots", ptr(b["Origin"]), ptr(b["C"]), ptr(b["World"]), ptr(b["Tags"]), ptr(b["Queue"]), s)
        call("stratum_planBounds", ptr(b["Queue"]), ptr(b["Args"]), s)

    def refresh_chunk(self, chunk):
        """The reference's chunked build (src/engine.js:71): leaves, then 6 levels."""
        b, s = self.buffers, self._s()
        base = chunk * BUILD_CHUNK
        call("stratum_buildGroupBounds", ptr(b["Queue"]), ptr(b["World"]), ptr(b["Nodes"]), base, s)
        for first in (32, 16, 8, 4, 2, 1):
            call("stratum_reduceGroupBounds", ptr(b["Queue"]), ptr(b["Nodes"]), first, base, s)

    def refresh(self):
        b, s = self.buffers, self._s()
        if self.use_drop_in_build:
            for c in range(BUILD_CHUNKS):
                self.refresh_chunk(c)
        else:
            call("stratum_buildBVH", ptr(b["Queue"]), ptr(b["World"]), ptr(b["Nodes"]), s)

    def draw(self):
        b, s, w, h = self.buffers, self._s(), self.width, self.height
        for y in range(0, h, ROWS):
            call("stratum_tracePrimary", ptr(b["World"]), ptr(b["Nodes"]), ptr(b["Origin"]), ptr(b["C"]),
                 ptr(b["Hit"]), ptr(b["Surface"]), w, h, y, min(ROWS, h - y), s)
        for y in range(0, h, ROWS):
            call("stratum_shadePixels", ptr(b["World"]), ptr(b["Origin"]), ptr(b["C"]), ptr(b["Hit"]),
                 ptr(b["Surface"]), ptr(b["Linear"]), w, h, y, min(ROWS, h - y), s)
        call("stratum_resolveFrame", ptr(b["Linear"]), ptr(b["History"]), ptr(b["Pixels"]), ptr(b["C"]),
             ptr(b["Hit"]), ptr(b["Surface"]), w, h, s)

    def frame(self, dt=1 / 60, draw=True, timed=False):
        if self.disposed:
            raise RuntimeError("Renderer disposed")
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if timed else None
        if ev:
            ev[0].record(self.stream)
        self.prepare(dt)
        self.refresh()
        if ev:
            ev[1].record(self.stream)
        if draw:
            self.draw()
        if ev:
            ev[2].record(self.stream)
            ev[2].synchronize()
            self.timings = [{"label": "World + bounds", "ms": ev[0].elapsed_time(ev[1])},
                            {"label": "Trace + shade + resolve", "ms": ev[1].elapsed_time(ev[2])}]
        self.frames += 1

    # -- inspection ------------------------------------------------------------
    def inspect(self):
        b = self.buffers
        self.stream.synchronize()
        c = b["C"].cpu()
        o = b["Origin"].cpu().numpy().view("uint32").astype("int64")
        q = int(b["Queue"][0].item()) & 0xFFFFFFFF

        def signed(lo, hi):
            v = (int(hi) << 32) | int(lo)
            return v - (1 << 64) if v >= (1 << 63) else v

        total = sum(t.numel() * t.element_size() for t in b.values())
        return {"build": BUILD_ID, "mode": "exact-shared-grammar", "camera": c.tolist(),
                "origin": {"x": str(signed(o[0], o[1])), "z": str(signed(o[2], o[3]))}, "refreshedLots": q,
                "accelerationLots": WORLD_LOTS, "far": 2000, "geometryModels": 1, "primitivePageAllocation": 0,
                "accelerationBytes": b["Nodes"].numel() * 4, "allocatedBytes": total, "width": self.width,
                "height": self.height, "frames": self.frames, "timings": self.timings}

    def screenshot_pixels(self):
        self.stream.synchronize()
        return self.buffers["Pixels"].cpu().numpy().view("uint8").reshape(self.height, self.width, 4)

    def reset(self, seed=1788):
        self.stream.synchronize()
        self.input.zero_()
        b = self.buffers
        for n in ("World", "Tags", "History"):
            b[n].zero_()
        call("stratum_initCamera", ptr(b["C"]), ptr(b["Origin"]), int(seed), self._s())
        self.frame(0.0, draw=False)
        self.stream.synchronize()

    def dispose(self):
        if self.disposed:
            return
        if self.stream is not None:
            self.stream.synchronize()
        self.disposed = True
        self.buffers.clear()
