"""Per-view device state for the plain per-frame path.

A `View` owns one view's buffers (one 128x128 lot table, its 64 MiB
hierarchy and the frame buffers) and drives them through the C ABI in the
reference engine's order.  `frame()` is the single C-ABI call
`stratum_frame`; `frame_parts()` issues the same sequence entry point by
entry point so a caller can bracket the trace launches with CUDA events.
"""
from __future__ import annotations

import numpy as np
import torch

from . import BUILD_CHUNKS, GROUP_CACHE_ENTRIES, GROUP_NODES, LOT_FLOATS, WORLD_LOTS, call, lib, ptr

ROWS = 64


def _s(stream):
    return (stream or torch.cuda.current_stream()).cuda_stream


class View:
    def __init__(self, width: int, height: int, device="cuda"):
        self.width, self.height = int(width), int(height)
        f32, i32 = torch.float32, torch.int32
        P = self.width * self.height
        z = lambda n, dt: torch.zeros(n, dtype=dt, device=device)  # noqa: E731
        self.C, self.Origin, self.I = z(64, f32), z(4, i32), z(32, f32)
        self.World, self.Tags = z(WORLD_LOTS * LOT_FLOATS, f32), z(WORLD_LOTS * 4, i32)
        self.Nodes = z(WORLD_LOTS * GROUP_NODES * 8, f32)
        self.Queue, self.Args = z(WORLD_LOTS + 1, i32), z(BUILD_CHUNKS * 21, i32)
        self.Hit, self.Surface = z(P * 4, f32), z(P * 4, f32)
        self.Linear, self.History = z(P * 4, f32), z(P * 4, f32)
        self.Pixels = z(P, i32)
        self.Groups = None  # group cache of the table (batched trace only)

    @property
    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.C, self.Origin, self.I, self.World, self.Tags,
                                                          self.Nodes, self.Queue, self.Args, self.Hit, self.Surface,
                                                          self.Linear, self.History, self.Pixels)) + (
            0 if self.Groups is None else self.Groups.numel() * 4)

    def enable_group_cache(self, entries: int = GROUP_CACHE_ENTRIES, stream=None):
        """Give the table a group cache of `entries` groups (read and filled by
        the batched trace; results are the same with or without it).  0
        removes it."""
        if entries <= 0:
            self.Groups = None
            return
        n = int(lib().stratum_groupCacheBytes(int(entries)))
        self.Groups = torch.empty((n + 3) // 4, dtype=torch.int32, device=self.World.device)
        call("stratum_groupCacheInit", ptr(self.Groups), int(entries), _s(stream))

    def set_pose(self, seed, origin, pos, yaw, pitch, shadows=True, stream=None):
        """initCamera(seed), place the camera in the lot frame of `origin`,
        stepCamera(dt=0) (which rebases), then refresh the whole table."""
        s = _s(stream)
        call("stratum_initCamera", ptr(self.C), ptr(self.Origin), int(seed), s)
        c = self.C.cpu()
        c[0], c[1], c[2] = pos
        c[3], c[4] = yaw, pitch
        c[18] = 0.0 if shadows else 1.0
        self.C.copy_(c)
        self.Origin.copy_(torch.from_numpy(np.asarray(origin, np.uint32).view(np.int32)))
        call("stratum_stepCamera", ptr(self.C), ptr(self.Origin), ptr(self.I), 0.0, self.width, self.height, s)
        # the first drawn frame is sample 1 (stepCamera in the frame advances it)
        self.C[19] = 0.0
        self.refresh(stream)

    def save_ppm(self, path) -> None:
        """Write the last resolved frame (Pixels, RGBA8) as a binary PPM (P6):
        the reference harness's image format (tests/native_harness.cpp:115),
        rows in buffer order, R, G, B from the low three bytes."""
        px = self.Pixels.cpu().numpy().view(np.uint8).reshape(self.height, self.width, 4)[..., :3]
        with open(path, "wb") as f:
            f.write(f"P6\n{self.width} {self.height}\n255\n".encode())
            f.write(np.ascontiguousarray(px).tobytes())

    def refresh(self, stream=None):
        s = _s(stream)
        call("stratum_clearQueue", ptr(self.Queue), s)
        call("stratum_prepareLots", ptr(self.Origin), ptr(self.C), ptr(self.World), ptr(self.Tags), ptr(self.Queue), s)
        call("stratum_planBounds", ptr(self.Queue), ptr(self.Args), s)
        call("stratum_buildBVH", ptr(self.Queue), ptr(self.World), ptr(self.Nodes), s)

    def frame(self, dt=0.0, stream=None):
        """One frame through the single C-ABI call (src/engine.js:72-83)."""
        call("stratum_frame", ptr(self.C), ptr(self.Origin), ptr(self.I), float(dt), ptr(self.World), ptr(self.Tags),
             ptr(self.Nodes), ptr(self.Queue), ptr(self.Args), ptr(self.Hit), ptr(self.Surface), ptr(self.Linear),
             ptr(self.History), ptr(self.Pixels), self.width, self.height, 1, _s(stream))

    def frame_parts(self, dt=0.0, stream=None, trace_events=None):
        """The same sequence as `frame`, entry point by entry point.  With
        `trace_events=(start, end)` the trace strips are bracketed.  Returns
        the number of kernel launches issued."""
        s = _s(stream)
        w, h = self.width, self.height
        call("stratum_stepCamera", ptr(self.C), ptr(self.Origin), ptr(self.I), float(dt), w, h, s)
        self.refresh(stream)
        n = 5
        if trace_events:
            trace_events[0].record(stream)
        for y in range(0, h, ROWS):
            call("stratum_tracePrimary", ptr(self.World), ptr(self.Nodes), ptr(self.Origin), ptr(self.C), ptr(self.Hit),
                 ptr(self.Surface), w, h, y, min(ROWS, h - y), s)
            n += 1
        if trace_events:
            trace_events[1].record(stream)
        for y in range(0, h, ROWS):
            call("stratum_shadePixels", ptr(self.World), ptr(self.Origin), ptr(self.C), ptr(self.Hit), ptr(self.Surface),
                 ptr(self.Linear), w, h, y, min(ROWS, h - y), s)
            n += 1
        call("stratum_resolveFrame", ptr(self.Linear), ptr(self.History), ptr(self.Pixels), ptr(self.C), ptr(self.Hit),
             ptr(self.Surface), w, h, s)
        return n + 1
