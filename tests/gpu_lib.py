"""Drive the CUDA path through the C ABI for tests (device buffers from torch)."""
from __future__ import annotations

import numpy as np
import torch

import stratum_hyperdetail_b200 as sb
from stratum_hyperdetail_b200 import call, ptr

WORLD_LOTS = 16384


def s():
    return torch.cuda.current_stream().cuda_stream


def u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


class GpuWorld:
    def __init__(self):
        dev = "cuda"
        self.C = torch.zeros(64, dtype=torch.float32, device=dev)
        self.Origin = torch.zeros(4, dtype=torch.int32, device=dev)
        self.I = torch.zeros(32, dtype=torch.float32, device=dev)
        self.World = torch.zeros(WORLD_LOTS * 16, dtype=torch.float32, device=dev)
        self.Tags = torch.zeros(WORLD_LOTS * 4, dtype=torch.int32, device=dev)
        self.Nodes = torch.zeros(WORLD_LOTS * 128 * 8, dtype=torch.float32, device=dev)
        self.Queue = torch.zeros(WORLD_LOTS + 1, dtype=torch.int32, device=dev)
        self.Args = torch.zeros(8 * 21, dtype=torch.int32, device=dev)

    def refresh(self, drop_in=False):
        call("stratum_clearQueue", ptr(self.Queue), s())
        call("stratum_prepareLots", ptr(self.Origin), ptr(self.C), ptr(self.World), ptr(self.Tags), ptr(self.Queue), s())
        call("stratum_planBounds", ptr(self.Queue), ptr(self.Args), s())
        if drop_in:
            for c in range(8):
                call("stratum_buildGroupBounds", ptr(self.Queue), ptr(self.World), ptr(self.Nodes), c * 2048, s())
                for first in (32, 16, 8, 4, 2, 1):
                    call("stratum_reduceGroupBounds", ptr(self.Queue), ptr(self.Nodes), first, c * 2048, s())
        else:
            call("stratum_buildBVH", ptr(self.Queue), ptr(self.World), ptr(self.Nodes), s())


def setup_pose(seed, pos, yaw, pitch, width, height, sample=1, shadows=True, origin=None, drop_in=False):
    g = GpuWorld()
    call("stratum_initCamera", ptr(g.C), ptr(g.Origin), int(seed), s())
    c = g.C.cpu()
    c[0], c[1], c[2] = pos
    c[3], c[4] = yaw, pitch
    c[18] = 0.0 if shadows else 1.0
    g.C.copy_(c)
    if origin is not None:
        g.Origin.copy_(torch.from_numpy(np.asarray(origin, np.uint32).view(np.int32)))
    call("stratum_stepCamera", ptr(g.C), ptr(g.Origin), ptr(g.I), 0.0, int(width), int(height), s())
    g.C[19] = float(sample)
    g.refresh(drop_in)
    torch.cuda.synchronize()
    return g


class Frame:
    def __init__(self, width, height):
        P = width * height
        dev = "cuda"
        self.width, self.height = width, height
        self.Hit = torch.zeros(P * 4, dtype=torch.float32, device=dev)
        self.Surface = torch.zeros(P * 4, dtype=torch.float32, device=dev)
        self.Linear = torch.zeros(P * 4, dtype=torch.float32, device=dev)
        self.History = torch.zeros(P * 4, dtype=torch.float32, device=dev)
        self.Pixels = torch.zeros(P, dtype=torch.int32, device=dev)

    def render(self, g: GpuWorld, rows=64):
        w, h = self.width, self.height
        for y in range(0, h, rows):
            call("stratum_tracePrimary", ptr(g.World), ptr(g.Nodes), ptr(g.Origin), ptr(g.C), ptr(self.Hit),
                 ptr(self.Surface), w, h, y, min(rows, h - y), s())
        for y in range(0, h, rows):
            call("stratum_shadePixels", ptr(g.World), ptr(g.Origin), ptr(g.C), ptr(self.Hit), ptr(self.Surface),
                 ptr(self.Linear), w, h, y, min(rows, h - y), s())
        call("stratum_resolveFrame", ptr(self.Linear), ptr(self.History), ptr(self.Pixels), ptr(g.C), ptr(self.Hit),
             ptr(self.Surface), w, h, s())
        torch.cuda.synchronize()
        return self.numpy()

    def numpy(self):
        return {k: getattr(self, k).cpu().numpy() for k in ("Hit", "Surface", "Linear", "History")} | {
            "Pixels": u32(self.Pixels)}


def compare_frames(gpu: dict, orc: dict, second: np.ndarray, tol_t=1e-5, tol_n=1e-5, tol_c=1 / 1024):
    """Identity, distance, normal and colour comparison with the tie rule.

    Returns a report dict; `identity_bad` counts rays whose identity differs
    although their nearest and second-nearest candidates are farther apart
    than the distance tolerance."""
    gh, oh = gpu["Hit"].reshape(-1, 4), orc["Hit"].reshape(-1, 4)
    gs, os_ = gpu["Surface"].reshape(-1, 4), orc["Surface"].reshape(-1, 4)
    same_id = (gh[:, 1] == oh[:, 1]) & (gs[:, 3] == os_[:, 3])
    tie = np.abs(second - oh[:, 0]) <= tol_t * np.maximum(oh[:, 0], 1e-3)
    identity_bad = int((~same_id & ~tie).sum())
    t_err = np.abs(gh[:, 0] - oh[:, 0]) / np.maximum(np.abs(oh[:, 0]), 1e-6)
    n_err = np.abs(gs[:, :3] - os_[:, :3]).max(axis=1)
    m = same_id
    lin_err = np.abs(gpu["Linear"].reshape(-1, 4) - orc["Linear"].reshape(-1, 4)).max(axis=1)
    hist_err = np.abs(gpu["History"].reshape(-1, 4) - orc["History"].reshape(-1, 4)).max(axis=1)
    px_g = gpu["Pixels"].view(np.uint8).reshape(-1, 4).astype(int)
    px_o = orc["Pixels"].view(np.uint8).reshape(-1, 4).astype(int)
    return {
        "rays": int(len(gh)),
        "identity_mismatch": int((~same_id).sum()),
        "identity_bad": identity_bad,
        "t_bad": int((t_err[m] > tol_t).sum()),
        "t_max_rel": float(t_err[m].max()) if m.any() else 0.0,
        "n_bad": int((n_err[m] > tol_n).sum()),
        "material_bad": int((gh[m, 2:] != oh[m, 2:]).any(axis=1).sum()),
        "linear_bad": int((lin_err > tol_c).sum()),
        "linear_max": float(lin_err.max()),
        "history_bad": int((hist_err > tol_c).sum()),
        "pixels_off_by_more_than_1": int((np.abs(px_g - px_o).max(axis=1) > 1).sum()),
        "bit_exact_hit": bool(np.array_equal(gh.view(np.uint32), oh.view(np.uint32))),
        "bit_exact_linear": bool(np.array_equal(gpu["Linear"].view(np.uint32), orc["Linear"].view(np.uint32))),
    }
