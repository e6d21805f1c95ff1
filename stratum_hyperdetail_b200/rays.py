"""Arbitrary rays against a view's lot table, and the hierarchy-vs-exhaustive check.

`trace` is stratum_traceRays: the nearest hit of each ray through the
hierarchy, or exhaustively (every group of every visited lot, no culling).
`retest` is stratum_retestFeatures: one named (slot, fid) feature on one ray.
`compare_hierarchy` is the reference's hierarchy-vs-exhaustive test
(tests/native_harness.cpp:68-79) at any scale: distances must agree bit for
bit, and where the two answers name different features, both features are
re-tested on that ray -- equal distances bit for bit make the pair an exact
tie (the two traversals visit tied features in different orders and keep the
first), anything else is a real disagreement.
"""
from __future__ import annotations

import torch

from . import call, ptr

FAR = 2000.0


def _s(stream):
    return (stream or torch.cuda.current_stream()).cuda_stream


def trace(view, rays: torch.Tensor, exhaustive: bool, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """rays: (n, 7) f32 [ro.xyz, rd.xyz, cone] on the device -> (n, 8) [t, fid, material, seed, n.xyz, slot]."""
    n = rays.shape[0]
    if out is None:
        out = torch.empty((n, 8), dtype=torch.float32, device=rays.device)
    call("stratum_traceRays", ptr(view.World), ptr(view.Nodes), ptr(view.Origin), ptr(rays), n, int(exhaustive),
         ptr(out), _s(stream))
    return out


def retest(view, rays: torch.Tensor, ids: torch.Tensor, stream=None) -> torch.Tensor:
    """ids: (n, 2) i32 [slot, fid] -> (n, 4) [t, n.xyz] of that feature on that ray (t = FAR if missed)."""
    n = rays.shape[0]
    out = torch.empty((n, 4), dtype=torch.float32, device=rays.device)
    if n:
        call("stratum_retestFeatures", ptr(view.World), ptr(view.Origin), ptr(rays.contiguous()),
             ptr(ids.contiguous()), n, ptr(out), _s(stream))
    return out


def compare_hierarchy(view, rays: torch.Tensor, h: torch.Tensor, e: torch.Tensor, stream=None) -> dict:
    """Hierarchy result `h` vs exhaustive result `e` of the same rays (both (n, 8)).

    Returns counts: distance_mismatches (t differs in any bit),
    identity_mismatches (fid or slot differs), identity_ties (both named
    features give the reported distance bit for bit on the ray) and
    identity_mismatches_non_tie (the rest; must be 0)."""
    hb, eb = h.view(torch.int32), e.view(torch.int32)
    same_t = hb[:, 0] == eb[:, 0]
    diff_id = (h[:, 1] != e[:, 1]) | (h[:, 7] != e[:, 7])
    idx = torch.nonzero(diff_id & same_t).flatten()
    ties = 0
    if idx.numel():
        r = rays[idx]
        t_ref = h[idx, 0]

        def side(res):
            ids = torch.stack([res[idx, 7], res[idx, 1]], 1).to(torch.int32)
            t = retest(view, r, ids, stream)[:, 0]
            # the ground plane (fid -1) is not a feature: its distance is the reported one
            return torch.where(res[idx, 1] == -1, t_ref, t)

        th, te = side(h), side(e)
        tie = (th.view(torch.int32) == te.view(torch.int32)) & (th.view(torch.int32) == t_ref.view(torch.int32))
        ties = int(tie.sum())
    mism = int(diff_id.sum())
    return {"distance_mismatches": int((~same_t).sum()), "identity_mismatches": mism, "identity_ties": ties,
            "identity_mismatches_non_tie": mism - ties}
