"""Streaming world on the GPU: a camera flies 10 km at 40 m altitude and
40 m/s (15,000 frames at 60 Hz) across the 64-bit carry of the x lot address
(start xl = 0xFFFFFFF0), one stepCamera + lot refresh + hierarchy refresh per
frame.

Checks:
  * every cell crossing refreshes exactly one 128-lot column, other frames none;
  * at the carry and at checkpoints along the flight, the incrementally
    maintained table (World, Tags, Nodes) equals a table built from scratch by
    the CPU oracle for the same origin, bit for bit;
  * at every 12th cell crossing and around the carry, 65,536 uniformly random
    rays agree hierarchy-vs-exhaustive on the GPU: distance bit for bit on
    every ray, and where the two name different features, both features are
    re-tested on the ray (GPU and oracle) and must give that distance bit for
    bit -- an exact tie, not a disagreement; a subset agrees with the oracle's
    hierarchy query bit for bit.
"""
import math

import numpy as np
import pytest
import torch

import oracle_lib as ol

pytestmark = pytest.mark.gpu
RAYS = 65536


def random_rays(rng, n):
    ro = np.stack([rng.uniform(-900, 900, n), rng.uniform(0.5, 60.0, n), rng.uniform(-900, 900, n)], 1)
    d = rng.normal(size=(n, 3))
    d[:, 1] = -np.abs(d[:, 1]) * 0.35
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([ro, d, np.full((n, 1), 0.0015)], 1).astype(np.float32)


def trace_rays(v, rays, exhaustive):
    import stratum_hyperdetail_b200 as sb
    R = torch.from_numpy(rays).cuda()
    out = torch.zeros(len(rays) * 8, dtype=torch.float32, device="cuda")
    sb.call("stratum_traceRays", sb.ptr(v.World), sb.ptr(v.Nodes), sb.ptr(v.Origin), sb.ptr(R), len(rays),
            int(exhaustive), sb.ptr(out), torch.cuda.current_stream().cuda_stream)
    return out.cpu().numpy().reshape(-1, 8)


FRAMES = 15000          # 10 km at 40 m/s, 60 Hz
CARRY_FRAME = 837       # xl 0xFFFFFFFF -> 0, xh 0 -> 1
TABLE_CHECKS = {500, 836, 837, 1000, 7500, 15000}


def test_flight_across_the_carry(cuda, oracle):
    import stratum_hyperdetail_b200 as sb
    import stratum_hyperdetail_b200.rays as sr
    from stratum_hyperdetail_b200.views import View
    s = torch.cuda.current_stream().cuda_stream
    v = View(256, 144)
    v.set_pose(0x5EED, (0xFFFFFFF0, 0, 7, 0), (0.0, 40.0, 0.0), math.pi / 2, 0.0)
    v.C[12] = 40.0  # m/s
    v.I[0] = 1.0    # forward
    rng = np.random.default_rng(1)
    prev = v.Origin.cpu().numpy().view(np.uint32).copy()
    checked, crossings, ties = [], 0, 0
    for frame in range(1, FRAMES + 1):
        sb.call("stratum_stepCamera", sb.ptr(v.C), sb.ptr(v.Origin), sb.ptr(v.I), 1.0 / 60.0, 256, 144, s)
        v.refresh()
        org = v.Origin.cpu().numpy().view(np.uint32).copy()
        refreshed = int(v.Queue[0].item())
        moved = int((int(org[0]) - int(prev[0])) & 0xFFFFFFFF)
        # 40 m/s at 60 Hz is 0.67 m a frame: at most one 36 m cell per frame
        assert moved in (0, 1) and org[2] == prev[2] and org[3] == prev[3], (frame, prev, org)
        assert refreshed == 128 * moved, (frame, moved, refreshed)
        if org[1] != prev[1]:
            assert org[0] == 0 and prev[0] == 0xFFFFFFFF and org[1] == prev[1] + 1, (frame, prev, org)
        crossings += moved
        prev = org
        rays_check = frame in (CARRY_FRAME - 1, CARRY_FRAME) or (moved and crossings % 12 == 0)
        if frame in TABLE_CHECKS or rays_check:
            torch.cuda.synchronize()
            C = v.C.cpu().numpy()
            # incremental GPU table == from-scratch CPU table for this origin
            ref = ol.World()
            ref.Origin[:] = org
            ref.C[:] = C
            oracle.f("clearQueue")(ref.Queue)
            oracle.f("prepareLots")(ref.Origin, ref.C, ref.World, ref.Tags, ref.Queue)
            oracle.build_bounds(ref.Queue, ref.World, ref.Nodes)
            assert np.array_equal(v.World.cpu().numpy().view(np.uint32), ref.World.view(np.uint32)), frame
            assert np.array_equal(v.Tags.cpu().numpy().view(np.uint32), ref.Tags), frame
            assert np.array_equal(v.Nodes.cpu().numpy(), ref.Nodes), frame
            if not rays_check:
                continue
            # hierarchy vs exhaustive over 65,536 random rays
            rays = random_rays(rng, RAYS)
            h, e = trace_rays(v, rays, False), trace_rays(v, rays, True)
            same_t = h[:, 0].view(np.uint32) == e[:, 0].view(np.uint32)
            assert same_t.all(), np.where(~same_t)[0][:10]
            # an identity may differ only where two features tie exactly: re-test both on the ray
            R = torch.from_numpy(rays).cuda()
            rep = sr.compare_hierarchy(v, R, torch.from_numpy(h).cuda(), torch.from_numpy(e).cuda())
            assert rep["distance_mismatches"] == 0 and rep["identity_mismatches_non_tie"] == 0, (frame, rep)
            diff = np.flatnonzero((h[:, 1] != e[:, 1]) | (h[:, 7] != e[:, 7]))
            if len(diff):
                for res in (h, e):
                    ids = np.stack([res[diff, 7], res[diff, 1]], 1).astype(np.int32)
                    g = sr.retest(v, R[torch.from_numpy(diff).cuda()], torch.from_numpy(ids).cuda()).cpu().numpy()
                    o = oracle.retest_features(ref.World, ref.Origin, rays[diff], ids)
                    feat = res[diff, 1] >= 0
                    assert np.array_equal(g[feat].view(np.uint32), o[feat].view(np.uint32)), frame
                    assert np.array_equal(g[feat, 0].view(np.uint32), h[diff[feat], 0].view(np.uint32)), frame
            ties += rep["identity_ties"]
            sub = rays[:2048]
            o = oracle.trace_rays(ref.World, ref.Nodes, ref.Origin, sub, False)
            assert np.array_equal(h[:2048].view(np.uint32), o.view(np.uint32))
            checked.append((frame, int(org[0]), int(org[1]), int((h[:, 1] >= 0).sum())))
    # the carry was crossed: xl wrapped past 0 and xh went from 0 to 1
    # 15,000 frames x 0.67 m = 10 km = 278 cells: xl 0xFFFFFFF0 -> 0x106 with xh 0 -> 1 (carry at frame 837)
    assert crossings == 278 and tuple(prev[:2]) == (0x106, 1), (crossings, prev)
    assert any(c[1:3] == (0xFFFFFFFF, 0) for c in checked) and any(c[1:3] == (0, 1) for c in checked), checked
    assert len(checked) >= 24, checked
    print("streaming checkpoints (frame, xl, xh, hits of 65,536):", checked, "exact ties:", ties)
