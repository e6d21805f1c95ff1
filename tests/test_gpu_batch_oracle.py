"""The batched renderer against the CPU oracle directly (not only against the
drop-in path), through the C ABI.

* Debug view modes C[11] = 1 (palette), 2 (group ids), 3 (normals) and the
  shadows-off switch C[18] = 1 (kernels/shade.cu:78,97-99) rendered by the
  batched launch, all four at once in one batch, against the oracle.
* A streaming flight on the batched path (stepViews with a forward input,
  refresh of the entering lot column, build, trace, shade, resolve per 60 Hz
  frame) from xl = 0xFFFFFFF0 across the 64-bit carry: at the carry frame and
  at the last frame the rendered frame is compared with the oracle's render of
  the same camera state over a table built from scratch for the same origin
  (the running History is handed to the oracle so the accumulation step is
  compared exactly).
* Frames of 1x1, 7x3, 9x5, 33x17, 16,384 x 4 (the maximum width) and 3 x 2,000,
  batched and through the drop-in strips, against the oracle.

The oracle evaluates camera angles as the device does (double precision
rounded once), so Hit and Surface must be bit-identical; colour within 1/1024.
"""
import math

import numpy as np
import pytest
import torch

import oracle_lib as ol
from gpu_lib import compare_frames

pytestmark = pytest.mark.gpu
TOL_T, TOL_N, TOL_C = 1e-5, 1e-5, 1.0 / 1024.0


def host_frame(v):
    out = {k: getattr(v, k).cpu().numpy() for k in ("Hit", "Surface", "Linear", "History")}
    out["Pixels"] = v.Pixels.cpu().numpy().view(np.uint32)
    return out


def check(tag, got, want, second):
    rep = compare_frames(got, want, second, TOL_T, TOL_N, TOL_C)
    print(tag, {k: rep[k] for k in ("rays", "identity_bad", "t_bad", "n_bad", "linear_bad", "history_bad",
                                     "bit_exact_hit")})
    assert rep["bit_exact_hit"], (tag, rep)
    assert rep["identity_bad"] == 0 and rep["t_bad"] == 0 and rep["n_bad"] == 0, (tag, rep)
    assert rep["linear_bad"] <= max(2, rep["rays"] // 10000) and rep["history_bad"] <= max(2, rep["rays"] // 10000), rep


def test_debug_views_and_shadows_off_batched(cuda, oracle):
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    pos, origin, yaw, pitch, w, h = (17.0, 1.7, 0.0), (0, 0, 0, 0), 0.3, 0.0, 192, 108
    modes = [(1, False), (2, False), (3, False), (0, True)]
    views = []
    for mode, shadows_off in modes:
        v = View(w, h)
        v.set_pose(0x5EED, origin, pos, yaw, pitch, shadows=not shadows_off)
        v.C[11] = float(mode)
        v.C[19] = 1.0
        views.append(v)
    b = Batch(views)
    b.render()
    torch.cuda.synchronize()
    with ol.device_angles(oracle):
        for (mode, shadows_off), v in zip(modes, views):
            o = ol.setup_pose(oracle, 0x5EED, pos, yaw, pitch, w, h, shadows=not shadows_off, origin=origin)
            o.C[11] = np.float32(mode)
            second = np.zeros(w * h, np.float32)
            want = ol.render(oracle, o, w, h, second=second)
            check(f"batched view mode {mode} shadows {'off' if shadows_off else 'on'}", host_frame(v), want, second)


def test_streaming_flight_frames_against_oracle(cuda, oracle):
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    w, h = 256, 144
    v = View(w, h)
    v.set_pose(0x5EED, (0xFFFFFFF0, 0, 7, 0), (0.0, 40.0, 0.0), math.pi / 2, 0.0)
    v.C[12] = 40.0  # m/s
    v.I[0] = 1.0    # forward
    b = Batch([v])
    b.set_dt(1.0 / 60.0)
    compared = []
    for frame in range(1, 901):
        if frame in (837, 900):  # the carry (xl 0xFFFFFFFF -> 0, xh 0 -> 1), and the last frame
            torch.cuda.synchronize()
            history = v.History.cpu().numpy().copy()
        b.frame()
        if frame not in (837, 900):
            continue
        torch.cuda.synchronize()
        org = v.Origin.cpu().numpy().view(np.uint32).copy()
        C = v.C.cpu().numpy().copy()
        with ol.device_angles(oracle):
            s = ol.World()
            s.Origin[:] = org
            s.C[:] = C
            oracle.f("clearQueue")(s.Queue)
            oracle.f("prepareLots")(s.Origin, s.C, s.World, s.Tags, s.Queue)
            oracle.build_bounds(s.Queue, s.World, s.Nodes)
            assert np.array_equal(v.World.cpu().numpy().view(np.uint32), s.World.view(np.uint32)), frame
            assert np.array_equal(v.Tags.cpu().numpy().view(np.uint32), s.Tags), frame
            assert np.array_equal(v.Nodes.cpu().numpy(), s.Nodes), frame
            second = np.zeros(w * h, np.float32)
            want = ol.render(oracle, s, w, h, second=second, history=history)
        check(f"flight frame {frame} origin {org[:2]}", host_frame(v), want, second)
        compared.append((frame, int(org[0]), int(org[1])))
    assert compared[0][1:] == (0, 1), compared  # the carry frame: xl wrapped to 0, xh incremented
    assert compared[-1][2] == 1, compared


def test_tiny_ragged_and_extreme_frames_against_oracle(cuda, oracle):
    """Frames smaller than one 8x4 tile, with ragged edges, and at the maximum
    width (16,384 x 4) and a 3 x 2,000 column, rendered by the batched launch
    and by the drop-in strips (64 rows, the last one asking for more rows than
    remain), each against the oracle."""
    import stratum_hyperdetail_b200 as sb
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    sizes = [(1, 1), (7, 3), (9, 5), (33, 17), (16384, 4), (3, 2000)]
    poses = [((3.0 * i, 1.7 + 9.0 * i, -2.0), 0.4 * i + 0.1, -0.05 * i) for i in range(len(sizes))]
    views = []
    for i, ((w, h), (pos, yaw, pitch)) in enumerate(zip(sizes, poses)):
        v = View(w, h)
        v.set_pose(100 + i, (i, 0, 2 * i, 0), pos, yaw, pitch)
        v.C[19] = 1.0
        views.append(v)
    b = Batch(views, (64, 2, 1))
    b.render()
    torch.cuda.synchronize()
    batched = [host_frame(v) for v in views]
    s = torch.cuda.current_stream().cuda_stream
    for v in views:
        v.History.zero_()
        w, h = v.width, v.height
        for y in range(0, h, 64):
            sb.call("stratum_tracePrimary", sb.ptr(v.World), sb.ptr(v.Nodes), sb.ptr(v.Origin), sb.ptr(v.C),
                    sb.ptr(v.Hit), sb.ptr(v.Surface), w, h, y, 64, s)
            sb.call("stratum_shadePixels", sb.ptr(v.World), sb.ptr(v.Origin), sb.ptr(v.C), sb.ptr(v.Hit),
                    sb.ptr(v.Surface), sb.ptr(v.Linear), w, h, y, 64, s)
        sb.call("stratum_resolveFrame", sb.ptr(v.Linear), sb.ptr(v.History), sb.ptr(v.Pixels), sb.ptr(v.C),
                sb.ptr(v.Hit), sb.ptr(v.Surface), w, h, s)
    torch.cuda.synchronize()
    with ol.device_angles(oracle):
        for i, ((w, h), (pos, yaw, pitch), v) in enumerate(zip(sizes, poses, views)):
            o = ol.setup_pose(oracle, 100 + i, pos, yaw, pitch, w, h, origin=(i, 0, 2 * i, 0))
            second = np.zeros(w * h, np.float32)
            want = ol.render(oracle, o, w, h, second=second)
            check(f"{w}x{h} batched", batched[i], want, second)
            check(f"{w}x{h} drop-in", host_frame(v), want, second)
