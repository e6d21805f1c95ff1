"""The allocation-free batched entry point (stratum_renderViewsNoAlloc).

It exists for callers that cannot give the library device memory: an
embedding whose own pool owns all of HBM, a binding with no device allocator,
or a frame loop that must not allocate.  It renders from the library's static
scratch array instead of a caller buffer.  Here it must give exactly the
frames of stratum_renderViews (the batched path is bit-exact against the
single-view path, so the tolerance is zero), on two calls in a row.

This file sorts last so that a run stopping at its first failure has already
run every other test; it also passes alone in a fresh process (its first call
on the device performs the one-time address look-up, outside any capture).
"""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# (seed, origin, pos, yaw, pitch, width, height)
VIEWS = [
    (0x5EED, [0, 0, 0, 0], (32.0, 1.7, 32.0), np.pi / 4, 0.0, 256, 144),
    (1788, [0xFFFFFFF0, 5, 3, 0xFFFFFFFF], (14.0, 40.0, 14.0), 1.2, -0.2, 173, 97),
    (99, [1, 0, 8, 0], (0.0, 2.0, -16.0), 0.0, 0.0, 120, 68),
]
BUFFERS = ("C", "Hit", "Surface", "Linear", "History", "Pixels")


def make_batch():
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    views = []
    for seed, origin, pos, yaw, pitch, w, h in VIEWS:
        v = View(w, h)
        v.set_pose(seed, origin, pos, yaw, pitch)
        views.append(v)
    return Batch(views)


def test_no_alloc_matches_scratch_entry_point_on_two_calls(cuda):
    import stratum_hyperdetail_b200 as sb
    ref, noalloc = make_batch(), make_batch()
    s = torch.cuda.current_stream().cuda_stream
    for call_index in range(2):
        for b in (ref, noalloc):
            sb.call("stratum_stepViews", sb.ptr(b.table), b.n, s)
            b.refresh()
        ref.render()
        noalloc.render_no_alloc()
        torch.cuda.synchronize()
        for i, (a, b) in enumerate(zip(ref.views, noalloc.views)):
            for k in BUFFERS:
                assert torch.equal(getattr(a, k), getattr(b, k)), f"call {call_index}: view {i} {k} differs"


def test_no_alloc_rejects_more_views_than_its_static_scratch_holds(cuda):
    import stratum_hyperdetail_b200 as sb
    b = make_batch()
    status = sb.lib().stratum_renderViewsNoAlloc(sb.ptr(b.table), sb.NOALLOC_MAX_VIEWS + 1, None,
                                                 torch.cuda.current_stream().cuda_stream)
    assert status == sb.ELIMIT
