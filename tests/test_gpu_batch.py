"""Batched multi-view path: each view's result in a batch equals rendering it
alone through the single-view entry points (bit-exact), for every tune, in
eager mode and under CUDA-graph replay."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# (seed, origin, pos, yaw, pitch, width, height)
VIEWS = [
    (0x5EED, [0, 0, 0, 0], (32.0, 1.7, 32.0), np.pi / 4, 0.0, 320, 180),
    (1788, [0xFFFFFFF0, 5, 3, 0xFFFFFFFF], (14.0, 40.0, 14.0), 1.2, -0.2, 200, 113),
    (7, [28, 0, 1, 0], (0.0, 0.5, 0.0), 0.0, 0.0, 131, 77),
    (424242, [1, 0, 8, 0], (0.0, 300.0, -16.0), 2.5, -0.6, 97, 55),
]


def make_views():
    from stratum_hyperdetail_b200.views import View
    out = []
    for seed, origin, pos, yaw, pitch, w, h in VIEWS:
        v = View(w, h)
        v.set_pose(seed, origin, pos, yaw, pitch)
        out.append(v)
    torch.cuda.synchronize()
    return out


def snapshot(v):
    return {k: getattr(v, k).clone() for k in ("C", "Origin", "World", "Tags", "Nodes", "Hit", "Surface", "Linear",
                                             "History", "Pixels")}


def assert_same(a, b, what):
    for k in a:
        assert torch.equal(a[k], b[k]), f"{what}: {k} differs"


def plain_frames(frames):
    views = make_views()
    out = []
    for _ in range(frames):
        for v in views:
            v.frame(0.0)
        torch.cuda.synchronize()
        out.append([snapshot(v) for v in views])
    return out


@pytest.mark.parametrize("tune", [(128, 1, 1), (64, 2, 0), (256, 4, 1), (128, 16, 0)])
def test_batch_equals_plain(cuda, tune):
    from stratum_hyperdetail_b200.batch import Batch
    want = plain_frames(2)
    views = make_views()
    b = Batch(views, tune)
    for f in range(2):
        b.frame()
        torch.cuda.synchronize()
        for i, v in enumerate(views):
            assert_same(snapshot(v), want[f][i], f"tune {tune} frame {f} view {i}")


def test_graph_replay_equals_eager(cuda):
    from stratum_hyperdetail_b200.batch import Batch
    want = plain_frames(3)
    views = make_views()
    b = Batch(views)
    b.frame()  # eager frame 0 (initialises launch parameters)
    torch.cuda.synchronize()
    for i, v in enumerate(views):
        assert_same(snapshot(v), want[0][i], f"eager view {i}")
    b.capture()  # capturing runs nothing
    for f in (1, 2):
        b.replay()
        torch.cuda.synchronize()
        for i, v in enumerate(views):
            assert_same(snapshot(v), want[f][i], f"replay {f} view {i}")


def test_autotune_picks_a_valid_tune_and_keeps_state(cuda):
    from stratum_hyperdetail_b200.batch import Batch
    views = make_views()
    b = Batch(views)
    b.frame()
    torch.cuda.synchronize()
    before = [v.History.clone() for v in views]
    ms = b.autotune()
    assert ms > 0
    assert b.tune.threads in (64, 128, 256) and 1 <= b.tune.grab <= 16 and b.tune.order in (0, 1)
    for v, h in zip(views, before):
        assert torch.equal(v.History, h)
    # the queues reset themselves: a frame after tuning still covers every pixel
    want = plain_frames(2)[1]
    b.frame()
    torch.cuda.synchronize()
    for i, v in enumerate(views):
        assert_same(snapshot(v), want[i], f"after autotune view {i}")
