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


@pytest.mark.parametrize("tune", [(128, 1, 1), (64, 2, 0), (256, 4, 1), (128, 16, 0), (64, 1, 3), (128, 1, 2), (256, 1, 3)])
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


def cache_header(v):
    """(next, capacity, resets, fills) of a view's group cache."""
    return tuple(int(x) for x in v.Groups[:4].cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("entries", [0, 4, 65536])
def test_group_cache_size_does_not_change_results(cuda, entries):
    """No cache, a 4-group cache (full at once: most groups built by the
    grammar, emptied every 8 frames) and the default cache give the plain
    path's bits over 10 frames."""
    from stratum_hyperdetail_b200.batch import Batch
    want = plain_frames(10)
    views = make_views()
    b = Batch(views, (128, 1, 1), group_cache=entries)
    for f in range(10):
        b.frame()
        torch.cuda.synchronize()
        for i, v in enumerate(views):
            assert_same(snapshot(v), want[f][i], f"cache {entries} frame {f} view {i}")
    for v in views:
        if entries == 0:
            assert v.Groups is None
            continue
        nxt, cap, resets, fills = cache_header(v)
        assert cap == entries and fills > 0
        if entries == 4:
            assert resets == 1  # full from the first frame, emptied at the 8th
        else:
            assert resets == 0 and nxt == fills  # everything fits; no group filled twice per slot change


def test_group_cache_survives_a_table_moved_by_the_drop_in_path(cuda):
    """A warm cache whose table is then re-described by the single-view entry
    points (set_pose at another address) must not serve stale groups."""
    from stratum_hyperdetail_b200.batch import Batch
    views = make_views()
    b = Batch(views, (128, 1, 1))
    b.frame()
    torch.cuda.synchronize()
    # same seeds (the table is keyed by address), origins moved by a few lots:
    # some slots keep their lots and cached groups, the others are re-described
    moved = [(s, [o[0] + 3, o[1], o[2] ^ 5, o[3]], p, y, t, w, h) for s, o, p, y, t, w, h in VIEWS]
    from stratum_hyperdetail_b200.views import View
    fresh = []
    for v, (seed, origin, pos, yaw, pitch, w, h) in zip(views, moved):
        v.set_pose(seed, origin, pos, yaw, pitch)
        v.History.zero_()
        f = View(w, h)
        f.set_pose(seed, origin, pos, yaw, pitch)
        fresh.append(f)
    b.frame()
    for f in fresh:
        f.frame(0.0)
    torch.cuda.synchronize()
    for i, (v, f) in enumerate(zip(views, fresh)):
        for k in ("Hit", "Surface", "Linear", "Pixels"):
            assert torch.equal(getattr(v, k), getattr(f, k)), f"view {i} {k} differs after the move"


def test_random_views_equal_plain(cuda):
    """Twelve random views (widths 64-160, altitude 1.5-300 m, any yaw, pitch
    -45..10 deg, random 64-bit addresses and seeds) over five frames: the
    batched path with its group cache equals the single-view path bit for bit.
    Distant, grazing and high views exercise the culling of staged records."""
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    rng = np.random.Generator(np.random.Philox(11))
    specs = []
    for _ in range(12):
        w = int(rng.integers(64, 161))
        specs.append((int(rng.integers(0, 1 << 24)), [int(x) for x in rng.integers(0, 2**32, 4, dtype=np.uint64)],
                      (float(rng.uniform(-18, 18)), float(rng.uniform(1.5, 300)), float(rng.uniform(-18, 18))),
                      float(rng.uniform(0, 2 * np.pi)), float(np.radians(rng.uniform(-45, 10))), w, (w * 9) // 16))

    def views():
        out = []
        for seed, origin, pos, yaw, pitch, w, h in specs:
            v = View(w, h)
            v.set_pose(seed, origin, pos, yaw, pitch)
            out.append(v)
        return out
    plain, batched = views(), views()
    b = Batch(batched, (128, 1, 1))
    for f in range(5):
        for v in plain:
            v.frame(0.0)
        b.frame()
        torch.cuda.synchronize()
        for i, (p, q) in enumerate(zip(plain, batched)):
            for k in ("Hit", "Surface", "Linear", "History", "Pixels"):
                assert torch.equal(getattr(p, k), getattr(q, k)), f"frame {f} view {i}: {k} differs"


def test_tiny_and_ragged_views_equal_plain(cuda):
    """Views smaller than one 8x4 tile or with ragged edges (1x1, 7x3, 8x4,
    9x5, 33x17) mixed in one batch: every pixel equals the single-view path."""
    from stratum_hyperdetail_b200.batch import Batch
    from stratum_hyperdetail_b200.views import View
    sizes = [(1, 1), (7, 3), (8, 4), (9, 5), (33, 17)]

    def views():
        out = []
        for i, (w, h) in enumerate(sizes):
            v = View(w, h)
            v.set_pose(100 + i, [i, 0, 2 * i, 0], (3.0 * i, 1.7 + 10 * i, -2.0), 0.4 * i, -0.1 * i)
            out.append(v)
        return out
    plain, batched = views(), views()
    b = Batch(batched, (64, 2, 1))
    for f in range(3):
        for v in plain:
            v.frame(0.0)
        b.frame()
        torch.cuda.synchronize()
        for i, (p, q) in enumerate(zip(plain, batched)):
            for k in ("Hit", "Surface", "Linear", "History", "Pixels"):
                assert torch.equal(getattr(p, k), getattr(q, k)), f"frame {f} view {sizes[i]}: {k} differs"
