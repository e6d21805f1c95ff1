"""Pin the CPU oracle (oracle/stratum_oracle.cpp) to the reference.

Against the committed golden fixtures (made from the reference itself by
tests/golden/make_golden.py) and, where the reference build oracle/_ref is
present, directly against the reference's kernels on fresh random inputs.
Everything here is bit-exact.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import render, setup_pose

GOLDEN = Path(__file__).resolve().parent / "golden"


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def test_probe_fixtures_exact(oracle):
    fixtures = json.loads((GOLDEN / "probes.json").read_text())
    assert len(fixtures) == 54
    for f in fixtures:
        got = oracle.probe(np.array(f["input"], np.float32))
        want = np.array(f["expected"], np.float32)
        # the harness prints with 6 significant digits (std::cout default)
        assert np.allclose(got, want, rtol=1e-5, atol=1e-4), (f["input"], got, want)


def test_address_and_descriptor_vectors_exact(oracle):
    for c in json.loads((GOLDEN / "lots.json").read_text()):
        if c["origin"] is not None:
            tag = oracle.offset_tag(np.array(c["origin"], np.uint32), c["dx"], c["dz"])
            assert [int(t) for t in tag] == c["tag"], c
        lot = oracle.describe_lot(np.array(c["tag"], np.uint32), c["seed"])
        assert [int(b) for b in lot.view(np.uint32)] == c["lot_bits"], c


def test_carry_borrow_known_answers(oracle):
    # tests/native_harness.cpp:86-87 of the reference
    a = oracle.offset_tag(np.zeros(4, np.uint32), -1, -1)
    assert a[0] == 0xFFFFFFFF and a[1] == 0xFFFFFFFF and a[3] == 0xFFFFFFFF
    b = oracle.offset_tag(np.array([0xFFFFFFF0, 37, 9, 0], np.uint32), 32, 0)
    assert b[0] == 16 and b[1] == 38


@pytest.mark.parametrize("name", ["config1_320x180", "street_160x90", "rooftop_160x90", "aerial_160x90"])
def test_frame_digests_exact(oracle, name):
    g = json.loads((GOLDEN / "frames.json").read_text())[name]
    s = setup_pose(oracle, g["seed"], g["pos"], g["yaw"], g["pitch"], g["width"], g["height"])
    assert [int(b) for b in s.C.view(np.uint32)] == g["C_bits"]
    assert [int(x) for x in s.Origin] == g["origin"]
    for k in ("World", "Tags", "Nodes"):
        assert digest(getattr(s, k)) == g[k], k
    f = render(oracle, s, g["width"], g["height"])
    for k in ("Hit", "Surface", "Linear", "History", "Pixels"):
        assert digest(f[k]) == g[k], k


def test_grammar_and_bounds_match_reference(oracle, ref):
    rng = np.random.default_rng(11)
    for _ in range(40):
        tag = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        seed = int(rng.integers(0, 100000))
        lot = oracle.describe_lot(tag, seed)
        assert np.array_equal(lot.view(np.uint32), ref.describe_lot(tag, seed).view(np.uint32))
        for ty in range(6):  # every lot family
            l2 = lot.copy()
            l2[3] = ty
            for g in range(64):
                a, b = oracle.enumerate(l2, g), ref.enumerate(l2, g)
                assert a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32)), (ty, g)
                assert np.array_equal(oracle.group_bounds(l2, g), ref.group_bounds(l2, g))


def test_feature_hit_matches_reference(oracle, ref):
    rng = np.random.default_rng(5)
    lot = oracle.describe_lot(np.array([3, 0, 9, 0], np.uint32), 1788)
    feats = []
    for ty in (0, 1, 2, 3, 4):
        l2 = lot.copy()
        l2[3] = ty
        for g in range(64):
            feats.extend(oracle.enumerate(l2, g))
    feats = np.array(feats)
    for i in rng.choice(len(feats), 400, replace=False):
        f = feats[i]
        for _ in range(4):
            ro = (f[:3] + rng.normal(0, 6, 3)).astype(np.float32)
            rd = (f[:3] + rng.normal(0, 0.5, 3) - ro).astype(np.float32)
            rd /= np.linalg.norm(rd)
            cone = float(rng.choice([0.0, 0.0012, 0.006]))
            a, b = oracle.feature_hit(f, ro, rd, cone), ref.feature_hit(f, ro, rd, cone)
            assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32), (f, ro, rd, a, b)
            if a < 2000:
                pt = ro + rd * np.float32(a)
                assert np.array_equal(oracle.feature_normal(f, pt), ref.feature_normal(f, pt))


def test_hierarchy_vs_exhaustive(oracle):
    """tests/native_harness.cpp:68-79 of the reference, on the oracle: the
    culled hierarchy query equals the exhaustive minimum over all features."""
    from oracle_lib import GROUP_NODES
    rays = hits = 0
    worst = 0.0
    for v in range(24):
        tag = oracle.offset_tag(np.zeros(4, np.uint32), v * 71 - 830, v * 39 - 191)
        lot = oracle.describe_lot(tag, 1788)
        if v < 6:
            lot[3] = v
        queue = np.array([1, 0] + [0] * 16383, np.uint32)
        world = np.zeros(16384 * 16, np.float32)
        world[:16] = lot
        nodes = np.zeros(16384 * GROUP_NODES * 8, np.float32)
        oracle.build_bounds(queue, world, nodes, 1)
        blk = nodes[:GROUP_NODES * 8].copy()
        for i in range(96):
            a = (i * 111 + v) % 628 / 100.0
            ro = np.array([np.cos(a) * 27, (i * 7 + v) % 65 - 0.1, np.sin(a) * 27], np.float32)
            target = np.array([(i * 17) % 18 - 9, ((i * 59) % 100) / 100 * lot[2], (i * 83) % 18 - 9], np.float32)
            rd = (target - ro).astype(np.float32)
            rd /= np.float32(np.linalg.norm(rd))
            t1, f1, _ = oracle.query_lot(lot, blk, ro, rd)
            t2, f2, _ = oracle.query_lot_exhaustive(lot, ro, rd)
            worst = max(worst, abs(t1 - t2))
            rays += 1
            hits += f1 >= 0
    assert worst == 0.0 and hits > 1000, (worst, hits, rays)
