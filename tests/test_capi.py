"""The C-ABI library loads and exports exactly what include/stratum.h declares.

No compute calls: this runs without a GPU.  Argument checks that return before
any CUDA call are exercised (they must not touch the device).
"""
import ctypes as ct
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "stratum.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(stratum_\w+)\s*\(", text)))


def test_header_declares_reference_entry_points():
    names = declared_symbols()
    for ref_name in ("initCamera", "stepCamera", "clearQueue", "prepareLots", "planBounds", "buildGroupBounds",
                     "reduceGroupBounds", "tracePrimary", "shadePixels", "resolveFrame", "probeGrammar"):
        assert f"stratum_{ref_name}" in names
    for alias in ("initWorld", "schedulePages", "commitPages", "buildBVH", "frame"):
        assert f"stratum_{alias}" in names


def test_library_exports_every_declared_symbol():
    import stratum_hyperdetail_b200 as sb
    L = sb.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    assert b"sm_100a" in L.stratum_version()


def test_python_signatures_cover_header():
    import stratum_hyperdetail_b200 as sb
    # the three non-status functions are typed separately in lib(); the server's in server.py
    names = {n for n in declared_symbols() if not n.startswith("stratum_server_")}
    assert names - {"stratum_version", "stratum_batchScratchBytes", "stratum_groupCacheBytes"} <= set(sb.SIGNATURES)
    from stratum_hyperdetail_b200 import server
    L = server._lib()
    for n in declared_symbols():
        if n.startswith("stratum_server_"):
            assert getattr(L, n).argtypes is not None, n


def test_bad_arguments_are_rejected_before_launch():
    import stratum_hyperdetail_b200 as sb
    L = sb.lib()
    assert L.stratum_initCamera(None, None, 1, None) == sb.EINVAL
    assert L.stratum_tracePrimary(None, None, None, None, None, None, 320, 180, 0, 64, None) == sb.EINVAL
    assert L.stratum_reduceGroupBounds(ct.c_void_p(16), ct.c_void_p(16), 3, 0, None) == sb.EINVAL
    assert L.stratum_resolveFrame(None, None, None, None, None, None, -1, 5, None) == sb.EINVAL
    assert L.stratum_enumerateGroups(None, None, 1, 65, None, None, None) == sb.EINVAL
    # tunes outside the accepted set (block size 64/128/256, queue depth 1..16,
    # order 0..3: tile order in bit 0, the block-pooled trace in bit 1)
    fake = ct.c_void_p(256)
    for bad in ((128, 1, 4), (96, 1, 0), (128, 0, 0), (128, 17, 1), (64, 1, -1)):
        t = sb.Tune(*bad)
        assert L.stratum_renderViews(fake, 1, fake, 1 << 30, ct.byref(t), None) == sb.EINVAL, bad


def test_abi_constants_match_reference():
    # kernels/common.cu:2-16 == src/engine.js:2 of the reference
    text = (ROOT / "include" / "stratum.h").read_text()
    want = {"WORLD_SIDE": 128, "WORLD_LOTS": 16384, "LOT_FLOATS": 16, "CLUSTERS": 64, "GROUP_NODES": 128,
            "MAX_FEATURES": 64, "BUILD_CHUNK": 2048, "BUILD_CHUNKS": 8, "RAY_DISTANCE": 2000}
    for k, v in want.items():
        assert re.search(rf"#define STRATUM_{k} {v}\b", text), k
    assert want["GROUP_NODES"] == 2 * want["CLUSTERS"]
    assert want["RAY_DISTANCE"] < (want["WORLD_SIDE"] / 2 - 2) * 36


def test_engine_fails_loudly_without_gpu():
    import torch
    import stratum_hyperdetail_b200 as sb
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError):
        sb.Engine().init(320, 180)


def test_group_cache_sizes():
    """Group cache buffer = 256 B header + 16,384 x 64 directory words + entries
    of 2,192 B (64 B tag, 56 records of 32 B, 14 run boxes of 24 B)."""
    import stratum_hyperdetail_b200 as sb
    L = sb.lib()
    base = 256 + 16384 * 64 * 4
    assert L.stratum_groupCacheBytes(0) == base
    assert L.stratum_groupCacheBytes(1) == base + 2192
    assert L.stratum_groupCacheBytes(sb.GROUP_CACHE_ENTRIES) == base + 2192 * sb.GROUP_CACHE_ENTRIES
    assert L.stratum_groupCacheBytes(-1) == 0
    assert L.stratum_groupCacheInit(None, 16, None) == sb.EINVAL
    assert L.stratum_groupCacheInit(ct.c_void_p(256), 1 << 24, None) == sb.EINVAL  # above the 24-bit entry index
