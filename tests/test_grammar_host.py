"""The device grammar, compiled for the host, against the oracle (CPU only).

Both forms of the CUDA feature grammar -- the sequential emitter (grammar.cuh)
and the random-access form (grammar_ra.cuh, feature #i computed directly) --
must reproduce the oracle's enumeration bit for bit for every lot family,
floor count and group, including out-of-range floors and groups.
"""
import ctypes as ct
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "stratum_hyperdetail_b200" / "csrc"
GEN = ROOT / "stratum_hyperdetail_b200" / "_build" / "gen"
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def hg(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    if not (GEN / "trig_table.h").exists():
        from stratum_hyperdetail_b200 import build
        build.gen_tables()
    out = tmp_path_factory.mktemp("hg") / "libhg.so"
    subprocess.run([nvcc, "-x", "cu", "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler",
                    "-ffp-contract=off", "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(CSRC), "-I", str(GEN),
                    str(ROOT / "tests" / "host_grammar.cu"), "-o", str(out)], check=True)
    lib = ct.CDLL(str(out))
    for n in ("hg_sequential", "hg_random_access"):
        getattr(lib, n).argtypes = [f32p, ct.c_int, f32p, ct.c_int]
        getattr(lib, n).restype = ct.c_int
    return lib


def run(fn, lot, g):
    out = np.zeros((64, 10), np.float32)
    n = fn(np.ascontiguousarray(lot, np.float32), g, out, 64)
    return out[:min(n, 64)].copy(), n


def test_sequential_and_random_access_match_oracle(hg, oracle):
    rng = np.random.default_rng(21)
    checked = 0
    for t in range(60):
        tag = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        base = oracle.describe_lot(tag, int(rng.integers(0, 60000)))
        for ty in range(6):
            for floors in ([-1, 0, 1, 2, 3, 4, 5, 6, 7] if t < 3 else [int(base[5])]):
                lot = base.copy()
                lot[3] = ty
                lot[5] = floors
                for g in range(-1, 65):
                    want = oracle.enumerate(lot, g)
                    seq, n1 = run(hg.hg_sequential, lot, g)
                    ra, n2 = run(hg.hg_random_access, lot, g)
                    assert n1 == len(want) == n2, (ty, floors, g, n1, n2, len(want))
                    assert np.array_equal(seq.view(np.uint32), want.view(np.uint32)), (ty, floors, g)
                    assert np.array_equal(ra.view(np.uint32), want.view(np.uint32)), (ty, floors, g)
                    checked += len(want)
    assert checked > 500_000
