"""Build libstratum.so (sm_100a) in-tree.

    python -m stratum_hyperdetail_b200.build [--verbose] [--define NAME ...]

Steps: compile and run csrc/gen_tables.cpp (the grammar's trig constants,
evaluated with the host C library) into _build/gen/trig_table.h, compile every
csrc/*.cu and csrc/*.cpp with nvcc for sm_100a, link libstratum.so next to
this file.  All device code is built with --fmad=false: the reference's CPU
build never fuses a multiply and an add, and its results are matched bit for bit.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
GEN = BUILD / "gen"
LIB = PKG / "libstratum.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # The image sets CXX to a compiler without OpenMP; the PATH g++ is the system one.
    return shutil.which("g++") or "g++"


def run(cmd, verbose=False):
    if verbose:
        print(" ".join(map(str, cmd)), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def gen_tables(verbose=False):
    GEN.mkdir(parents=True, exist_ok=True)
    exe = BUILD / "gen_tables"
    run([host_cxx(), "-std=c++17", "-O0", str(CSRC / "gen_tables.cpp"), "-o", str(exe)], verbose)
    out = run([str(exe)], verbose)
    (GEN / "trig_table.h").write_text(out)


def compile_one(src: Path, defines, verbose=False, ptxas_verbose=False) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-I", str(GEN), "-c", str(src), "-o", str(obj)]
    cmd += [f"-D{d}" for d in defines]
    if ptxas_verbose and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    log = run(cmd, verbose)
    return obj, log


def build(verbose=False, defines=(), ptxas_verbose=False, out: Path | None = None) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    gen_tables(verbose)
    sources = sorted(CSRC.glob("*.cu")) + sorted(p for p in CSRC.glob("*.cpp") if p.name != "gen_tables.cpp")
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: compile_one(s, defines, verbose, ptxas_verbose), sources))
    objs = [o for o, _ in results]
    if ptxas_verbose:
        for (o, log) in results:
            if log.strip():
                print(f"== {o.name}\n{log}")
    target = out or LIB
    tmp = target.with_suffix(".so.tmp")
    run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)], verbose)
    os.replace(tmp, target)
    return target


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print registers/spills per kernel")
    ap.add_argument("--define", action="append", default=[])
    ap.add_argument("--out", type=Path, default=None)
    a = ap.parse_args(argv)
    print(build(a.verbose, a.define, a.ptxas, a.out))


if __name__ == "__main__":
    sys.exit(main())
