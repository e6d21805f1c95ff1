"""Regenerate the golden fixtures from the reference itself.

    make -C oracle ref && python tests/golden/make_golden.py

Runs the reference renderer built from its own sources (oracle/_ref: the
reference harness `stratum-native` and its kernels behind ref_driver.cpp) and
writes, next to this file:

  probes.json  the 54 probeGrammar fixtures printed by `stratum-native fixtures`
               (the generator of the reference's tests/probes.json)
  lots.json    64-bit address arithmetic and lot descriptors: offset_tag cases
               around the carry/borrow edges, describe_lot of those tags
  frames.json  per-pose digests (sha256 of the raw little-endian arrays) of the
               table (World, Tags, Nodes) and of Hit, Surface, Linear, History
               and Pixels after one sample, plus hit/sky counts

Floats are stored as their 32-bit patterns so the fixtures are exact.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
from oracle_lib import REF_BIN, RefLib, render, setup_pose  # noqa: E402

SEED = 0x5EED
# name -> (camera position before rebase, yaw, pitch, width, height)
POSES = {
    "config1_320x180": ((32.0, 1.7, 32.0), 0.7853981633974483, 0.0, 320, 180),
    "street_160x90": ((14.0, 1.7, 14.0), 0.0, 0.0, 160, 90),
    "rooftop_160x90": ((14.0, 40.0, 14.0), 1.5707963267948966, 0.0, 160, 90),
    "aerial_160x90": ((14.0, 300.0, 14.0), 0.6, -0.5235987755982988, 160, 90),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def bits(a) -> list[int]:
    return [int(x) for x in np.asarray(a, np.float32).view(np.uint32)]


def main():
    ref = RefLib()
    # probes.json from the reference harness itself
    out = subprocess.run([str(REF_BIN), "fixtures"], check=True, capture_output=True, text=True).stdout
    (HERE / "probes.json").write_text(json.dumps(json.loads(out)) + "\n")

    cases = []
    origins = [(0, 0, 0, 0), (0xFFFFFFF0, 37, 9, 0), (0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF),
               (5, 0, 0xFFFFFFC0, 7), (0x80000000, 0x7FFFFFFF, 123456, 0x80000000)]
    offsets = [(0, 0), (-1, -1), (32, 0), (-64, 63), (17, -40), (-1, 64), (1, 1)]
    for o in origins:
        for dx, dz in offsets:
            tag = ref.offset_tag(np.array(o, np.uint32), dx, dz)
            lot = ref.describe_lot(tag, 1788)
            cases.append({"origin": list(o), "dx": dx, "dz": dz, "tag": [int(t) for t in tag], "seed": 1788,
                          "lot_bits": bits(lot)})
    rng = np.random.default_rng(7)
    for _ in range(32):
        tag = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        seed = int(rng.integers(0, 10000))
        cases.append({"origin": None, "tag": [int(t) for t in tag], "seed": seed,
                      "lot_bits": bits(ref.describe_lot(tag, seed))})
    (HERE / "lots.json").write_text(json.dumps(cases) + "\n")

    frames = {}
    for name, (pos, yaw, pitch, w, h) in POSES.items():
        s = setup_pose(ref, SEED, pos, yaw, pitch, w, h)
        f = render(ref, s, w, h)
        fid = f["Hit"][1::4]
        frames[name] = {
            "seed": SEED, "pos": pos, "yaw": yaw, "pitch": pitch, "width": w, "height": h,
            "C_bits": bits(s.C), "origin": [int(x) for x in s.Origin],
            "World": digest(s.World), "Tags": digest(s.Tags), "Nodes": digest(s.Nodes),
            "Hit": digest(f["Hit"]), "Surface": digest(f["Surface"]), "Linear": digest(f["Linear"]),
            "History": digest(f["History"]), "Pixels": digest(f["Pixels"]),
            "sky": int((fid == -10000).sum()), "ground": int((fid == -1).sum()), "features": int((fid >= 0).sum()),
        }
    (HERE / "frames.json").write_text(json.dumps(frames, indent=1) + "\n")
    print("wrote", [p.name for p in HERE.glob("*.json")])


if __name__ == "__main__":
    main()
