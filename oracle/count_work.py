"""Algorithmic work of the frame path per shaded ray (test infrastructure).

    python oracle/count_work.py            # prints the per-pose table bench.py carries

The frame path is bound by FP32 instruction issue, so its roofline counts FP32
lane operations.  The count is fixed from the reference algorithm, not from
compiled code: the instrumented CPU oracle counts how often each unit of work
runs for each benchmark pose (lot DDA cells, node tests, feature emissions and
tests, tests past the slab check by shape, leaf-grid cells, masonry-relief
steps, shaded pixels by material class, shadow DDA cells), and each unit
carries a weight = the FP32 operations (add, sub, mul, div, sqrt, min, max,
compare, abs, floor, float<->int, transcendental: 1 each) of the reference
function that performs it, counted from its source:

  unit            weight  reference source
  ray             70      common.cu:63-70 rayDirection + trace.cu:33-45 ground, slab, DDA set-up
  dda             14      trace.cu:47-57 one lot cell (bounds check, lot frame, step)
  node            47      trace.cu:2-7 nodeNear (count test + boxRange with six safeInv + tests)
  group           8       assets.cu:3-8 group prologue, trace.cu:22 sink set-up
  emit            10      sink.cu:10-26 roof rescale test + feature placement arithmetic + accept test
  feat            47      geometry.cu:33-38 localPoint + boxRange + interval test
  pass_box        4       geometry.cu:39,79-80 t select, positivity and relief tests
  pass_ellipsoid  36      geometry.cu:40-43
  pass_cylinder   52      geometry.cu:44-53
  pass_prism      30      geometry.cu:54-64
  pass_arch       72      geometry.cu:65-74
  foliage         40      geometry.cu:17-29 one leaf-grid cell
  masonry         95      geometry.cu:87 one relief step (masonryHeight, common.cu:79-87)
  hit             45      geometry.cu:92-114 featureNormal + turnWorld of the winner
  sky             200     materials.cu:11-16 sky with cloud fbm, per sky pixel
  shade           420     shade.cu:45-102 without surfaceColor: sky, haze, fog, GGX, 3x3 ambient
  shade_masonry   1150    materials.cu:3-10,34-61 + shade.cu:68-75 brick/stone albedo and relief normal
  sdda            50      shade.cu:9-20 one shadow DDA cell (lot + slab test)
  resolve         60      shade.cu:104-123 per pixel (mean, vignette, ACES, gamma, pack)
  resolve_tap     40      shade.cu:111-113 one contact-occlusion tap (8 per pixel nearer than 250 m)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "tests"))

WEIGHTS = {"ray": 70, "dda": 14, "node": 47, "group": 8, "emit": 10, "feat": 47, "pass_box": 4,
           "pass_ellipsoid": 36, "pass_cylinder": 52, "pass_prism": 30, "pass_arch": 72, "foliage": 40,
           "masonry": 95, "hit": 45, "sky": 200, "shade": 420, "shade_masonry": 1150, "sdda": 50, "resolve": 60,
           "resolve_tap": 40}

# Oracle counter index of each unit (oracle/stratum_oracle.h).
INDEX = {"ray": 0, "dda": 1, "node": 2, "group": 3, "feat": 4, "foliage": 5, "masonry": 6, "sdda": 7, "shade": 8,
         "shade_masonry": 9, "pass_box": 10, "pass_ellipsoid": 11, "pass_cylinder": 12, "pass_prism": 13,
         "pass_arch": 14}


def count_pose(lib, pose, width=1600, height=900, row_stride=4, seed=0x5EED):
    import oracle_lib as ol
    s = ol.setup_pose(lib, seed, pose["pos"], pose["yaw"], pose["pitch"], width, height, origin=pose["origin"])
    cn = np.zeros(32, np.int64)
    P = width * height
    hit = np.zeros(P * 4, np.float32)
    surf = np.zeros(P * 4, np.float32)
    lin = np.zeros(P * 4, np.float32)
    for y in range(0, height, row_stride):
        lib.trace(s.World, s.Nodes, s.Origin, s.C, hit, surf, width, height, row0=y, rows=1, counters=cn)
        lib.shade(s.World, s.Origin, s.C, hit, surf, lin, width, height, row0=y, rows=1, counters=cn)
    rays = cn[0]
    units = {k: int(cn[i]) for k, i in INDEX.items()}
    units["emit"] = units["feat"]
    h = hit.reshape(-1, 4)[::1]
    rows = np.zeros(height, bool)
    rows[::row_stride] = True
    h = hit.reshape(height, width, 4)[rows].reshape(-1, 4)
    units["hit"] = int((h[:, 1] >= 0).sum())
    units["sky"] = int((h[:, 1] == -10000).sum())
    units["resolve"] = int(rays)
    units["resolve_tap"] = int(8 * ((h[:, 1] != -10000) & (h[:, 0] < 250.0)).sum())
    ops = sum(WEIGHTS[k] * units[k] for k in WEIGHTS)
    return {"rays": int(rays), "ops_per_ray": ops / rays, "per_ray": {k: units[k] / rays for k in WEIGHTS},
            "trace_ops_per_ray": sum(WEIGHTS[k] * units[k] for k in WEIGHTS
                                     if k not in ("sky", "shade", "shade_masonry", "sdda", "resolve", "resolve_tap"))
            / rays}


def main():
    import oracle_lib as ol
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    from bench import POSES
    lib = ol.Oracle()
    out = {name: count_pose(lib, p) for name, p in POSES.items()}
    for k, v in out.items():
        print(f"{k:10s} ops/ray {v['ops_per_ray']:9.1f}  trace ops/ray {v['trace_ops_per_ray']:9.1f}  "
              + " ".join(f"{u}={x:.2f}" for u, x in v["per_ray"].items() if x))
    print(json.dumps({k: [round(v["ops_per_ray"], 1), round(v["trace_ops_per_ray"], 1)] for k, v in out.items()}))


if __name__ == "__main__":
    main()
