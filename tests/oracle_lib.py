"""ctypes access to the CPU oracle (test infrastructure).

`Oracle` wraps oracle/_build/liboracle.so, this repository's CPU restatement
of the reference frame path.  `RefLib` wraps oracle/_ref/libstratum_ref.so,
the reference's own kernels compiled from its sources (present only where the
reference tree was available when `make -C oracle ref` ran).  Both expose the
same numpy-level calls so a test can run either side of a comparison.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_SO = ORACLE_DIR / "_build" / "liboracle.so"
REF_SO = ORACLE_DIR / "_ref" / "libstratum_ref.so"
REF_BIN = ORACLE_DIR / "_ref" / "stratum-native"

WORLD_LOTS = 16384
LOT_FLOATS = 16
GROUP_NODES = 128
CLUSTERS = 64
FAR = 2000.0

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build_oracle() -> Path:
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < (ORACLE_DIR / "stratum_oracle.cpp").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return ORACLE_SO


def _opt(p):
    return None if p is None else p


class _Lib:
    prefix = ""

    def __init__(self, path: Path):
        self.lib = ct.CDLL(str(path))
        p = self.prefix
        L = self.lib
        sig = {
            "offset_tag": (None, [u32p, ct.c_int, ct.c_int, u32p]),
            "describe_lot": (None, [u32p, ct.c_int, f32p]),
            "initCamera": (None, [f32p, u32p, ct.c_int]),
            "stepCamera": (None, [f32p, u32p, f32p, ct.c_float, ct.c_int, ct.c_int]),
            "clearQueue": (None, [u32p]),
            "prepareLots": (None, [u32p, f32p, f32p, u32p, u32p]),
            "planBounds": (None, [u32p, u32p]),
            "probeGrammar": (None, [f32p, f32p]),
            "enumerate": (ct.c_int, [f32p, ct.c_int, f32p, ct.c_int]),
            "group_bounds": (None, [f32p, ct.c_int, f32p]),
            "featureHit": (ct.c_float, [f32p, f32p, f32p, ct.c_float]),
            "featureNormal": (None, [f32p, f32p, f32p]),
            "queryLot": (ct.c_float, [f32p, f32p, f32p, f32p, ct.c_float, ct.c_float, ct.POINTER(ct.c_int), f32p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, p + name)
            fn.restype = res
            fn.argtypes = args
        self.hashfn = getattr(L, p + ("hashU"))
        self.hashfn.restype = ct.c_uint32
        self.hashfn.argtypes = [ct.c_uint32]
        rr = getattr(L, p + "renderRows")
        rr.restype = None
        rr.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p, f32p, f32p, u32p, ct.c_int, ct.c_int, i32p, ct.c_int,
                       ct.c_int]
        self.taghash = getattr(L, p + "tag_hash")
        self.taghash.restype = ct.c_uint32
        self.taghash.argtypes = [u32p, ct.c_int]

    def f(self, name):
        return getattr(self.lib, self.prefix + name)

    def render_rows(self, s, bufs, width, height, rows, nthreads=0):
        """trace + shade + resolve of the listed rows of a frame (timing samples)."""
        hit, surf, lin, hist, px = bufs
        self.f("renderRows")(s.World, s.Nodes, s.Origin, s.C, hit, surf, lin, hist, px, int(width), int(height),
                             np.ascontiguousarray(rows, np.int32), len(rows), nthreads)

    # -- world -------------------------------------------------------------
    def offset_tag(self, origin, dx, dz):
        out = np.zeros(4, np.uint32)
        self.f("offset_tag")(np.ascontiguousarray(origin, np.uint32), int(dx), int(dz), out)
        return out

    def describe_lot(self, tag, seed):
        out = np.zeros(16, np.float32)
        self.f("describe_lot")(np.ascontiguousarray(tag, np.uint32), int(seed), out)
        return out

    def enumerate(self, lot16, group):
        out = np.zeros((64, 10), np.float32)
        n = self.f("enumerate")(np.ascontiguousarray(lot16, np.float32), int(group), out, 64)
        return out[:n].copy()

    def group_bounds(self, lot16, group):
        out = np.zeros(7, np.float32)
        self.f("group_bounds")(np.ascontiguousarray(lot16, np.float32), int(group), out)
        return out

    def feature_hit(self, f10, ro, rd, cone=0.0):
        return self.f("featureHit")(np.ascontiguousarray(f10, np.float32), np.ascontiguousarray(ro, np.float32),
                                    np.ascontiguousarray(rd, np.float32), float(cone))

    def feature_normal(self, f10, pt):
        out = np.zeros(3, np.float32)
        self.f("featureNormal")(np.ascontiguousarray(f10, np.float32), np.ascontiguousarray(pt, np.float32), out)
        return out

    def query_lot(self, lot16, nodes128, ro, rd, best=FAR, cone=0.0):
        fid = ct.c_int(0)
        f10 = np.zeros(10, np.float32)
        t = self.f("queryLot")(np.ascontiguousarray(lot16, np.float32), np.ascontiguousarray(nodes128, np.float32),
                               np.ascontiguousarray(ro, np.float32), np.ascontiguousarray(rd, np.float32),
                               float(best), float(cone), ct.byref(fid), f10)
        return t, fid.value, f10

    def probe(self, inputs17):
        out = np.zeros(16, np.float32)
        self.f("probeGrammar")(np.ascontiguousarray(inputs17, np.float32), out)
        return out


class Oracle(_Lib):
    prefix = "orc_"

    def __init__(self, path: Path | None = None):
        super().__init__(path or build_oracle())
        L = self.lib
        L.orc_buildBounds.argtypes = [u32p, f32p, f32p, ct.c_int]
        L.orc_tracePrimary.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p, ct.c_int, ct.c_int, ct.c_int, ct.c_int,
                                       ct.c_int, ct.c_void_p, ct.c_void_p]
        L.orc_shadePixels.argtypes = [f32p, u32p, f32p, f32p, f32p, f32p, ct.c_int, ct.c_int, ct.c_int, ct.c_int,
                                      ct.c_int, ct.c_void_p]
        L.orc_resolveFrame.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p, ct.c_int, ct.c_int, ct.c_int]
        L.orc_resolveRows.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p] + [ct.c_int] * 5
        L.orc_traceRays.argtypes = [f32p, f32p, u32p, f32p, ct.c_int, ct.c_int, f32p, ct.c_int]
        L.orc_featureHit_f64.restype = ct.c_double
        L.orc_featureHit_f64.argtypes = [f32p, f64p, f64p, ct.c_double]
        L.orc_featureNormal_f64.argtypes = [f32p, f64p, f64p]
        L.orc_queryLot_exhaustive.restype = ct.c_float
        L.orc_queryLot_exhaustive.argtypes = [f32p, f32p, f32p, ct.c_float, ct.c_float, ct.POINTER(ct.c_int), f32p]
        L.orc_initNeural.argtypes = [f32p, f32p, f32p, f32p, ct.c_int]
        L.orc_materialStep.argtypes = [f32p, u32p, f32p, f32p, f32p, f32p, f32p, f32p, f32p, ct.c_void_p, ct.c_int,
                                       ct.c_int]
        L.orc_predictSubstrate.argtypes = [f32p, f32p, ct.c_int, f32p]
        L.orc_shadePixelsNeural.argtypes = [f32p, u32p, f32p, f32p, f32p, f32p, f32p, f32p] + [ct.c_int] * 5
        L.orc_setAngleRounding.argtypes = [ct.c_int]
        L.orc_setAngleRounding.restype = None
        L.orc_angleRounding.restype = ct.c_int
        L.orc_cameraBasis.argtypes = [f32p, f32p]
        L.orc_retestFeatures.argtypes = [f32p, u32p, f32p, i32p, ct.c_int, f32p, ct.c_int]
        L.orc_reintersectF64.argtypes = [f32p, u32p, f32p, f32p, f32p, ct.c_int, ct.c_int, f64p, f64p, i32p, ct.c_int]

    def build_bounds(self, queue, world, nodes, nthreads=0):
        self.lib.orc_buildBounds(queue, world, nodes, nthreads)

    def trace(self, world, nodes, origin, C, hit, surface, w, h, row0=0, rows=None, nthreads=0, counters=None,
              second=None):
        rows = h if rows is None else rows
        self.lib.orc_tracePrimary(world, nodes, origin, C, hit, surface, w, h, row0, rows, nthreads,
                                  None if counters is None else counters.ctypes.data,
                                  None if second is None else second.ctypes.data)

    def shade(self, world, origin, C, hit, surface, linear, w, h, row0=0, rows=None, nthreads=0, counters=None):
        rows = h if rows is None else rows
        self.lib.orc_shadePixels(world, origin, C, hit, surface, linear, w, h, row0, rows, nthreads,
                                 None if counters is None else counters.ctypes.data)

    def resolve(self, linear, history, pixels, C, hit, surface, w, h, nthreads=0):
        self.lib.orc_resolveFrame(linear, history, pixels, C, hit, surface, w, h, nthreads)

    def resolve_rows(self, linear, history, pixels, C, hit, surface, w, h, row0, rows, nthreads=0):
        self.lib.orc_resolveRows(linear, history, pixels, C, hit, surface, w, h, row0, rows, nthreads)

    def trace_rays(self, world, nodes, origin, rays, exhaustive=False, nthreads=0):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        out = np.zeros((n, 8), np.float32)
        self.lib.orc_traceRays(world, nodes, np.ascontiguousarray(origin, np.uint32), rays, n, int(exhaustive), out,
                               nthreads)
        return out

    def feature_hit_f64(self, f10, ro, rd, cone=0.0):
        return self.lib.orc_featureHit_f64(np.ascontiguousarray(f10, np.float32), np.ascontiguousarray(ro, np.float64),
                                           np.ascontiguousarray(rd, np.float64), float(cone))

    def feature_normal_f64(self, f10, pt):
        out = np.zeros(3, np.float64)
        self.lib.orc_featureNormal_f64(np.ascontiguousarray(f10, np.float32), np.ascontiguousarray(pt, np.float64), out)
        return out

    def angle_rounding(self, mode=None):
        """Get (and with `mode`, set) how camera/sun/tap angles are evaluated: 0 = the C library's
        float sinf/cosf (the reference's CPU build), 1 = double rounded once (the CUDA path)."""
        old = self.lib.orc_angleRounding()
        if mode is not None:
            self.lib.orc_setAngleRounding(int(mode))
        return old

    # -- the optional material surrogate (learning.cu) ----------------------
    def init_neural(self, seed):
        """(W, M, V, Brain) of a fresh surrogate."""
        W, M, V, B = np.zeros(291, np.float32), np.zeros(291, np.float32), np.zeros(291, np.float32), np.zeros(32, np.float32)
        self.lib.orc_initNeural(W, M, V, B, int(seed))
        return W, M, V, B

    def material_step(self, s, hit, surface, net, width, height, work=None):
        """One training step on a frame (s: World/Origin/C), updating net = (W, M, V, Brain) in place."""
        W, M, V, B = net
        self.lib.orc_materialStep(s.World, s.Origin, s.C, np.ascontiguousarray(hit, np.float32),
                                  np.ascontiguousarray(surface, np.float32), W, M, V, B,
                                  None if work is None else work.ctypes.data, int(width), int(height))

    def predict_substrate(self, W, queries):
        q = np.ascontiguousarray(queries, np.float32)
        out = np.zeros((len(q), 3), np.float32)
        self.lib.orc_predictSubstrate(W, q, len(q), out)
        return out

    def shade_neural(self, s, hit, surface, linear, W, brain, width, height, nthreads=0):
        self.lib.orc_shadePixelsNeural(s.World, s.Origin, s.C, hit, surface, linear, W, brain, int(width), int(height),
                                       0, int(height), nthreads)

    def camera_basis(self, C, mode):
        """Forward and right vectors of camera state C with angle mode `mode` (bits)."""
        prev = self.angle_rounding(mode)
        out = np.zeros(6, np.float32)
        self.lib.orc_cameraBasis(np.ascontiguousarray(C, np.float32), out)
        self.angle_rounding(prev)
        return out

    def basis_matches_reference(self, C):
        """True when the device's camera basis equals the reference CPU build's for C."""
        return bool(np.array_equal(self.camera_basis(C, 0).view(np.uint32), self.camera_basis(C, 1).view(np.uint32)))

    def retest_features(self, world, origin, rays, ids, nthreads=0):
        """[t, n.xyz] of feature ids[i] = (slot, fid) on ray i, in its lot frame as the trace forms it."""
        rays = np.ascontiguousarray(rays, np.float32)
        ids = np.ascontiguousarray(ids, np.int32)
        out = np.zeros((len(rays), 4), np.float32)
        self.lib.orc_retestFeatures(world, np.ascontiguousarray(origin, np.uint32), rays, ids, len(rays), out, nthreads)
        return out

    def reintersect_f64(self, world, origin, C, hit, surface, w, h, nthreads=0):
        """FP64 re-intersection of every pixel's winning feature: (t64 [P], n64 [P, 6], status [P]).
        n64[:, :3] is the normal at the FP64 hit, n64[:, 3:] the FP64 normal at the frame's float hit point.
        status & 7: 0 sky, 1 ground, 2 feature, 3 foliage leaf disc, 4 not re-found in FP64;
        (status >> 3) & 15: the feature's shape; status >> 8: its material."""
        P = w * h
        t64 = np.zeros(P, np.float64)
        n64 = np.zeros(P * 6, np.float64)
        st = np.zeros(P, np.int32)
        self.lib.orc_reintersectF64(world, np.ascontiguousarray(origin, np.uint32), np.ascontiguousarray(C, np.float32),
                                    np.ascontiguousarray(hit, np.float32), np.ascontiguousarray(surface, np.float32),
                                    int(w), int(h), t64, n64, st, nthreads)
        return t64, n64.reshape(P, 6), st

    def query_lot_exhaustive(self, lot16, ro, rd, best=FAR, cone=0.0):
        fid = ct.c_int(0)
        f10 = np.zeros(10, np.float32)
        t = self.lib.orc_queryLot_exhaustive(np.ascontiguousarray(lot16, np.float32), np.ascontiguousarray(ro, np.float32),
                                             np.ascontiguousarray(rd, np.float32), float(best), float(cone),
                                             ct.byref(fid), f10)
        return t, fid.value, f10


class RefLib(_Lib):
    prefix = "ref_"

    def __init__(self, path: Path | None = None):
        super().__init__(path or REF_SO)
        L = self.lib
        L.ref_buildBounds.argtypes = [u32p, f32p, f32p, ct.c_int]
        L.ref_tracePrimary.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p] + [ct.c_int] * 5
        L.ref_shadePixels.argtypes = [f32p, u32p, f32p, f32p, f32p, f32p] + [ct.c_int] * 5
        L.ref_resolveFrame.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p] + [ct.c_int] * 3
        L.ref_resolveRows.argtypes = [f32p, f32p, u32p, f32p, f32p, f32p] + [ct.c_int] * 5

    def build_bounds(self, queue, world, nodes, nthreads=0):
        self.lib.ref_buildBounds(queue, world, nodes, nthreads)

    def trace(self, world, nodes, origin, C, hit, surface, w, h, row0=0, rows=None, nthreads=0, counters=None,
              second=None):
        rows = h if rows is None else rows
        self.lib.ref_tracePrimary(world, nodes, origin, C, hit, surface, w, h, row0, rows, nthreads)

    def shade(self, world, origin, C, hit, surface, linear, w, h, row0=0, rows=None, nthreads=0, counters=None):
        rows = h if rows is None else rows
        self.lib.ref_shadePixels(world, origin, C, hit, surface, linear, w, h, row0, rows, nthreads)

    def resolve(self, linear, history, pixels, C, hit, surface, w, h, nthreads=0):
        self.lib.ref_resolveFrame(linear, history, pixels, C, hit, surface, w, h, nthreads)

    def resolve_rows(self, linear, history, pixels, C, hit, surface, w, h, row0, rows, nthreads=0):
        self.lib.ref_resolveRows(linear, history, pixels, C, hit, surface, w, h, row0, rows, nthreads)


class device_angles:
    """Within this block the oracle evaluates camera, sun and resolve-tap angles
    as the CUDA path does (double precision rounded once to float)."""

    def __init__(self, orc):
        self.orc = orc

    def __enter__(self):
        self.prev = self.orc.angle_rounding(1)
        return self.orc

    def __exit__(self, *a):
        self.orc.angle_rounding(self.prev)


def ref_available() -> bool:
    return REF_SO.exists()


# ---- frame-level helpers ----------------------------------------------------
class World:
    """Host-side table state: World, Tags, Nodes, Queue, Args, C, Origin."""

    def __init__(self):
        self.World = np.zeros(WORLD_LOTS * LOT_FLOATS, np.float32)
        self.Tags = np.zeros(WORLD_LOTS * 4, np.uint32)
        self.Nodes = np.zeros(WORLD_LOTS * GROUP_NODES * 8, np.float32)
        self.Queue = np.zeros(WORLD_LOTS + 1, np.uint32)
        self.Args = np.zeros(8 * 21, np.uint32)
        self.C = np.zeros(64, np.float32)
        self.Origin = np.zeros(4, np.uint32)
        self.I = np.zeros(32, np.float32)


def setup_pose(lib, seed, pos, yaw, pitch, width, height, sample=1, shadows=True, origin=None, nthreads=0):
    """initCamera(seed), set the pose, stepCamera(dt=0) (rebases), force C[19]=sample,
    then describe and bound the whole table.  Mirrors the reference harness's
    render() set-up (tests/native_harness.cpp:100-105)."""
    s = World()
    lib.f("initCamera")(s.C, s.Origin, int(seed))
    if origin is not None:
        s.Origin[:] = np.asarray(origin, np.uint32)
    s.C[0], s.C[1], s.C[2] = pos
    s.C[3], s.C[4] = yaw, pitch
    s.C[18] = 0.0 if shadows else 1.0
    lib.f("stepCamera")(s.C, s.Origin, s.I, ct.c_float(0.0), int(width), int(height))
    s.C[19] = float(sample)
    lib.f("clearQueue")(s.Queue)
    lib.f("prepareLots")(s.Origin, s.C, s.World, s.Tags, s.Queue)
    lib.f("planBounds")(s.Queue, s.Args)
    lib.build_bounds(s.Queue, s.World, s.Nodes, nthreads)
    return s


def render(lib, s: World, width, height, nthreads=0, counters=None, second=None, history=None):
    P = width * height
    hit = np.zeros(P * 4, np.float32)
    surf = np.zeros(P * 4, np.float32)
    lin = np.zeros(P * 4, np.float32)
    hist = np.zeros(P * 4, np.float32) if history is None else history
    px = np.zeros(P, np.uint32)
    lib.trace(s.World, s.Nodes, s.Origin, s.C, hit, surf, width, height, nthreads=nthreads, counters=counters,
              second=second)
    lib.shade(s.World, s.Origin, s.C, hit, surf, lin, width, height, nthreads=nthreads, counters=counters)
    lib.resolve(lin, hist, px, s.C, hit, surf, width, height, nthreads=nthreads)
    return dict(Hit=hit, Surface=surf, Linear=lin, History=hist, Pixels=px)
