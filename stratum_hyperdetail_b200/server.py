"""Render server over the C ABI (continuous batching, HBM-budget admission).

    srv = Server(budget_bytes=150 << 30, max_views=16, streams=3)
    sid = srv.open(seed, 1600, 900)
    rid = srv.submit(sid, Pose(origin, pos, yaw, pitch), samples=1)
    info = srv.wait(rid, timeout_ms=1000)
    srv.stats()
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import Tune, check, lib

OK, QUEUE_STALLED, BUDGET_EXCEEDED, NOT_FOUND = 0, 1, 2, 3


class Pose(ct.Structure):
    _fields_ = [("origin", ct.c_uint * 4), ("pos", ct.c_float * 3), ("yaw", ct.c_float), ("pitch", ct.c_float)]

    @classmethod
    def make(cls, origin, pos, yaw, pitch):
        p = cls()
        for i in range(4):
            p.origin[i] = int(origin[i]) & 0xFFFFFFFF
        for i in range(3):
            p.pos[i] = float(pos[i])
        p.yaw, p.pitch = float(yaw), float(pitch)
        return p


class Stats(ct.Structure):
    _fields_ = [(n, ct.c_longlong) for n in ("submitted", "completed", "failed", "batches", "admissions", "evictions",
                                             "resident_sessions")] + [
        ("resident_bytes", ct.c_ulonglong), ("budget_bytes", ct.c_ulonglong)] + [
        (n, ct.c_double) for n in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "rays", "first_submit_s", "last_done_s")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class RequestInfo(ct.Structure):
    _fields_ = [("status", ct.c_int), ("samples_done", ct.c_int), ("latency_ms", ct.c_double),
                ("queue_ms", ct.c_double)]


_typed = False


def _lib():
    global _typed
    L = lib()
    if not _typed:
        vp = ct.c_void_p
        L.stratum_server_create.restype = vp
        L.stratum_server_create.argtypes = [ct.c_ulonglong, ct.c_int, ct.c_int, ct.POINTER(Tune)]
        L.stratum_server_destroy.restype = None
        L.stratum_server_destroy.argtypes = [vp]
        L.stratum_server_open.argtypes = [vp, ct.c_int, ct.c_int, ct.c_int, ct.POINTER(ct.c_int)]
        L.stratum_server_close.argtypes = [vp, ct.c_int]
        L.stratum_server_submit.argtypes = [vp, ct.c_int, ct.POINTER(Pose), ct.c_int, vp, ct.POINTER(ct.c_longlong)]
        L.stratum_server_wait.argtypes = [vp, ct.c_longlong, ct.c_int, ct.POINTER(RequestInfo)]
        L.stratum_server_stats_get.argtypes = [vp, ct.POINTER(Stats)]
        L.stratum_server_inject.argtypes = [vp, ct.c_int, ct.c_int]
        L.stratum_server_read.argtypes = [vp, ct.c_int, vp, vp]
        L.stratum_server_set_group_cache.argtypes = [vp, ct.c_int]
        for n in ("open", "close", "submit", "wait", "stats_get", "inject", "read", "set_group_cache"):
            getattr(L, "stratum_server_" + n).restype = ct.c_int
        _typed = True
    return L


class Server:
    def __init__(self, budget_bytes: int, max_views: int = 16, streams: int = 3, tune=(64, 1, 1),
                 group_cache: int | None = None):
        """`group_cache`: group cache entries per session (None: the library's
        default of 16,384; 0: none)."""
        self.L = _lib()
        t = Tune(*tune)
        self.h = self.L.stratum_server_create(int(budget_bytes), int(max_views), int(streams), ct.byref(t))
        if not self.h:
            raise RuntimeError("stratum_server_create failed")
        if group_cache is not None and self.L.stratum_server_set_group_cache(self.h, int(group_cache)) != 0:
            raise ValueError("bad group cache size")
        self.sizes = {}

    def close(self):
        if self.h:
            self.L.stratum_server_destroy(self.h)
            self.h = None

    __del__ = close

    def open(self, seed, width, height) -> int:
        sid = ct.c_int()
        check("stratum_server_open", self.L.stratum_server_open(self.h, int(seed), int(width), int(height),
                                                                 ct.byref(sid)))
        self.sizes[sid.value] = (int(width), int(height))
        return sid.value

    def close_session(self, sid) -> int:
        return self.L.stratum_server_close(self.h, int(sid))

    def submit(self, sid, pose: Pose, samples=1, out: np.ndarray | None = None) -> int:
        rid = ct.c_longlong()
        ptr = out.ctypes.data if out is not None else None
        check("stratum_server_submit", self.L.stratum_server_submit(self.h, int(sid), ct.byref(pose), int(samples),
                                                                     ptr, ct.byref(rid)))
        return rid.value

    def wait(self, rid, timeout_ms=10000) -> RequestInfo:
        info = RequestInfo()
        self.L.stratum_server_wait(self.h, int(rid), int(timeout_ms), ct.byref(info))
        return info

    def wait_status(self, rid, timeout_ms=10000) -> int:
        return self.L.stratum_server_wait(self.h, int(rid), int(timeout_ms), None)

    def stats(self) -> dict:
        st = Stats()
        check("stratum_server_stats_get", self.L.stratum_server_stats_get(self.h, ct.byref(st)))
        return st.as_dict()

    def inject_alloc_failures(self, count: int):
        check("stratum_server_inject", self.L.stratum_server_inject(self.h, 1, int(count)))

    def inject_launch_failures(self, count: int):
        """The next `count` batches fail after refreshViews, with part of their work queued."""
        check("stratum_server_inject", self.L.stratum_server_inject(self.h, 2, int(count)))

    def read(self, sid):
        w, h = self.sizes[sid]
        px = np.zeros(w * h, np.uint32)
        hist = np.zeros(w * h * 4, np.float32)
        check("stratum_server_read", self.L.stratum_server_read(self.h, int(sid), px.ctypes.data, hist.ctypes.data))
        return px, hist
