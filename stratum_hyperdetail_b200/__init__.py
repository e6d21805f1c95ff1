"""B200 implementation of the STRATUM frame path.

`lib()` loads the in-tree CUDA library (libstratum.so, sm_100a) and returns
it with every C-ABI entry point of include/stratum.h typed for ctypes.  The
`Engine` class mirrors the reference's host engine (src/engine.js): the same
buffers, the same per-frame order and the same error behaviour, over device
tensors.  There is no CPU fallback: without the library or a GPU every call
raises.
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libstratum.so"

WORLD_SIDE = 128
WORLD_LOTS = 16384
LOT_FLOATS = 16
CLUSTERS = 64
GROUP_NODES = 128
MAX_FEATURES = 64
BUILD_CHUNK = 2048
BUILD_CHUNKS = 8
RAY_DISTANCE = 2000.0
SKY_ID = -10000
NN_PARAMS = 291
GROUND_ID = -1

OK = 0
EINVAL = -100000
ELIMIT = -100001  # a fixed capacity of the library was exceeded
NOALLOC_MAX_VIEWS = 64
GROUP_CACHE_ENTRIES = 65536  # default group cache of a batched view: 137 MiB + 4 MiB directory
QUEUE_STALLED = 1
BUDGET_EXCEEDED = 2
NOT_FOUND = 3


class StratumError(RuntimeError):
    def __init__(self, name: str, status: int):
        super().__init__(f"{name} failed with status {status}")
        self.status = status


_P = ct.c_void_p  # device pointer
_I = ct.c_int
_F = ct.c_float
_S = ct.c_void_p  # stream

# name -> argument types (all return int status), in include/stratum.h order
SIGNATURES: dict[str, list] = {
    "stratum_initCamera": [_P, _P, _I, _S],
    "stratum_stepCamera": [_P, _P, _P, _F, _I, _I, _S],
    "stratum_clearQueue": [_P, _S],
    "stratum_prepareLots": [_P, _P, _P, _P, _P, _S],
    "stratum_planBounds": [_P, _P, _S],
    "stratum_buildGroupBounds": [_P, _P, _P, _I, _S],
    "stratum_reduceGroupBounds": [_P, _P, _I, _I, _S],
    "stratum_tracePrimary": [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _S],
    "stratum_shadePixels": [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _S],
    "stratum_resolveFrame": [_P, _P, _P, _P, _P, _P, _I, _I, _S],
    "stratum_probeGrammar": [_P, _P, _S],
    "stratum_initWorld": [_P, _P, _I, _S],
    "stratum_schedulePages": [_P, _P, _P, _P, _P, _S],
    "stratum_commitPages": [_P, _P, _S],
    "stratum_buildBVH": [_P, _P, _P, _S],
    "stratum_frame": [_P, _P, _P, _F, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _S],
    "stratum_enumerateGroups": [_P, _P, _I, _I, _P, _P, _S],
    "stratum_featureQuery": [_P, _I, _P, _S],
    "stratum_traceRays": [_P, _P, _P, _P, _I, _I, _P, _S],
    "stratum_retestFeatures": [_P, _P, _P, _P, _I, _P, _S],
    "stratum_initNeural": [_P, _P, _P, _P, _I, _S],
    "stratum_materialStep": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _S],
    "stratum_predictSubstrate": [_P, _P, _I, _P, _S],
    "stratum_shadePixelsNeural": [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _S],
    "stratum_applyPoses": [_P, _P, _P, _I, _S],
    "stratum_stepViews": [_P, _I, _S],
    "stratum_refreshViews": [_P, _I, _S],
    "stratum_buildViews": [_P, _I, _S],
    "stratum_traceViews": [_P, _I, _P, ct.c_ulonglong, _P, _S],
    "stratum_shadeViews": [_P, _I, _P, ct.c_ulonglong, _P, _S],
    "stratum_renderViews": [_P, _I, _P, ct.c_ulonglong, _P, _S],
    "stratum_frameViews": [_P, _I, _P, ct.c_ulonglong, _P, _S],
    "stratum_autotune": [_P, _I, _P, ct.c_ulonglong, _P, _P, _S],
    "stratum_renderViewsNoAlloc": [_P, _I, _P, _S],
    "stratum_groupCacheInit": [_P, _I, _S],
    "stratum_issueProbe": [_P, _I, _I, _S],
}


class Tune(ct.Structure):
    """stratum_tune: block size, tiles per queue claim, tile order (bit 0) and
    the block-pooled trace (bit 1 of order)."""
    _fields_ = [("threads", ct.c_int), ("grab", ct.c_int), ("order", ct.c_int)]


class ViewRecord(ct.Structure):
    """stratum_view: one view of a batch (device pointers + size)."""
    _fields_ = [(n, ct.c_void_p) for n in ("C", "Origin", "I", "World", "Tags", "Nodes", "Queue", "Hit", "Surface",
                                            "Linear", "History", "Pixels", "Groups")] + [
        ("width", ct.c_int), ("height", ct.c_int), ("dt", ct.c_float), ("tileBase", ct.c_int), ("tilesX", ct.c_int),
        ("reserved", ct.c_int)]

_lib = None


def lib() -> ct.CDLL:
    """The loaded CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m stratum_hyperdetail_b200.build`")
        L = ct.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ct.c_int
        L.stratum_version.restype = ct.c_char_p
        L.stratum_version.argtypes = []
        L.stratum_batchScratchBytes.restype = ct.c_ulonglong
        L.stratum_batchScratchBytes.argtypes = [ct.c_int]
        L.stratum_groupCacheBytes.restype = ct.c_ulonglong
        L.stratum_groupCacheBytes.argtypes = [ct.c_int]
        _lib = L
    return _lib


def check(name: str, status: int) -> None:
    if status != OK:
        raise StratumError(name, status)


def call(name: str, *args) -> None:
    """Invoke a C-ABI entry point and raise on a non-zero status."""
    check(name, getattr(lib(), name)(*args))


def ptr(t) -> int:
    """Device address of a CUDA tensor (or 0 for None)."""
    if t is None:
        return 0
    if not t.is_cuda:
        raise ValueError("stratum buffers must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("stratum buffers must be contiguous")
    return t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


from .engine import Engine  # noqa: E402  (mirror of src/engine.js)

__all__ = ["lib", "call", "ptr", "stream_handle", "Engine", "StratumError"]
