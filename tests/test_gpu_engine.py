"""The host engine mirror (stratum_hyperdetail_b200.engine.Engine, the
reference's src/engine.js:7-92) on the GPU against the CPU oracle driven
through the same sequence.

init rounds the size up (width to 64, height to 8), runs initCamera and one
warm-up prepare + full-table build with the resize flag set (I[23] = 1); every
frame(dt) then runs stepCamera with the engine's input and dt clamped to
[0, 0.1], the tag-compare refresh, the hierarchy build of the queued lots and
trace / shade / resolve (src/engine.js:67-83).  The oracle evaluates camera
angles as the CUDA path does (double precision rounded once); with that, after
each frame the engine's Origin and camera state equal the oracle's bit for bit,
and the frame -- table, hierarchy, Hit, Surface, Linear, History, Pixels -- is
compared.  inspect() reports the signed 64-bit
origin, the refreshed-lot count and the frame count; reset(seed) clears the
table and History and restarts from initCamera (src/engine.js:91); a disposed
engine refuses to draw.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

import oracle_lib as ol
from gpu_lib import compare_frames

pytestmark = pytest.mark.gpu
TOL_T, TOL_N, TOL_C = 1e-5, 1e-5, 1.0 / 1024.0


class OracleEngine:
    """The src/engine.js sequence on the CPU oracle."""

    def __init__(self, orc, width, height, seed):
        self.orc, self.w, self.h = orc, width, height
        self.s = ol.World()
        orc.f("initCamera")(self.s.C, self.s.Origin, int(seed))
        P = width * height
        self.hist = np.zeros(P * 4, np.float32)
        I = np.zeros(32, np.float32)
        I[23] = 1.0  # init's resize flag
        self.step(I, 0.0)
        self.refresh()

    def step(self, I, dt):
        self.orc.f("stepCamera")(self.s.C, self.s.Origin, np.ascontiguousarray(I, np.float32),
                                 ct.c_float(max(0.0, min(0.1, dt))), self.w, self.h)

    def refresh(self):
        s = self.s
        self.orc.f("clearQueue")(s.Queue)
        self.orc.f("prepareLots")(s.Origin, s.C, s.World, s.Tags, s.Queue)
        self.orc.f("planBounds")(s.Queue, s.Args)
        self.orc.build_bounds(s.Queue, s.World, s.Nodes)

    def draw(self, second):
        return ol.render(self.orc, self.s, self.w, self.h, second=second, history=self.hist)


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def test_engine_frames_against_oracle(cuda, oracle):
    with ol.device_angles(oracle):
        engine_frames(oracle)


def engine_frames(oracle):
    from stratum_hyperdetail_b200.engine import Engine
    eng = Engine().init(300, 170, seed=1788)
    assert (eng.width, eng.height) == (320, 176)
    w, h = eng.width, eng.height
    ref = OracleEngine(oracle, w, h, 1788)
    b = eng.buffers
    assert np.array_equal(u32(b["Origin"]), ref.s.Origin)
    assert np.array_equal(b["World"].cpu().numpy().view(np.uint32), ref.s.World.view(np.uint32))
    # inputs per frame: (index, value) pairs of I[32], dt
    script = [({}, 1 / 60), ({}, 1 / 60), ({0: 1.0, 5: 1.0}, 0.1), ({0: 1.0, 5: 1.0}, 0.5),
              ({3: 30.0, 4: -10.0}, 1 / 60), ({9: 1.0}, 1 / 30), ({14: 1.0}, 1 / 60), ({}, 1 / 60), ({}, 1 / 60)]
    for f, (inp, dt) in enumerate(script):
        eng.input.zero_()
        I = np.zeros(32, np.float32)
        for k, val in inp.items():
            eng.input[k] = val
            I[k] = val
        eng.frame(dt)
        torch.cuda.synchronize()
        ref.step(I, dt)
        gc = b["C"].cpu().numpy()
        assert np.array_equal(u32(b["Origin"]), ref.s.Origin), f
        assert np.array_equal(gc.view(np.uint32), ref.s.C.view(np.uint32)), (f, np.flatnonzero(gc != ref.s.C))
        ref.refresh()
        assert np.array_equal(b["World"].cpu().numpy().view(np.uint32), ref.s.World.view(np.uint32)), f
        assert np.array_equal(u32(b["Tags"]), ref.s.Tags), f
        assert np.array_equal(b["Nodes"].cpu().numpy(), ref.s.Nodes), f
        assert int(u32(b["Queue"])[0]) == int(ref.s.Queue[0]), f
        second = np.zeros(w * h, np.float32)
        want = ref.draw(second)
        got = {k: b[k].cpu().numpy() for k in ("Hit", "Surface", "Linear", "History")}
        got["Pixels"] = u32(b["Pixels"])
        rep = compare_frames(got, want, second, TOL_T, TOL_N, TOL_C)
        print("engine frame", f, "sample", gc[19], rep)
        assert rep["identity_bad"] == 0 and rep["t_bad"] == 0 and rep["n_bad"] == 0, (f, rep)
        assert rep["linear_bad"] <= 2 and rep["history_bad"] <= 2, (f, rep)
        # the oracle keeps the engine's History so accumulation continues from the same state
        ref.hist[:] = got["History"]
    info = eng.inspect()
    o = ref.s.Origin.astype(np.int64)
    sx = (int(o[1]) << 32 | int(o[0]))
    sx = sx - (1 << 64) if sx >= 1 << 63 else sx
    assert info["origin"]["x"] == str(sx) and info["frames"] == len(script)
    assert info["refreshedLots"] == int(ref.s.Queue[0]) and info["accelerationBytes"] == 64 << 20
    assert (info["width"], info["height"]) == (w, h)
    # reset(seed): World, Tags, History cleared, initCamera(seed), one frame without drawing
    eng.reset(4242)
    ref2 = ol.World()
    oracle.f("initCamera")(ref2.C, ref2.Origin, 4242)
    oracle.f("stepCamera")(ref2.C, ref2.Origin, ref2.I, ct.c_float(0.0), w, h)
    oracle.f("clearQueue")(ref2.Queue)
    oracle.f("prepareLots")(ref2.Origin, ref2.C, ref2.World, ref2.Tags, ref2.Queue)
    torch.cuda.synchronize()
    assert np.array_equal(u32(b["Origin"]), ref2.Origin)
    assert np.array_equal(b["C"].cpu().numpy().view(np.uint32), ref2.C.view(np.uint32))
    assert np.array_equal(b["World"].cpu().numpy().view(np.uint32), ref2.World.view(np.uint32))
    assert int(u32(b["Queue"])[0]) == 16384
    assert not b["History"].any()
    eng.dispose()
    with pytest.raises(RuntimeError, match="Renderer disposed"):
        eng.frame()
