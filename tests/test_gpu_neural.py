"""The optional material surrogate (kernels/learning.cu of the reference) on
the GPU against the oracle's restatement, through the C ABI.

Its transcendentals are evaluated in double precision and rounded once on the
device, so the oracle runs with the same rounding (oracle_lib.device_angles):
initialisation and the first step's sample rows are bit-identical, 120 training
steps on a street frame track the oracle's parameters, moments and gate within
1e-5, the surrogate's colours agree within 1e-6, and the surrogate-shaded frame
agrees within 1/1024 per channel (the rest of the shading uses the device's
float functions).  With the surrogate switched off (C[16] = 0) the shade is
bit-identical to the drop-in shadePixels."""
import numpy as np
import pytest
import torch

import oracle_lib as ol
from bench import POSES, SEED
from gpu_lib import Frame, s, setup_pose

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_surrogate_training_and_shading_match_the_oracle(cuda, oracle):
    sb = cuda
    call, P = sb.call, sb.ptr
    p = POSES["street"]
    w, h = 320, 180
    g = setup_pose(SEED, p["pos"], p["yaw"], p["pitch"], w, h, origin=p["origin"])
    fr = Frame(w, h)
    fr.render(g)
    with ol.device_angles(oracle):
        o = ol.setup_pose(oracle, SEED, p["pos"], p["yaw"], p["pitch"], w, h, origin=p["origin"])
        hit, surf = fr.Hit.cpu().numpy(), fr.Surface.cpu().numpy()
        # initialisation: bit-identical
        net = oracle.init_neural(1788)
        W, M, V, B = (torch.zeros(n, dtype=torch.float32, device="cuda") for n in (291, 291, 291, 32))
        call("stratum_initNeural", P(W), P(M), P(V), P(B), 1788, s())
        for got, want in zip((W, M, V, B), net):
            assert np.array_equal(got.cpu().numpy().view(np.uint32), want.view(np.uint32))
        work = torch.zeros(64 * 64, dtype=torch.float32, device="cuda")
        owork = np.zeros(64 * 64, np.float32)
        worst = 0.0
        for k in range(120):
            g.C[6] = float(4 * k)
            o.C[6] = np.float32(4 * k)
            call("stratum_materialStep", P(g.World), P(g.Origin), P(g.C), P(fr.Hit), P(fr.Surface), P(W), P(M), P(V),
                 P(B), P(work), w, h, s())
            oracle.material_step(o, hit, surf, net, w, h, work=owork)
            if k == 0:
                assert np.array_equal(work.cpu().numpy().view(np.uint32), owork.view(np.uint32))
            for got, want in zip((W, M, V, B), net):
                d = np.abs(got.cpu().numpy() - want) / np.maximum(np.abs(want), 1e-3)
                worst = max(worst, float(d.max()))
        print("surrogate after 120 steps: Brain", B[:6].cpu().numpy(), "worst relative difference", worst)
        assert worst <= 1e-5, worst
        assert B[4].item() == net[3][4] == 1.0  # the gate opened on both
        # the surrogate's colours
        rng = np.random.default_rng(5)
        Q = np.stack([rng.uniform(-20, 20, 4096), rng.uniform(0, 30, 4096), rng.integers(0, 65536, 4096),
                      rng.integers(0, 2, 4096)], 1).astype(np.float32)
        out = torch.zeros(4096 * 3, dtype=torch.float32, device="cuda")
        call("stratum_predictSubstrate", P(W), P(dev(Q)), 4096, P(out), s())
        want = oracle.predict_substrate(net[0], Q)
        assert np.allclose(out.cpu().numpy().reshape(-1, 3), want, rtol=0, atol=1e-6)
        # the surrogate-shaded frame (C[16] = 1, gate open) against the oracle's
        g.C[16] = 1.0
        o.C[16] = np.float32(1.0)
        lin = torch.zeros(w * h * 4, dtype=torch.float32, device="cuda")
        call("stratum_shadePixelsNeural", P(g.World), P(g.Origin), P(g.C), P(fr.Hit), P(fr.Surface), P(lin), P(W),
             P(B), w, h, 0, h, s())
        olin = np.zeros(w * h * 4, np.float32)
        oracle.shade_neural(o, hit, surf, olin, W.cpu().numpy(), B.cpu().numpy(), w, h)
        err = np.abs(lin.cpu().numpy() - olin).reshape(-1, 4).max(axis=1)
        plain = np.zeros(w * h * 4, np.float32)
        oracle.shade(o.World, o.Origin, o.C, hit, surf, plain, w, h)
        changed = int((np.abs(plain - olin).reshape(-1, 4).max(axis=1) > 0).sum())
        print("surrogate-shaded pixels differing from the procedural substrate:", changed, "max error", err.max())
        assert changed > 1000 and int((err > 1.0 / 1024).sum()) == 0
    # switched off: the drop-in shade, bit for bit
    g.C[16] = 0.0
    call("stratum_shadePixelsNeural", P(g.World), P(g.Origin), P(g.C), P(fr.Hit), P(fr.Surface), P(lin), P(W), P(B),
         w, h, 0, h, s())
    ref = torch.zeros_like(lin)
    call("stratum_shadePixels", P(g.World), P(g.Origin), P(g.C), P(fr.Hit), P(fr.Surface), P(ref), w, h, 0, h, s())
    assert torch.equal(lin, ref)
