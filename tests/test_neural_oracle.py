"""The oracle's restatement of the optional material surrogate
(kernels/learning.cu of the reference) learns what the reference intends:
trained on a street frame's brick and stone pixels, its held-out error falls
well below the constant-colour baseline and its validation gate opens, with
either rounding of the transcendentals.  (CPU; the GPU is compared with this
restatement in test_gpu_neural.py.)"""
import numpy as np
import pytest

import oracle_lib as ol
from bench import POSES, SEED


@pytest.mark.parametrize("mode", [0, 1])
def test_surrogate_learns_and_opens_its_gate(oracle, mode):
    prev = oracle.angle_rounding(mode)
    try:
        p = POSES["street"]
        w, h = 320, 180
        s = ol.setup_pose(oracle, SEED, p["pos"], p["yaw"], p["pitch"], w, h, origin=p["origin"])
        f = ol.render(oracle, s, w, h)
        net = oracle.init_neural(1788)
        W0 = net[0].copy()
        assert np.all(net[0][216:288] == 0) and tuple(net[0][288:]) == (np.float32(0.36), np.float32(0.29), np.float32(0.20))
        opened = None
        for k in range(200):
            s.C[6] = 4 * k  # a training frame
            oracle.material_step(s, f["Hit"], f["Surface"], net, w, h)
            if opened is None and net[3][4] > 0.5:
                opened = k
        B = net[3]
        assert B[0] == 200 and B[1] >= 256 and B[5] >= 40, B[:6]
        assert opened is not None and opened < 150, opened
        assert B[2] < 0.2 * B[3], B[:6]
        assert not np.array_equal(W0, net[0])
        # frames that are not a multiple of 4, or frozen by C[21], do not train
        before = [a.copy() for a in net]
        s.C[6] = 5
        oracle.material_step(s, f["Hit"], f["Surface"], net, w, h)
        s.C[6], s.C[21] = 8, 1.0
        oracle.material_step(s, f["Hit"], f["Surface"], net, w, h)
        assert all(np.array_equal(a, b) for a, b in zip(before, net))
    finally:
        oracle.angle_rounding(prev)
