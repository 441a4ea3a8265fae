"""The benchmark's end-to-end round trip (bench.HostRoundTrip: particle rows and u0 in pinned
host memory, copied in, one mixed cycle through the C ABI, copied out, every step): the
pipelined form, whose copies out and next copies in run on two more streams ordered row by row
with events, leaves the same host state as the serial form after three steps from the same
initial state (positions and velocities within 1e-6 of their scale, PGID equal, u0 within
1e-6), the host rows have moved, and the device rows equal the host rows after the last copy
in (nothing is copied over a row still in use)."""
import os
import sys

import numpy as np
import pytest

from athenak_b200.inputs import make_state
from athenak_b200.mesh import uniform_mesh

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PHYS = dict(scheme=2, drag_solver=2)
DT = 2e-3
TOL = 1e-6


def round_trip(st, pipelined, steps=3):
    sys.path.insert(0, ROOT)
    import bench
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    dev = DeviceDust(st, PHYS)
    mx = MixedDust(dev=dev, do_import=False)
    rt = bench.HostRoundTrip(dev, mx, pipelined=pipelined)
    for _ in range(steps):
        rt.step(DT)
    rt.drain()
    torch.cuda.synchronize()
    assert dev.error_word() == 0
    return rt


def test_pipelined_round_trip_matches_serial():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=27, vel_noise=0.05, gas_noise=1e-2)
    n = st.npart
    a = round_trip(st, pipelined=False)
    b = round_trip(st, pipelined=True)
    pa, pb = a.h_pr.numpy(), b.h_pr.numpy()
    for r in (0, 1, 2, 3, 4, 5):
        sc = np.abs(pa[r]).max()
        assert np.abs(pa[r] - pb[r]).max() <= TOL * sc, r
        assert np.abs(pa[r] - st.pr[r, :n]).max() > 0.0, r
    np.testing.assert_array_equal(a.h_pi.numpy(), b.h_pi.numpy())
    ua, ub = a.h_u0.numpy(), b.h_u0.numpy()
    for v in range(4):
        sc = np.abs(ua[:, v]).max()
        assert np.abs(ua[:, v] - ub[:, v]).max() <= TOL * sc, v
    # after the last copy in, the device holds what the host holds
    for rt in (a, b):
        dpr = rt.dev.t["pr"].cpu().numpy()
        for r in (0, 1, 2, 3, 4, 5, 15, 16):
            np.testing.assert_array_equal(dpr[r], rt.h_pr.numpy()[r])
        np.testing.assert_array_equal(rt.dev.t["pi"][0].cpu().numpy(), rt.h_pi.numpy()[0])
        np.testing.assert_array_equal(rt.dev.t["u0"].cpu().numpy(), rt.h_u0.numpy())
