"""ParticleHistory's row (the phst output, src/dust/dust_science.cpp:391-482): the oracle
against an independent numpy restatement (CPU), and the device form against the oracle."""
import numpy as np
import pytest

from athenak_b200.inputs import make_state
from athenak_b200.mesh import uniform_mesh
from oracle.oracle import Oracle


def chunk_sums(st):
    """The particle sums in the reference's order: chunks of 4096 particles, each summed in
    particle order, then the chunks in order (plain Python floats: one rounding per add)."""
    pr = st.pr
    tot = [0.0] * 7
    for c0 in range(0, st.npart, 4096):
        a = [0.0] * 7
        for p in range(c0, min(c0 + 4096, st.npart)):
            m = float(pr[16, p])
            if m == 0.0:
                continue
            v1, v2, v3, z = float(pr[1, p]), float(pr[3, p]), float(pr[5, p]), float(pr[4, p])
            a[0] += 1.0; a[1] += m
            a[2] += m * v1; a[3] += m * v2; a[4] += m * v3
            a[5] += 0.5 * m * (v1 * v1 + v2 * v2 + v3 * v3)
            a[6] += m * z * z
        for q in range(7):
            tot[q] += a[q]
    return tot


def tsc_density(st, n, lo, dx):
    """m/V with TSC weights on one periodic block of n^3 cells (the ghost deposits folded)."""
    rho = np.zeros((n, n, n))
    pr = st.pr
    for p in range(st.npart):
        w, idx = [], []
        for a, r in enumerate((0, 2, 4)):
            cell = (pr[r, p] - lo) * (n / (n * dx))
            ig = int(cell + 1.0) - 1
            d = cell - (ig + 0.5)
            w.append((0.5 * (0.5 - d) ** 2, 0.75 - d * d, 0.5 * (0.5 + d) ** 2))
            idx.append(ig)
        for c in range(3):
            for b in range(3):
                for a in range(3):
                    rho[(idx[2] + c - 1) % n, (idx[1] + b - 1) % n, (idx[0] + a - 1) % n] += \
                        pr[16, p] / dx ** 3 * w[2][c] * w[1][b] * w[0][a]
    return rho


def test_oracle_phst_matches_restatement():
    ms = uniform_mesh((12, 12, 12), (12, 12, 12), 2, (-0.06,) * 3, (0.06,) * 3)
    st = make_state(ms, [0.1, 1.0], [1.0, 0.5], 3, seed=8, vel_noise=0.1, hp=0.01)
    st.pr[16, 5] = 0.0                      # an outflow tombstone: not counted
    o = Oracle(st, dict(scheme=2))
    row, err = o.phst(chi=0.25)
    assert err == 0
    s = chunk_sums(st)
    assert list(row[:6]) == s[:6]
    assert row[6] == np.sqrt(s[6] / s[1])
    rho = tsc_density(st, 12, -0.06, 0.01)
    k, j, i = np.unravel_index(np.argmax(rho), rho.shape)
    assert abs(row[7] - rho.max()) <= 1e-12 * rho.max()
    assert np.allclose(row[8:11], [-0.06 + (i + 0.5) * 0.01, -0.06 + (j + 0.5) * 0.01,
                                   -0.06 + (k + 0.5) * 0.01], rtol=0, atol=1e-15)
    assert row[11] == 0.0 and row[12] == 0.25 and row[13] == -1.0


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["periodic", "strat_outflow"])
def test_device_phst_matches_oracle(case):
    """Rows 0-6 bit for bit (the same summation order), the densest cell's value within
    1e-12 (its deposit sums in atomic order) and its centre exactly."""
    import torch
    from athenak_b200.drag import DeviceDust
    if case == "periodic":
        ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
        st = make_state(ms, [0.01, 0.1, 1.0], [0.5, 0.5, 0.5], 3, seed=3, vel_noise=0.05)
    else:
        ms = uniform_mesh((16, 16, 32), (8, 8, 16), 2, (-0.05, -0.05, -0.1), (0.05, 0.05, 0.1),
                          x3bc=2)
        st = make_state(ms, [0.1], [1.0], 4, seed=6, vel_noise=0.3, hp=0.05)
    st.pr[16, 7] = 0.0
    phys = dict(scheme=2)
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    chi = torch.tensor([0.5], dtype=torch.float64, device="cuda")
    rg = g.phst(chi).cpu().numpy()
    ro, err = o.phst(chi=0.5)
    assert err == 0 and g.error_word() == 0
    np.testing.assert_array_equal(rg[:7], ro[:7])
    assert abs(rg[7] - ro[7]) <= 1e-12 * ro[7]
    np.testing.assert_array_equal(rg[8:], ro[8:])
