"""Refinable clouds on a uniform 3-D mesh on the GPU (FP64, reference layout) against the
oracle on the same seeded inputs: the cloud Q/P deposit (FP64 atomics: within 1e-12 of each
field's scale), the gather pack of u* (bit-exact), the linear-moment gather-kick (velocities
and rates bit-exact: the gather sums in the same leaf order; the deposited impulse within
1e-12), mixed cloud levels 0-3, the error bit of lobed codes, and the unsupported layouts."""
import numpy as np
import pytest

from athenak_b200.inputs import make_state
from athenak_b200.mesh import uniform_mesh
from oracle.oracle import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def pair(levels, seed=5, lobed=(), phys=None):
    from athenak_b200.drag import DeviceDust
    ms = uniform_mesh((16, 32, 16), (8, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05))
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=seed, vel_noise=0.05, gas_noise=1e-2)
    n = st.npart
    st.pi[3, :n] = np.asarray(levels)[np.arange(n) % len(levels)]
    for p in lobed:
        st.pi[3, p] = 1 | (2 << 4)
    phys = dict(scheme=2) if phys is None else phys
    return ms, st, Oracle(st, phys), DeviceDust(st, phys)


def rel_fields(a, b):
    return max(np.abs(a[:, v] - b[:, v]).max() / max(np.abs(b[:, v]).max(), 1e-300)
               for v in range(a.shape[1]))


@pytest.mark.parametrize("levels", [(0,), (0, 1, 2, 3)])
def test_cloud_deposit_matches_oracle(levels):
    ms, st, o, g = pair(levels)
    assert o.cloud_deposit_qp(1.3e-3, 0.0) == 0
    g.cloud_deposit_qp(1.3e-3, 0.0)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    assert rel_fields(g.host("qdep")[:, :4], o.qdep[:, :4]) < 1e-12


@pytest.mark.parametrize("levels", [(0,), (0, 1, 2, 3)])
def test_cloud_gather_kick_matches_oracle(levels):
    ms, st, o, g = pair(levels, seed=11)
    rng = np.random.default_rng(6)
    us = rng.standard_normal(o.ustar.shape) * 0.05
    o.ustar[...] = us
    g.t["ustar"].copy_(torch.from_numpy(us))
    o.ghost_copy("ustar", 3, 0)
    g.ghost_copy("ustar", 3, 0)
    gp_o = o.gather_pack()
    assert o.cloud_gather_kick(2e-3, 0.0, gp_o) == 0
    gp_g = g.cloud_gather_kick(2e-3, 0.0)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    np.testing.assert_array_equal(gp_g[:gp_o.size].cpu().numpy(), gp_o.reshape(-1))
    n = st.npart
    gpr = g.host("pr")
    for r in (1, 3, 5, 12, 13, 14):
        np.testing.assert_array_equal(gpr[r], o.st.pr[r, :n])
    assert rel_fields(g.host("dmom"), o.dmom) < 1e-12


def test_lobed_codes_and_unsupported_meshes():
    from athenak_b200.drag import DeviceDust
    ms, st, o, g = pair((0,), lobed=(3, 17))
    assert o.cloud_deposit_qp(1e-3, 0.0) == 0x100
    g.cloud_deposit_qp(1e-3, 0.0)
    torch.cuda.synchronize()
    assert g.error_word() == 0x100
    assert rel_fields(g.host("qdep")[:, :4], o.qdep[:, :4]) < 1e-12
    sb = uniform_mesh((16, 32, 16), (8, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05),
                      shear_x1=True)
    st2 = make_state(sb, [0.1], [1.0], 1, seed=2)
    g2 = DeviceDust(st2, dict(scheme=2, shearing_box=True))
    with pytest.raises(RuntimeError):
        g2.cloud_deposit_qp(1e-3, 0.0)


@pytest.mark.parametrize("solver", [0, 2, 3])
def test_cloud_imex_cycles_match_oracle(solver):
    """Three imex2+ cycles of clouds of levels 0-3 (the clouds' deposit, dc1 / dc2 sweeps,
    gather-kick and overlap split): particles within 1e-12 of each row's scale (PGID exact),
    the gas within 1e-11 (FP64 atomics in the deposits)."""
    ms, st, o, g = pair((0, 1, 2, 3), seed=17, phys=dict(scheme=2, drag_solver=solver))
    for _ in range(3):
        assert o.cloud_imex_cycle(2e-3) == 0
        g.cloud_imex_cycle(2e-3)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    n = st.npart
    gp, gi = g.host("pr"), g.host("pi")
    np.testing.assert_array_equal(gi, o.st.pi[:, :n])
    for r in range(17):
        sc = max(np.abs(o.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(gp[r] - o.st.pr[r, :n]).max() <= 1e-12 * sc, r
    gu = g.host("u0")
    for v in range(4):
        sc = max(np.abs(o.u0[:, v]).max(), 1e-300)
        assert np.abs(gu[:, v] - o.u0[:, v]).max() <= 1e-11 * sc, v


@pytest.mark.parametrize("solver", [0, 2])
def test_2d_cloud_deposit_gather_and_cycles_match_oracle(solver):
    """2-D clouds (cell areas, the 9-component pack): the deposit within 1e-12, the kick bit
    for bit, three cycles within 1e-12 of the oracle."""
    from athenak_b200.drag import DeviceDust
    ms = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=19, vel_noise=0.05, gas_noise=1e-2)
    n = st.npart
    st.pi[3, :n] = np.arange(n) % 4
    phys = dict(scheme=2, drag_solver=solver)
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    assert o.cloud_deposit_qp(1.1e-3, 0.0) == 0
    g.cloud_deposit_qp(1.1e-3, 0.0)
    torch.cuda.synchronize()
    assert rel_fields(g.host("qdep")[:, :4], o.qdep[:, :4]) < 1e-12
    o2, g2 = Oracle(st, phys), DeviceDust(st, phys)
    for _ in range(3):
        assert o2.cloud_imex_cycle(0.01) == 0
        g2.cloud_imex_cycle(0.01)
    torch.cuda.synchronize()
    assert g.error_word() == 0 and g2.error_word() == 0
    gp, gi = g2.host("pr"), g2.host("pi")
    np.testing.assert_array_equal(gi, o2.st.pi[:, :n])
    for r in range(17):
        sc = max(np.abs(o2.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(gp[r] - o2.st.pr[r, :n]).max() <= 1e-12 * sc, r
    gu = g2.host("u0")
    for v in range(4):
        sc = max(np.abs(o2.u0[:, v]).max(), 1e-300)
        assert np.abs(gu[:, v] - o2.u0[:, v]).max() <= 1e-11 * sc, v


@pytest.mark.parametrize("dims", [3, 2])
def test_cloud_pc2_cycles_match_oracle(dims):
    """Three pc2 cycles of clouds of levels 0-3 (the clouds' predictor and midpoint advance,
    a shearing box's Coriolis terms in 3-D): particles within 1e-12 of each row's scale, the
    gas within 1e-11, chi_max within 1e-12."""
    from athenak_b200.drag import DeviceDust
    if dims == 3:
        ms = uniform_mesh((16, 32, 16), (8, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05))
        phys = dict(scheme=2, shearing_box=True, stratified=True)
        st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=23, vel_noise=0.05,
                        gas_noise=1e-2, shearing_box=True)
        dt = 2e-3
    else:
        ms = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
        phys = dict(scheme=2)
        st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=23, vel_noise=0.05, gas_noise=1e-2)
        dt = 0.01
    n = st.npart
    st.pi[3, :n] = np.arange(n) % 4
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    g.init_gas_ghosts()
    o.ghost_copy("u0", 4, 0)
    for _ in range(3):
        err, chi_o = o.cloud_pc2_cycle(dt)
        assert err == 0
        chi_g = float(g.cloud_pc2_cycle(dt).item())
        assert abs(chi_g - chi_o) <= 1e-12 * max(abs(chi_o), 1e-300)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    gp, gi = g.host("pr"), g.host("pi")
    np.testing.assert_array_equal(gi, o.st.pi[:, :n])
    for r in range(17):
        sc = max(np.abs(o.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(gp[r] - o.st.pr[r, :n]).max() <= 1e-12 * sc, r
    gu = g.host("u0")
    for v in range(4):
        sc = max(np.abs(o.u0[:, v]).max(), 1e-300)
        assert np.abs(gu[:, v] - o.u0[:, v]).max() <= 1e-11 * sc, v


@pytest.mark.parametrize("coupling", ["imex", "pc2"])
def test_cloud_cycles_at_physical_x3_faces_match_oracle(coupling):
    """Clouds within a cell of reflecting x3 faces (their mirrored parts) through three imex2+
    or pc2 cycles of a stratified box: particles within 1e-12, the gas within 1e-11."""
    from athenak_b200.drag import DeviceDust
    from tests.test_clouds import setup_x3
    ms, st = setup_x3((0, 1, 2), seed=31)
    phys = dict(scheme=2, drag_solver=2, stratified=True)
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    g.init_gas_ghosts()
    u = g.host("u0")
    o.u0[...] = u
    for _ in range(3):
        if coupling == "imex":
            assert o.cloud_imex_cycle(2e-3) == 0
            g.cloud_imex_cycle(2e-3)
        else:
            assert o.cloud_pc2_cycle(2e-3)[0] == 0
            g.cloud_pc2_cycle(2e-3)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    n = o.st.npart
    gp, gi = g.host("pr"), g.host("pi")
    np.testing.assert_array_equal(gi, o.st.pi[:, :n])
    for r in range(17):
        sc = max(np.abs(o.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(gp[r] - o.st.pr[r, :n]).max() <= 1e-12 * sc, r
    gu = g.host("u0")
    for v in range(4):
        sc = max(np.abs(o.u0[:, v]).max(), 1e-300)
        assert np.abs(gu[:, v] - o.u0[:, v]).max() <= 1e-11 * sc, v
