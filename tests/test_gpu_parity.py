"""FP64 GPU kernels (C ABI, reference layout) against the CPU oracle on the same seeded
inputs.  Bar: particle-local arithmetic (push, route, weights, kick inputs) and every integer
output bit-exact; atomically accumulated fields within 1e-12 of the field's scale (the
deposit order of FP64 atomics differs from the oracle's sequential order)."""
import numpy as np
import pytest

from athenak_b200.mesh import uniform_mesh
from athenak_b200.inputs import make_state
from oracle.oracle import Oracle, imex2p_coeffs, GAMMA_DEFAULT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def fieldwise(a, b):
    """max over variables of the relative error of each variable's field"""
    return max(rel(a[:, v], b[:, v]) for v in range(a.shape[1]))


CASES = {
    "3d_random": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                      st=dict(taus=[0.01, 0.1, 1.0], eps=[0.5, 0.5, 0.5], ppc=2, seed=3,
                              vd=[0.1, -0.2, 0.3], gas_noise=1e-2, vel_noise=0.05),
                      phys=dict(scheme=2, drag_solver=2), dt=2e-3),
    "2d_lattice": dict(mesh=((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3),
                       st=dict(taus=[0.1, 0.03, 1.0], eps=[0.2, 0.5, 0.3], ppc=1,
                               placement="lattice", vd=[0.01 / 3, 0.02 / 3, 0.01],
                               gas_noise=0.0),
                       phys=dict(scheme=2, drag_solver=2), dt=0.0125),
    "sbox_nsh": dict(mesh=((32, 32, 32), (16, 16, 16), 2, (-0.05,) * 3, (0.05,) * 3),
                     st=dict(taus=[0.1], eps=[1.0], ppc=1, seed=1, shearing_box=True,
                             gas_noise=1e-3),
                     phys=dict(scheme=2, drag_solver=2, shearing_box=True), dt=1e-3,
                     sh=(1.5e-3, 1.5e-3)),
    "cic_dc2_noconsistent": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                                 st=dict(taus=[0.001, 1.0], eps=[2.0, 0.3], ppc=2, seed=9,
                                         vel_noise=0.02, gas_noise=1e-2),
                                 phys=dict(scheme=1, drag_solver=3, consistent_gas=False),
                                 dt=2e-3),
}


def build(name):
    from athenak_b200.drag import DeviceDust
    c = CASES[name]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    return Oracle(st, c["phys"]), DeviceDust(st, c["phys"]), c


def compare_particles(o, g, exact=False):
    n = o.st.npart
    gp, gi = g.host("pr"), g.host("pi")
    np.testing.assert_array_equal(gi, o.st.pi[:, :n])
    if exact:
        np.testing.assert_array_equal(gp, o.st.pr[:, :n])
    else:
        for r in range(17):
            assert rel(gp[r], o.st.pr[r, :n]) < TOL, r


@pytest.mark.parametrize("name", list(CASES))
def test_stage_tasks_parity(name):
    o, g, c = build(name)
    dt = c["dt"]
    sh = c.get("sh", (0.0, 0.0))[0]
    g0, g1, b, atw = imex2p_coeffs(GAMMA_DEFAULT)
    a_dt = GAMMA_DEFAULT * dt
    o.register_copy(); g.register_copy()
    compare_particles(o, g, exact=True)
    o.push_imex(g0[0], g1[0], b[0] * dt, 0.0); g.push_imex(g0[0], g1[0], b[0] * dt, 0.0)
    compare_particles(o, g, exact=True)
    assert o.route() == 0
    g.route()
    compare_particles(o, g, exact=True)
    assert o.deposit_qp(a_dt, sh) == 0
    g.deposit_qp(a_dt, sh)
    assert fieldwise(g.host("qdep")[:, :4], o.qdep[:, :4]) < TOL
    o.ghost_add("qdep", 5); g.ghost_add("qdep", 5)
    assert fieldwise(g.host("qdep")[:, :4], o.qdep[:, :4]) < TOL
    o.solve_ustar(); g.solve_ustar()
    assert fieldwise(g.host("ustar"), o.ustar) < TOL
    if c["phys"].get("drag_solver", 2) >= 2:
        assert o.dc1_sweep(a_dt, sh) == 0
        g.dc1_sweep(a_dt, sh)
        assert fieldwise(g.host("ustar"), o.ustar) < TOL
    o.ghost_copy("ustar", 3); g.ghost_copy("ustar", 3)
    assert fieldwise(g.host("ustar"), o.ustar) < TOL
    assert o.gather_kick_pmbr(a_dt, sh) == 0
    g.gather_kick_pmbr(a_dt, sh)
    compare_particles(o, g)
    assert fieldwise(g.host("dmom"), o.dmom) < TOL
    o.ghost_add("dmom", 3); g.ghost_add("dmom", 3)
    o.apply_pmbr(a_dt); g.apply_pmbr(a_dt)
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < TOL
    assert g.error_word() == 0


@pytest.mark.parametrize("name", list(CASES))
def test_imex_cycles_parity_and_conservation(name):
    o, g, c = build(name)
    sh = c.get("sh", (0.0, 0.0))
    p0 = sum(g.momentum())
    for _ in range(3):
        assert o.imex_cycle(c["dt"], sh=sh) == 0
        g.imex_cycle(c["dt"], sh=sh)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < 1e-11
    gm, dm = g.momentum()
    if not c["phys"].get("shearing_box"):
        scale = np.abs(p0).max()
        assert np.abs(gm + dm - p0).max() < 1e-13 * scale


def test_ghost_ops_bit_exact():
    o, g, c = build("3d_random")
    rng = np.random.default_rng(4)
    q = rng.standard_normal(o.qdep.shape)
    o.qdep[...] = q
    g.t["qdep"].copy_(torch.from_numpy(q))
    o.ghost_add("qdep", 5); g.ghost_add("qdep", 5)
    np.testing.assert_array_equal(g.host("qdep"), o.qdep)
    o.ghost_copy("qdep", 5, 0); g.ghost_copy("qdep", 5, 0)
    np.testing.assert_array_equal(g.host("qdep"), o.qdep)


def test_pc2_cycle_parity():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1], [1.0, 0.5], 2, seed=5, shearing_box=True, vel_noise=0.01)
    phys = dict(scheme=2, shearing_box=True)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    for _ in range(2):
        err, chi_o = o.pc2_cycle(2e-3)
        assert err == 0
        chi_g = float(g.pc2_cycle(2e-3).item())
        assert abs(chi_g - chi_o) <= 1e-12 * chi_o
    assert g.error_word() == 0
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < 1e-11


def test_sort_bit_exact_and_cell_index():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1], [1.0, 0.5], 3, seed=21, vel_noise=0.05)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, {}), DeviceDust(st, {})
    order_o, keys_o = o.sort_order()
    order_g, cstart = g.cell_index()
    np.testing.assert_array_equal(order_g.cpu().numpy(), order_o)
    counts = np.bincount(keys_o, minlength=ms.ncell_active)
    np.testing.assert_array_equal(np.diff(cstart.cpu().numpy()), counts)
    o.sort_particles()
    g.sort_by_cell()
    compare_particles(o, g, exact=True)


@pytest.mark.parametrize("dims", ["3d", "2d"])
def test_cloud_order_index_bit_exact(dims):
    """UpdateCloudOrder's index and tags against the oracle (bit-exact), its check before and
    after the rows are reordered, and the identity index a sort leaves."""
    from athenak_b200.drag import DeviceDust
    if dims == "3d":
        ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    else:
        ms = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
    st = make_state(ms, [0.01, 0.1], [1.0, 0.5], 3, seed=23, vel_noise=0.05)
    n = st.npart
    st.pi[1, :n:3] = -1 - np.arange(len(st.pi[1, :n:3]), dtype=np.int32)
    st.pi[4, :n:5] = 11
    o, g = Oracle(st, {}), DeviceDust(st, {})
    ord_o, tag_o = o.cloud_order()
    ord_g, tag_g = g.cloud_order()
    np.testing.assert_array_equal(ord_g.cpu().numpy(), ord_o)
    np.testing.assert_array_equal(tag_g.cpu().numpy().view(np.uint64), tag_o)
    assert g.cloud_order_check(ord_g, tag_g) == 0
    g.sort_by_cell()
    o.sort_particles()
    moved = o.cloud_order_check(ord_o, tag_o)
    assert moved > 0 and g.cloud_order_check(ord_g, tag_g) == moved
    ord_i, tag_i = g.cloud_order_identity()
    np.testing.assert_array_equal(ord_i.cpu().numpy(), np.arange(n))
    np.testing.assert_array_equal(tag_i.cpu().numpy().view(np.uint64), tag_o)
    assert g.cloud_order_check(ord_i, tag_i) == 0
    ord_r, tag_r = g.cloud_order()       # a rebuild on sorted rows is the identity
    np.testing.assert_array_equal(ord_r.cpu().numpy(), np.arange(n))
    bad = ord_i.clone()
    bad[:2] = torch.tensor([-1, n], dtype=torch.int32)
    assert g.cloud_order_check(bad, tag_i) == 2


def test_newdt_and_tstop_exact():
    o, g, c = build("sbox_nsh")
    dt_o = o.newdt() * 0.3
    dt_g = float(g.newdt(0.3).item())
    assert dt_g == dt_o
    ext = g.tstop_extrema().cpu().numpy()
    ext_o = o.tstop_extrema(1)
    np.testing.assert_array_equal(ext, ext_o)


def test_error_word_on_bad_particles():
    """Failure injection on the host: a particle four blocks away from its PGID block and
    one with an invalid stopping time; the kernels flag them and carry on."""
    from athenak_b200 import capi
    o, g, c = build("3d_random")
    pr = g.t["pr"]
    pr[0, 0] += 0.12          # 2.4 block widths (0.05) beyond: > 1 block away
    pr[15, 1] = -1.0
    g.route()
    g.tstop_extrema()
    torch.cuda.synchronize()
    w = g.error_word()
    assert w & capi.ERR_ROUTE
    assert w & capi.ERR_TSTOP


@pytest.mark.parametrize("drop", [False, True])
def test_ghost_add_x3_fold_bit_exact(drop):
    """Physical x3 faces: the fold of the ghost deposits beyond the faces (or their drop)
    matches the oracle bit for bit."""
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3, x3bc=1)
    st = make_state(ms, [0.1], [1.0], 1, seed=4)
    phys = dict(scheme=2, x3_deposit_drop=drop)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    rng = np.random.default_rng(5)
    q = rng.standard_normal(o.qdep.shape)
    o.qdep[...] = q
    g.t["qdep"].copy_(torch.from_numpy(q))
    o.ghost_add("qdep", 5)
    g.ghost_add("qdep", 5)
    np.testing.assert_array_equal(g.host("qdep"), o.qdep)


@pytest.mark.parametrize("coupling", ["imex", "pc2"])
def test_x3_reflect_stratified_cycles_parity(coupling):
    """A stratified shearing box with reflecting x3 faces (the boundaries of the stratified
    workload): routing at the faces, the u* x3 boundary values and the deposit fold, over
    cycles, against the oracle."""
    ms = uniform_mesh((16, 16, 32), (8, 8, 16), 2, (-0.05, -0.05, -0.1), (0.05, 0.05, 0.1),
                      x3bc=1)
    st = make_state(ms, [0.01, 0.1], [0.5, 0.5], 2, seed=17, shearing_box=True,
                    vel_noise=0.05, gas_noise=1e-2)
    phys = dict(scheme=2, drag_solver=2, shearing_box=True, stratified=True)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    for _ in range(3):
        if coupling == "imex":
            assert o.imex_cycle(2e-3) == 0
            g.imex_cycle(2e-3)
        else:
            err, chi_o = o.pc2_cycle(2e-3)
            assert err == 0
            chi_g = float(g.pc2_cycle(2e-3).item())
            assert abs(chi_g - chi_o) <= 1e-12 * chi_o
    torch.cuda.synchronize()
    assert g.error_word() == 0
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < 1e-11


def test_shear_ghost_ops_bit_exact():
    """Shear-periodic x1 faces: the PLM remap of the x1 ghost strips after the periodic copy
    and the remap of the ghost deposits beyond the faces match the oracle bit for bit."""
    ms = uniform_mesh((16, 32, 16), (8, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05),
                      x3bc=1, shear_x1=True)
    st = make_state(ms, [0.1], [1.0], 1, seed=4)
    phys = dict(scheme=2, shearing_box=True)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    for t in (0.0, 0.37, 5.3, 1.32):
        o.set_time(t)
        g.set_time(t)
        rng = np.random.default_rng(int(t * 100) + 1)
        q = rng.standard_normal(o.qdep.shape)
        o.qdep[...] = q
        g.t["qdep"].copy_(torch.from_numpy(q))
        o.ghost_add("qdep", 5)
        g.ghost_add("qdep", 5)
        np.testing.assert_array_equal(g.host("qdep"), o.qdep)
        u = rng.standard_normal(o.ustar.shape)
        o.ustar[...] = u
        g.t["ustar"].copy_(torch.from_numpy(u))
        o.ghost_copy("ustar", 3, 1)
        g.ghost_copy("ustar", 3, 1)
        np.testing.assert_array_equal(g.host("ustar"), o.ustar)


@pytest.mark.parametrize("coupling", ["imex", "pc2"])
def test_shearing_box_cycles_parity(coupling):
    """The unstratified shearing box with shear-periodic x1 faces (the small workload's
    boundaries): routing across the radial faces, the u* / gas ghost remaps and the deposit
    remap over cycles whose time advances, against the oracle."""
    ms = uniform_mesh((32, 32, 32), (16, 16, 16), 2, (-0.05,) * 3, (0.05,) * 3, shear_x1=True)
    st = make_state(ms, [0.1], [1.0], 1, seed=1, shearing_box=True, gas_noise=1e-3,
                    vel_noise=0.02)
    phys = dict(scheme=2, drag_solver=2, shearing_box=True)
    from athenak_b200.drag import DeviceDust
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    dt, t = 2e-3, 1.7
    for _ in range(3):
        o.set_time(t)
        g.set_time(t)
        if coupling == "imex":
            assert o.imex_cycle(dt) == 0
            g.imex_cycle(dt)
        else:
            err, chi_o = o.pc2_cycle(dt)
            assert err == 0
            chi_g = float(g.pc2_cycle(dt).item())
            assert abs(chi_g - chi_o) <= 1e-12 * chi_o
        t += dt
    torch.cuda.synchronize()
    assert g.error_word() == 0
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < 1e-11


@pytest.mark.parametrize("coupling", ["imex", "pc2"])
def test_dense_sorted_cells_parity(coupling):
    """Rows in cell order with about 64 particles per cell (the order a run keeps them in
    after SortParticles; most warps of the FP64 deposit kernels then add into the same 27
    cells): three imex2+/dc2 or pc2 cycles against the oracle, particles within 1e-12 of each
    row's scale (PGID exact), the gas within 1e-11, no error bit."""
    from athenak_b200.drag import DeviceDust
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 32, seed=29, vel_noise=0.05, gas_noise=1e-2)
    phys = dict(scheme=2, drag_solver=2)
    o, g = Oracle(st, phys), DeviceDust(st, phys)
    o.sort_particles()
    g.sort_by_cell()
    compare_particles(o, g, exact=True)
    for _ in range(3):
        if coupling == "imex":
            assert o.imex_cycle(2e-3) == 0
            g.imex_cycle(2e-3)
        else:
            assert o.pc2_cycle(2e-3)[0] == 0
            g.pc2_cycle(2e-3)
    torch.cuda.synchronize()
    assert g.error_word() == 0
    compare_particles(o, g)
    assert fieldwise(g.host("u0"), o.u0) < 1e-11
