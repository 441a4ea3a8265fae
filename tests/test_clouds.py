"""Refinable clouds on a uniform 3-D mesh (plain P1 hat clouds; the cloud level in PLEV), the
oracle's restatement of the reference's cloud deposit (CloudDepositImplicitT), gather pack
(PackGatherField3D) and linear-moment gather-kick (CloudGatherKickT) checked by properties
that pin it without the reference binary:
  * a level-0 cloud's weights are the TSC weights (a hat of half-width dx integrated over the
    cells is the quadratic B-spline): the cloud deposit equals the point particles' TSC
    deposit after its ghost exchange, to round-off;
  * every cloud of every level deposits its whole coupled mass (weights sum to one);
  * the linear gather reproduces a linear velocity field exactly at the particle (hat clouds
    are symmetric; central differences are exact for a linear field);
  * the kick and its deposited impulse conserve momentum;
  * a cloud code with lobe bits (transition clouds of refined meshes) is flagged, not used."""
import numpy as np
import pytest

from athenak_b200.inputs import _block_of, make_state
from athenak_b200.mesh import uniform_mesh
from oracle.oracle import Oracle

ERR_CLOUD = 0x100


def setup(levels=(0,), seed=5, ppc=2):
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], ppc, seed=seed, vel_noise=0.05,
                    gas_noise=1e-2)
    n = st.npart
    st.pi[3, :n] = np.asarray(levels)[np.arange(n) % len(levels)]
    return ms, st


def test_level0_cloud_deposit_is_the_tsc_deposit():
    ms, st = setup((0,))
    o_cloud = Oracle(st, dict(scheme=2))
    o_point = Oracle(st, dict(scheme=2))
    a_dt = 1.7e-3
    assert o_cloud.cloud_deposit_qp(a_dt) == 0
    assert o_point.deposit_qp(a_dt) == 0
    o_point.ghost_add("qdep", 5)
    qa, qb = ms.active(o_cloud.qdep)[:, :4], ms.active(o_point.qdep)[:, :4]
    for v in range(4):
        sc = np.abs(qb[:, v]).max()
        assert np.abs(qa[:, v] - qb[:, v]).max() < 1e-13 * sc, v


@pytest.mark.parametrize("levels", [(0,), (1,), (2,), (0, 1, 2, 3)])
def test_every_cloud_deposits_its_whole_mass(levels):
    ms, st = setup(levels)
    o = Oracle(st, dict(scheme=2))
    a_dt = 2e-3
    assert o.cloud_deposit_qp(a_dt) == 0
    n = st.npart
    want = (st.pr[16, :n] * a_dt / (st.pr[15, :n] + a_dt)).sum()
    got = ms.active(o.qdep)[:, 0].sum() * ms.cell_volume()
    assert abs(got - want) < 1e-13 * want
    # nothing lands in a ghost cell: the leaves are the owners' cells
    assert np.abs(o.qdep[:, 0]).sum() * ms.cell_volume() == pytest.approx(got, rel=1e-14)


@pytest.mark.parametrize("levels", [(0,), (1,), (0, 1, 2)])
def test_linear_gather_is_exact_for_a_linear_field(levels):
    ms, st = setup(levels, seed=9)
    o = Oracle(st, dict(scheme=2, back_reaction=False))
    n1, n2, n3 = ms.n
    is_, js, ks = ms.starts
    # a linear field over every block's padded cells (cell centres in global coordinates)
    us = np.zeros(ms.field_shape(3))
    coef = np.array([[0.3, 1.5, -2.0, 0.7], [-0.1, 0.4, 0.9, -1.3], [0.05, -0.6, 0.2, 2.1]])
    for m in range(ms.nmb):
        mb = ms.mb_size[m]
        x = mb[0] + (np.arange(n1) - is_ + 0.5) * mb[6]
        y = mb[1] + (np.arange(n2) - js + 0.5) * mb[7]
        z = mb[2] + (np.arange(n3) - ks + 0.5) * mb[8]
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        for c in range(3):
            us[m, c] = coef[c, 0] + coef[c, 1] * X + coef[c, 2] * Y + coef[c, 3] * Z
    o.arr["ustar"][...] = us
    n = st.npart
    v0 = st.pr[[1, 3, 5], :n].copy()
    a_dt = 1e300                               # c = 1: the kick sets v to the gathered ubar
    o.st.pr[15, :n] = 1.0
    assert o.cloud_gather_kick(a_dt) == 0
    xp = st.pr[[0, 2, 4], :n]
    want = coef[:, :1] + coef[:, 1:] @ xp
    got = o.st.pr[[1, 3, 5], :n]
    # (clouds whose support crosses the periodic wrap see the field's jump there: skip them)
    L = 0.1
    inner = np.all((xp > -L / 2 + 2 * 0.00625) & (xp < L / 2 - 2 * 0.00625), axis=0)
    assert inner.sum() > 100
    assert np.abs(got[:, inner] - want[:, inner]).max() < 1e-12
    assert not np.allclose(got, v0)


@pytest.mark.parametrize("levels", [(0,), (0, 1, 2)])
def test_kick_and_its_impulse_conserve_momentum(levels):
    ms, st = setup(levels, seed=3)
    o = Oracle(st, dict(scheme=2))
    rng = np.random.default_rng(2)
    o.arr["ustar"][...] = rng.standard_normal(o.arr["ustar"].shape) * 0.05
    n = st.npart
    m = st.pr[16, :n]
    p0 = (m * o.st.pr[[1, 3, 5], :n]).sum(axis=1)
    assert o.cloud_gather_kick(2e-3) == 0
    p1 = (m * o.st.pr[[1, 3, 5], :n]).sum(axis=1)
    dg = ms.active(o.arr["dmom"]).sum(axis=(0, 2, 3, 4)) * ms.cell_volume()
    scale = np.abs(p1 - p0).max()
    assert scale > 0 and np.abs((p1 - p0) + dg).max() < 1e-12 * scale
    assert np.abs(o.arr["dmom"]).sum() == pytest.approx(np.abs(ms.active(o.arr["dmom"])).sum())


def test_lobed_codes_are_flagged():
    ms, st = setup((0,))
    st.pi[3, 5] = 1 | (1 << 6)                 # a lobe along x1: a transition cloud
    o = Oracle(st, dict(scheme=2))
    assert o.cloud_deposit_qp(1e-3) == ERR_CLOUD


def lattice_pair():
    """one particle per cell at its centre, gas and dust of uniform (different) velocities"""
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.05], [2.0], 1, placement="lattice", vd=[0.03], gas_noise=0.0)
    return ms, st


def test_cloud_cycle_on_a_lattice_is_the_point_cycle():
    """On a lattice of level-0 clouds every cell gets the same Q and the linear gather of a
    uniform u* is u*: the cloud cycle (overlap split) equals the point-particle TSC cycle
    (centre split), whose damping rate the oracle's known-answer tests pin."""
    ms, st = lattice_pair()
    phys = dict(scheme=2, drag_solver=2)
    oc, op = Oracle(st, phys), Oracle(st, phys)
    for _ in range(4):
        assert oc.cloud_imex_cycle(0.004) == 0
        assert op.imex_cycle(0.004) == 0
    n = st.npart
    for r in (1, 3, 5, 12, 13, 14):
        sc = max(np.abs(op.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(oc.st.pr[r, :n] - op.st.pr[r, :n]).max() < 1e-12 * sc, r
    for v in range(1, 4):
        sc = max(np.abs(op.u0[:, v]).max(), 1e-300)
        assert np.abs(oc.u0[:, v] - op.u0[:, v]).max() < 1e-12 * sc, v


@pytest.mark.parametrize("solver", [0, 2, 3])
def test_cloud_cycles_conserve_momentum(solver):
    ms, st = setup((0, 1, 2), seed=13)
    o = Oracle(st, dict(scheme=2, drag_solver=solver))
    p0 = sum(o.momentum())
    for _ in range(3):
        assert o.cloud_imex_cycle(2e-3) == 0
    p1 = sum(o.momentum())
    n = st.npart
    scale = np.abs(st.pr[16, :n] * np.abs(st.pr[[1, 3, 5], :n]).max(axis=0)).sum()
    assert np.abs(p1 - p0).max() < 1e-13 * scale


# ---- 2-D clouds (LeafApi<LeafTraversal>: cell areas, m (a_dt / (t_s + a_dt)), 9-component pack)
def setup2d(levels=(0,), seed=5, ppc=2):
    ms = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], ppc, seed=seed, vel_noise=0.05,
                    gas_noise=1e-2)
    n = st.npart
    st.pi[3, :n] = np.asarray(levels)[np.arange(n) % len(levels)]
    return ms, st


def test_2d_level0_cloud_deposit_is_the_tsc_deposit_and_keeps_the_mass():
    ms, st = setup2d((0,))
    oc, op = Oracle(st, dict(scheme=2)), Oracle(st, dict(scheme=2))
    a_dt = 1.3e-3
    assert oc.cloud_deposit_qp(a_dt) == 0 and op.deposit_qp(a_dt) == 0
    op.ghost_add("qdep", 5)
    qa, qb = ms.active(oc.qdep)[:, :4], ms.active(op.qdep)[:, :4]
    for v in range(4):
        assert np.abs(qa[:, v] - qb[:, v]).max() < 1e-13 * np.abs(qb[:, v]).max(), v
    ms2, st2 = setup2d((0, 1, 2, 3))
    o = Oracle(st2, dict(scheme=2))
    assert o.cloud_deposit_qp(a_dt) == 0
    n = st2.npart
    want = (st2.pr[16, :n] * (a_dt / (st2.pr[15, :n] + a_dt))).sum()
    got = ms2.active(o.qdep)[:, 0].sum() * ms2.cell_volume()
    assert abs(got - want) < 1e-13 * want


def test_2d_linear_gather_and_lattice_cycle():
    ms, st = setup2d((0, 1, 2), seed=9)
    o = Oracle(st, dict(scheme=2, back_reaction=False))
    n1, n2, _ = ms.n
    is_, js, _ = ms.starts
    us = np.zeros(ms.field_shape(3))
    coef = np.array([[0.3, 1.5, -2.0], [-0.1, 0.4, 0.9], [0.05, -0.6, 0.2]])
    for m in range(ms.nmb):
        mb = ms.mb_size[m]
        x = mb[0] + (np.arange(n1) - is_ + 0.5) * mb[6]
        y = mb[1] + (np.arange(n2) - js + 0.5) * mb[7]
        Y, X = np.meshgrid(y, x, indexing="ij")
        for c in range(3):
            us[m, c, 0] = coef[c, 0] + coef[c, 1] * X + coef[c, 2] * Y
    o.arr["ustar"][...] = us
    n = st.npart
    o.st.pr[15, :n] = 1.0
    assert o.cloud_gather_kick(1e300) == 0
    xp = st.pr[[0, 2], :n]
    want = coef[:, :1] + coef[:, 1:] @ xp
    inner = np.all((xp > -0.5 + 2 / 32) & (xp < 0.5 - 2 / 32), axis=0)
    assert inner.sum() > 100
    assert np.abs(o.st.pr[[1, 3, 5], :n][:, inner] - want[:, inner]).max() < 1e-12
    # the lattice: the cloud cycle is the point cycle
    ms3 = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
    st3 = make_state(ms3, [0.05], [2.0], 1, placement="lattice", vd=[0.03], gas_noise=0.0)
    phys = dict(scheme=2, drag_solver=2)
    oc, op = Oracle(st3, phys), Oracle(st3, phys)
    for _ in range(3):
        assert oc.cloud_imex_cycle(0.01) == 0 and op.imex_cycle(0.01) == 0
    m3 = st3.npart
    for r in (1, 3, 12, 13):
        sc = max(np.abs(op.st.pr[r, :m3]).max(), 1e-300)
        assert np.abs(oc.st.pr[r, :m3] - op.st.pr[r, :m3]).max() < 1e-12 * sc, r


# ---- the clouds' pc2 (CloudPredictorT / CloudAdvanceT) ----
@pytest.mark.parametrize("dims", [3, 2])
def test_cloud_pc2_cycle_on_a_lattice_is_the_point_pc2_cycle(dims):
    if dims == 3:
        ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
        dt = 0.004
    else:
        ms = uniform_mesh((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3)
        dt = 0.01
    st = make_state(ms, [0.05], [2.0], 1, placement="lattice", vd=[0.03], gas_noise=0.0)
    phys = dict(scheme=2)
    oc, op = Oracle(st, phys), Oracle(st, phys)
    for _ in range(3):
        assert oc.cloud_pc2_cycle(dt)[0] == 0 and op.pc2_cycle(dt)[0] == 0
    n = st.npart
    for r in (0, 1, 2, 3, 12, 13):
        sc = max(np.abs(op.st.pr[r, :n]).max(), 1e-300)
        assert np.abs(oc.st.pr[r, :n] - op.st.pr[r, :n]).max() < 1e-12 * sc, r
    for v in range(1, 3):
        sc = max(np.abs(op.u0[:, v]).max(), 1e-300)
        assert np.abs(oc.u0[:, v] - op.u0[:, v]).max() < 1e-12 * sc, v


def test_cloud_pc2_cycles_conserve_momentum():
    ms, st = setup((0, 1, 2), seed=21)
    o = Oracle(st, dict(scheme=2, pc2_feedback_damping=False))
    p0 = sum(o.momentum())
    for _ in range(3):
        assert o.cloud_pc2_cycle(2e-3)[0] == 0
    p1 = sum(o.momentum())
    n = st.npart
    scale = np.abs(st.pr[16, :n] * np.abs(st.pr[[1, 3, 5], :n]).max(axis=0)).sum()
    assert np.abs(p1 - p0).max() < 1e-12 * scale


# ---- clouds at physical x3 faces: the mirrored part ----
def setup_x3(levels=(0, 1), seed=7, x3bc=1):
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3, x3bc=x3bc)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=seed, vel_noise=0.05, gas_noise=1e-2)
    n = st.npart
    st.pi[3, :n] = np.asarray(levels)[np.arange(n) % len(levels)]
    # a share of the clouds within a cell of the x3 faces
    st.pr[4, :n:5] = np.where(np.arange(len(st.pr[4, :n:5])) % 2, 0.05 - 0.004, -0.05 + 0.003)
    st.pr[10, :n] = st.pr[4, :n]
    st.pi[0, :n] = _block_of(ms, st.pr[0, :n], st.pr[2, :n], st.pr[4, :n])
    return ms, st


@pytest.mark.parametrize("x3bc", [1, 2])
def test_clouds_at_physical_x3_faces_keep_their_mass(x3bc):
    """The part of a cloud beyond a physical x3 face comes back as the mirrored part: the
    deposit holds every cloud's whole coupled mass, and nothing lands in a ghost cell."""
    ms, st = setup_x3(x3bc=x3bc)
    o = Oracle(st, dict(scheme=2))
    a_dt = 1.5e-3
    assert o.cloud_deposit_qp(a_dt) == 0
    n = st.npart
    want = (st.pr[16, :n] * a_dt / (st.pr[15, :n] + a_dt)).sum()
    got = ms.active(o.qdep)[:, 0].sum() * ms.cell_volume()
    assert abs(got - want) < 1e-13 * want
    assert np.abs(o.qdep[:, 0]).sum() * ms.cell_volume() == pytest.approx(got, rel=1e-14)


def test_cloud_cycles_at_a_reflecting_face_conserve_momentum():
    ms, st = setup_x3((0, 1, 2), seed=8)
    o = Oracle(st, dict(scheme=2, drag_solver=2))
    p0 = sum(o.momentum())
    for _ in range(3):
        assert o.cloud_imex_cycle(2e-3) == 0
    p1 = sum(o.momentum())
    n = o.st.npart
    scale = np.abs(st.pr[16, :n] * np.abs(st.pr[[1, 3, 5], :n]).max(axis=0)).sum()
    # (x1, x2: exact; x3: the reflections of crossing particles change p_z)
    assert np.abs(p1[:2] - p0[:2]).max() < 1e-12 * scale
