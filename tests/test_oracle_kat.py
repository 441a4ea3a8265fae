"""CPU checks of the oracle against the reference's known-answer tests and against
independent numpy restatements (no GPU needed).

Pins (the reference ships no golden output files):
* dust_damping ODE (src/pgen/tests/dust_damping.cpp:9-16): mean gas/dust velocities of the
  lattice set-up follow the linear ODE; the error must fall by > 2.5 when dt halves and the
  total momentum must hold to < 1e-12 (tst/test_suite/dust/check_cloud_imex3d.py:66-74,
  :112-121), for a resolved and a stiff (t_s = 1e-4) species mixture;
* the committed damping-ODE fixture tests/golden/damping_ode.json (make_golden.py);
* exact momentum conservation with random placement (dust_pm.cpp:17-21, :545-563);
* the NSH drift used by the generator solves the steady equations (dust_setup.hpp:58-65).
"""
import json
import os

import numpy as np
import pytest

from athenak_b200.mesh import uniform_mesh
from athenak_b200.inputs import make_state, nsh_gas, nsh_dust, hash_uniform01
from oracle.oracle import Oracle, GAMMA_DEFAULT

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def damping_run(dt, taus, eps, vd, tlim, nb=(8, 8, 1), ncells=(16, 16, 1)):
    ms = uniform_mesh(ncells, nb, 2, (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
    st = make_state(ms, taus, eps, 1, placement="lattice", vd=vd, gas_noise=0.0)
    o = Oracle(st, dict(scheme=2, drag_solver=2))
    n = int(round(tlim / dt))
    g0, d0 = o.momentum()
    for _ in range(n):
        assert o.imex_cycle(dt) == 0
    g1, d1 = o.momentum()
    u = o.mesh.active(o.u0)[:, 1].mean()
    pr, sp = o.st.pr, o.st.pi[2, :o.st.npart]
    v = [pr[1, :o.st.npart][sp == s].mean() for s in range(len(taus))]
    return np.array([u] + v), np.abs((g1 + d1) - (g0 + d0)).max(), n * dt


def ode_solution(taus, eps, vd, t):
    from scipy.linalg import expm
    N = len(taus)
    A = np.zeros((N + 1, N + 1))
    for s in range(N):
        A[0, 0] -= eps[s] / taus[s]
        A[0, 1 + s] += eps[s] / taus[s]
        A[1 + s, 1 + s] = -1.0 / taus[s]
        A[1 + s, 0] = 1.0 / taus[s]
    return expm(A * t) @ np.array([0.0] + list(vd))


@pytest.mark.parametrize("stiff", [False, True])
def test_damping_ode_convergence_and_conservation(stiff):
    taus = [1e-4 if stiff else 0.1, 0.03, 1.0]
    eps = [0.2, 0.5, 0.3]
    vd = [0.01 / 3, 0.02 / 3, 0.01]
    dt = 0.4 / 16
    y1, dp1, t1 = damping_run(dt, taus, eps, vd, 0.2)
    y2, dp2, t2 = damping_run(dt / 2, taus, eps, vd, 0.2)
    ex = ode_solution(taus, eps, vd, t1)
    e1 = np.abs(y1 - ex).max()
    e2 = np.abs(y2 - ex).max()
    assert dp1 < 1e-12 and dp2 < 1e-12
    assert e1 / e2 > 2.5, (e1, e2)
    assert e1 < 1e-4


def test_damping_matches_golden_fixture():
    with open(os.path.join(GOLDEN, "damping_ode.json")) as f:
        g = json.load(f)
    for case in g["cases"]:
        y, dp, t = damping_run(case["dt"], case["taus"], case["eps"], case["vd"], case["tlim"])
        exact = np.array(case["exact"])
        assert abs(t - case["t"]) < 1e-14
        assert np.abs(y - exact).max() < case["max_err"], (y, exact)
        assert dp < 1e-12


def test_ode_fixture_is_the_ode():
    with open(os.path.join(GOLDEN, "damping_ode.json")) as f:
        g = json.load(f)
    for case in g["cases"]:
        ex = ode_solution(case["taus"], case["eps"], case["vd"], case["t"])
        np.testing.assert_allclose(ex, case["exact"], rtol=1e-12, atol=1e-15)


def test_random_3d_conservation_multiblock():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1, 1.0], [0.5, 0.5, 0.5], 1, seed=3, vd=[0.1, -0.2, 0.3],
                    gas_noise=1e-2, vel_noise=0.05)
    o = Oracle(st, dict(scheme=2, drag_solver=2))
    g0, d0 = o.momentum()
    tot0 = g0 + d0
    for _ in range(3):
        assert o.imex_cycle(2e-3) == 0
    g1, d1 = o.momentum()
    scale = np.abs(g0).max() + np.abs(d0).max()
    assert np.abs((g1 + d1) - tot0).max() < 1e-13 * scale
    # drag moved momentum between the phases
    assert np.abs(d1 - d0).max() > 1e-6 * scale


def test_pc2_conservation():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1], [1.0, 0.5], 1, seed=5, vd=[0.1, -0.2], gas_noise=1e-2,
                    vel_noise=0.05)
    o = Oracle(st, dict(scheme=2))
    g0, d0 = o.momentum()
    for _ in range(2):
        err, chi = o.pc2_cycle(2e-3)
        assert err == 0 and chi > 0.0
    g1, d1 = o.momentum()
    scale = np.abs(g0).max() + np.abs(d0).max()
    assert np.abs((g1 + d1) - (g0 + d0)).max() < 1e-13 * scale


def test_nsh_drift_is_steady():
    om, q, ax = 1.0, 1.5, 0.1
    taus, eps = [0.01, 0.1, 1.0, 10.0], [0.5] * 4
    ugx, ugp = nsh_gas(om, q, ax, eps, taus)
    tot_x, tot_p = ugx, ugp
    for t, e in zip(taus, eps):
        vx, vp = nsh_dust(om, q, t, ugx, ugp)
        # dust steady state: 2 Om vp - (vx - ugx)/t = 0, -(2-q) Om vx - (vp - ugp)/t = 0
        assert abs(2 * om * vp - (vx - ugx) / t) < 1e-12
        assert abs(-(2 - q) * om * vx - (vp - ugp) / t) < 1e-12
        tot_x += e * vx
        tot_p += e * vp
    # gas steady state with forcing: total radial momentum zero, 2 Om (u_p + sum e v_p) = -ax
    assert abs(tot_x) < 1e-12 and abs(2 * om * tot_p + ax) < 1e-12


def test_hash_uniform_known_values():
    # SplitMix64 finaliser of key 0 (the published SplitMix64 output for state 0)
    z = (0x9E3779B97F4A7C15 ^ (0x9E3779B97F4A7C15 >> 30)) * 0xBF58476D1CE4E5B9 % 2**64
    z = (z ^ (z >> 27)) * 0x94D049BB133111EB % 2**64
    z ^= z >> 31
    assert z == 0xE220A8397B1DCDAF
    assert hash_uniform01(np.array([0], np.uint64))[0] == (z >> 11) / 2.0**53


# ---- independent restatements of the exchanges and the sort ---------------------------

def global_fold(ms, a):
    """Periodic fold of every cell of (nmb, nvar, n3, n2, n1) arrays onto the global mesh."""
    nb = ms.nblocks
    N = [ms.nx[i] * nb[i] for i in range(3)]
    nvar = a.shape[1]
    n1, n2, n3 = ms.n
    g = np.zeros((nvar, N[2], N[1], N[0]))
    is_, js, ks = ms.starts
    for m in range(ms.nmb):
        bi, bj, bk = m % nb[0], (m // nb[0]) % nb[1], m // (nb[0] * nb[1])
        I = (np.arange(n1) - is_ + bi * ms.nx[0]) % N[0]
        J = (np.arange(n2) - js + bj * ms.nx[1]) % N[1]
        K = (np.arange(n3) - ks + bk * ms.nx[2]) % N[2]
        np.add.at(g, (slice(None), K[:, None, None], J[None, :, None], I[None, None, :]), a[m])
    return g


def global_active(ms, a):
    nb = ms.nblocks
    N = [ms.nx[i] * nb[i] for i in range(3)]
    g = np.zeros((a.shape[1], N[2], N[1], N[0]))
    act = ms.active(a)
    for m in range(ms.nmb):
        bi, bj, bk = m % nb[0], (m // nb[0]) % nb[1], m // (nb[0] * nb[1])
        g[:, bk * ms.nx[2]:(bk + 1) * ms.nx[2], bj * ms.nx[1]:(bj + 1) * ms.nx[1],
          bi * ms.nx[0]:(bi + 1) * ms.nx[0]] = act[m]
    return g


@pytest.mark.parametrize("shape", [((16, 16, 16), (8, 8, 8)), ((12, 8, 1), (4, 4, 1)),
                                   ((8, 8, 8), (8, 4, 8))])
def test_ghost_add_is_periodic_fold(shape):
    ms = uniform_mesh(shape[0], shape[1], 2)
    st = make_state(ms, [0.1], [1.0], 1)
    o = Oracle(st, dict())
    rng = np.random.default_rng(0)
    o.qdep[...] = rng.standard_normal(o.qdep.shape)
    expect = global_fold(ms, o.qdep)
    o.ghost_add("qdep", 5)
    np.testing.assert_allclose(global_active(ms, o.qdep), expect, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("shape", [((16, 16, 16), (8, 8, 8)), ((12, 8, 1), (4, 4, 1))])
def test_ghost_copy_fills_periodic_images(shape):
    ms = uniform_mesh(shape[0], shape[1], 2)
    st = make_state(ms, [0.1], [1.0], 1)
    o = Oracle(st, dict())
    rng = np.random.default_rng(1)
    o.ustar[...] = rng.standard_normal(o.ustar.shape)
    g = global_active(ms, o.ustar)
    o.ghost_copy("ustar", 3)
    nb = ms.nblocks
    N = [ms.nx[i] * nb[i] for i in range(3)]
    n1, n2, n3 = ms.n
    is_, js, ks = ms.starts
    for m in range(ms.nmb):
        bi, bj, bk = m % nb[0], (m // nb[0]) % nb[1], m // (nb[0] * nb[1])
        I = (np.arange(n1) - is_ + bi * ms.nx[0]) % N[0]
        J = (np.arange(n2) - js + bj * ms.nx[1]) % N[1]
        K = (np.arange(n3) - ks + bk * ms.nx[2]) % N[2]
        np.testing.assert_array_equal(o.ustar[m], g[:, K[:, None, None], J[None, :, None], I[None, None, :]])


def test_sort_order_is_lexicographic():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2)
    st = make_state(ms, [0.1, 1.0], [0.5, 0.5], 2, seed=7)
    o = Oracle(st, dict())
    order, keys = o.sort_order()
    n = st.npart
    pr, pi = st.pr, st.pi
    mb = ms.mb_size
    m = pi[0, :n]
    i = np.clip(np.floor((pr[0, :n] - mb[m, 0]) / mb[m, 6]).astype(np.int64), 0, 7)
    j = np.clip(np.floor((pr[2, :n] - mb[m, 1]) / mb[m, 7]).astype(np.int64), 0, 7)
    k = np.clip(np.floor((pr[4, :n] - mb[m, 2]) / mb[m, 8]).astype(np.int64), 0, 7)
    key = m.astype(np.int64) * 512 + (k * 8 + j) * 8 + i
    np.testing.assert_array_equal(keys, key)
    np.testing.assert_array_equal(order, np.lexsort((np.arange(n), key)))
    o.sort_particles()
    np.testing.assert_array_equal(o.st.pi[1, :n], st.pi[1, order])


def test_cloud_order_index_tags_and_check():
    """UpdateCloudOrder (src/dust/dust_cloud_device.cpp:1992-2055): the index is the sort's
    permutation, each slot's tag is TagFromWords(PTAG, PTAGH) (src/athena.hpp:85-88, the words
    as unsigned 32-bit), and the check counts the slots whose particle changed."""
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2)
    st = make_state(ms, [0.1, 1.0], [0.5, 0.5], 2, seed=7)
    n = st.npart
    # tags beyond 2^31: negative low words and nonzero high words
    st.pi[1, :n:3] = -1 - np.arange(len(st.pi[1, :n:3]), dtype=np.int32)
    st.pi[4, :n:5] = 7
    st.pi[4, 1:n:7] = -2
    o = Oracle(st, dict())
    ord_, tag = o.cloud_order()
    order, _ = o.sort_order()
    np.testing.assert_array_equal(ord_, order)
    lo = st.pi[1, :n].astype(np.int64) & 0xFFFFFFFF
    hi = st.pi[4, :n].astype(np.int64) & 0xFFFFFFFF
    want = (hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)
    np.testing.assert_array_equal(tag, want[order])
    assert o.cloud_order_check(ord_, tag) == 0
    # reordered rows: every slot whose particle moved fails; out-of-range slots fail
    o.sort_particles()
    moved = int((order != np.arange(n)).sum())
    assert moved > 0 and o.cloud_order_check(ord_, tag) == moved
    # the identity index of the sorted rows carries the same tags (the sort's identity)
    ident = np.arange(n, dtype=np.int32)
    assert o.cloud_order_check(ident, tag) == 0
    ident[:3] = [-1, n, n + 5]
    assert o.cloud_order_check(ident, tag) == 3


def test_route_keeps_particles_in_their_blocks():
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1], [1.0], 2, seed=11, vel_noise=0.5)
    o = Oracle(st, dict())
    tags0 = o.st.pi[1, :st.npart].copy()
    # a push of up to ~0.6 cells moves many particles across block faces and the mesh edge
    o.register_copy()
    o.push_imex(1.0, 0.0, 2e-3, 0.0)
    assert o.route() == 0
    n = st.npart
    pr, pi, mb = o.st.pr, o.st.pi, ms.mb_size
    m = pi[0, :n]
    for a, (lo, hi) in enumerate(((0, 3), (1, 4), (2, 5))):
        x = pr[2 * a, :n]
        assert np.all(x >= mb[m, lo]) and np.all(x < mb[m, hi])
    np.testing.assert_array_equal(pi[1, :n], tags0)


@pytest.mark.parametrize("drop", [False, True])
def test_x3_fold_conserves_the_deposit(drop):
    """Physical x3 faces: folding the ghost deposits beyond a face back into the mirrored
    active cells (<dust>/x3_ghost_deposit = fold) keeps every particle's whole deposit
    (sum of Q over the active cells = sum of m c); dropping them (= drop) loses the part
    beyond the faces."""
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3, x3bc=1)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=7)
    o = Oracle(st, dict(scheme=2, x3_deposit_drop=drop))
    a_dt = 1e-3
    o.deposit_qp(a_dt)
    o.ghost_add("qdep", 5)
    q = ms.active(o.qdep)[:, 0].sum() * ms.cell_volume()
    n = st.npart
    expect = (st.pr[16, :n] * a_dt / (st.pr[15, :n] + a_dt)).sum()
    if drop:
        assert q < expect * (1.0 - 1e-3)
    else:
        assert abs(q - expect) < 1e-13 * expect


def shear_mesh(x3bc=0):
    return uniform_mesh((16, 32, 16), (8, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05),
                        x3bc=x3bc, shear_x1=True)


def test_shear_remap_of_ghost_strips_shifts_the_profile():
    """Shear-periodic x1 faces: after the plain periodic copy the x1 ghost strips are
    remapped (PLM) by the shear offset q Omega Lx t: the inner strip holds the outer edge's
    profile shifted by +offset in x2, the outer strip the inner edge's by -offset."""
    ms = shear_mesh()
    st = make_state(ms, [0.1], [1.0], 1, seed=2)
    o = Oracle(st, dict(scheme=2, shearing_box=True))
    t = 0.37
    o.set_time(t)
    N2 = 32
    dy = 0.2 / N2
    s_cells = 1.5 * 1.0 * 0.1 * t / dy                      # q Omega Lx t / dy
    is_, js, ks = ms.starts
    u = o.ustar
    for m in range(ms.nmb):
        b2 = int(round((ms.mb_size[m, 1] + 0.1) / (0.2 / 4)))
        rows = b2 * 8 + np.arange(-js, 8 + js)
        u[m, :, :, :, :] = np.sin(2 * np.pi * (rows + 0.5) / N2)[None, None, :, None]
    o.ghost_copy("ustar", 3, 0)
    for m in range(ms.nmb):
        b2 = int(round((ms.mb_size[m, 1] + 0.1) / (0.2 / 4)))
        rows = b2 * 8 + np.arange(-js, 8 + js)
        if ms.mb_size[m, 0] < -0.05 + 0.025:                # inner face: shifted by +s
            want = np.sin(2 * np.pi * (rows + 0.5 - s_cells) / N2)
            got = u[m, 0, ks, :, 0]
        elif ms.mb_size[m, 3] > 0.05 - 0.025:                # outer face: shifted by -s
            want = np.sin(2 * np.pi * (rows + 0.5 + s_cells) / N2)
            got = u[m, 0, ks, :, -1]
        else:
            continue
        assert np.abs(got - want).max() < 2e-2


@pytest.mark.parametrize("t", [0.73, 1.32])
@pytest.mark.parametrize("x3bc", [0, 1])
def test_shear_deposit_remap_conserves(x3bc, t):
    """The ghost deposits beyond the shear-periodic x1 faces are moved to the other face and
    shifted by the particles' shear offset (piecewise-constant overlaps): the total deposit
    is kept exactly.  t = 1.32 puts the offset 31.68 of 32 cells, within the ghost width of
    a full period, where the sources of a target cell include the ghost rows of the block
    column on the far side of the periodic x2 wrap."""
    ms = shear_mesh(x3bc)
    st = make_state(ms, [0.1, 0.01], [1.0, 0.5], 2, seed=11)
    o = Oracle(st, dict(scheme=2, shearing_box=True))
    o.set_time(t)
    a_dt = 1e-3
    o.deposit_qp(a_dt)
    o.ghost_add("qdep", 5)
    q = ms.active(o.qdep)[:, 0].sum() * ms.cell_volume()
    n = st.npart
    expect = (st.pr[16, :n] * a_dt / (st.pr[15, :n] + a_dt)).sum()
    assert abs(q - expect) < 1e-13 * expect


def test_shear_route_shifts_radial_crossers():
    """A particle leaving through the outer x1 face re-enters at the inner face shifted by
    +fmod(q Omega Lx t, Ly) in x2 (its register with it), routed to the inner-face block at
    the new x2; one leaving through the inner face the other way."""
    ms = shear_mesh()
    st = make_state(ms, [0.1], [1.0], 1, seed=5)
    o = Oracle(st, dict(scheme=2, shearing_box=True))
    t = 2.9
    o.set_time(t)
    ysh = np.fmod(1.5 * 1.0 * 0.1 * t, 0.2)
    n = o.st.npart
    pr, pi = o.st.pr, o.st.pi
    # two particles: one just past the outer face of an outer block, one past the inner face
    outer = [m for m in range(ms.nmb) if ms.mb_size[m, 3] > 0.05 - 0.025]
    inner = [m for m in range(ms.nmb) if ms.mb_size[m, 0] < -0.05 + 0.025]
    p0, p1 = 0, 1
    for p, m, x in ((p0, outer[3], 0.05 + 1e-4), (p1, inner[5], -0.05 - 1e-4)):
        pi[0, p] = m
        pr[0, p] = x
        pr[2, p] = 0.5 * (ms.mb_size[m, 1] + ms.mb_size[m, 4])
        pr[4, p] = 0.5 * (ms.mb_size[m, 2] + ms.mb_size[m, 5])
        pr[6, p], pr[8, p], pr[10, p] = pr[0, p], pr[2, p], pr[4, p]
    y0 = pr[2, [p0, p1]].copy()
    assert o.route() == 0
    def wrap(y):
        return (y + 0.1) % 0.2 - 0.1
    assert abs(pr[2, p0] - wrap(y0[0] + ysh)) < 1e-12
    assert abs(pr[2, p1] - wrap(y0[1] - ysh)) < 1e-12
    assert abs(pr[0, p0] - (0.05 + 1e-4 - 0.1)) < 1e-15 and abs(pr[0, p1] - (-0.05 - 1e-4 + 0.1)) < 1e-15
    for p in (p0, p1):
        m = pi[0, p]
        assert ms.mb_size[m, 0] <= pr[0, p] < ms.mb_size[m, 3]
        assert ms.mb_size[m, 1] <= pr[2, p] < ms.mb_size[m, 4]
        assert pr[8, p] - pr[2, p] == 0.0 or abs(pr[8, p] - pr[2, p]) < 1e-12
