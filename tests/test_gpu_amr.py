"""The general deposit remap on refined meshes, on the GPU against the oracle.

dustb_ghost_add_plan (GeneralApply, src/bvals/bvals_dep_general.cpp:1135-1175) applies the plan
of a refined 3-D mesh; it must equal the oracle's apply bit for bit (the same sums in the same
order, FP64 without contraction).  The point-particle deposit on a refined mesh (every block
deposits with its own cell size) followed by the remap must match the oracle's to 1e-12 of the
field's scale (the deposits are atomic sums), and put the particles' whole coupled mass into
active cells.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from athenak_b200.amr import (build_dep_plan, refined_mesh, refined_state, sphere_refine,
                              X3_FOLD)
from athenak_b200.drag import DeviceDust
from oracle import oracle

pytestmark = pytest.mark.gpu


def _mesh(x3bc=0):
    return refined_mesh((4, 4, 4), (8, 8, 8), 2, refine=sphere_refine((0.1, 0.05, -0.02), (0.3, 0.15)),
                        x3bc=x3bc)


@pytest.mark.parametrize("x3mode", [0, X3_FOLD])
def test_plan_apply_is_bit_exact(x3mode):
    ms = _mesh(0 if x3mode == 0 else 1)
    plan = build_dep_plan(ms, x3mode)
    st = refined_state(ms, [0.1], [1.0], 1, seed=2)
    g = DeviceDust(st, dict(scheme=2))
    g.set_dep_plan(plan)
    a = np.random.default_rng(7).standard_normal(ms.field_shape(3))
    g.t["work"].copy_(torch.from_numpy(a))
    g.ghost_add_plan("work", 3)
    torch.cuda.synchronize()
    ref = oracle.dep_apply(plan, a.copy())
    np.testing.assert_array_equal(g.t["work"].cpu().numpy(), ref)


@pytest.mark.parametrize("scheme", [1, 2])
def test_deposit_and_remap_on_a_refined_mesh(scheme):
    ms = _mesh()
    plan = build_dep_plan(ms, 0)
    st = refined_state(ms, [0.1, 1.0], [0.5, 0.5], 2, seed=4, vd=[0.01, -0.02])
    phys = dict(scheme=scheme, drag_solver=0)
    g = DeviceDust(st, phys)
    g.set_dep_plan(plan)
    o = oracle.Oracle(st, phys)
    a_dt = 0.01
    g.deposit_qp(a_dt)
    g.ghost_add_plan("qdep", 5)
    assert o.deposit_qp(a_dt) == 0
    oracle.dep_apply(plan, o.arr["qdep"])
    torch.cuda.synchronize()
    assert g.error_word() == 0
    q = g.t["qdep"].cpu().numpy()
    gg = ms.ng
    n1, n2, n3 = ms.n
    sl = (slice(None), slice(None), slice(gg, n3 - gg), slice(gg, n2 - gg), slice(gg, n1 - gg))
    qa, qo = q[sl], o.arr["qdep"][sl]
    for v in range(4):
        scale = np.abs(qo[:, v]).max()
        assert np.abs(qa[:, v] - qo[:, v]).max() <= 1e-12 * scale, v
    # the whole coupled mass m c of every particle lands in active cells
    vol = ms.mb_size[:, 6] * ms.mb_size[:, 7] * ms.mb_size[:, 8]
    total = (qa[:, 0].sum(axis=(1, 2, 3)) * vol).sum()
    n = st.npart
    c = a_dt / (st.pr[15, :n] + a_dt)
    want = (st.pr[16, :n] * c).sum()
    assert abs(total - want) <= 1e-12 * want


def test_route_across_levels_matches_the_oracle():
    """SetNewPrtclGID on a refined mesh (src/bvals/bvals_part.cpp:115-471): after a drift of up
    to 0.9 of each particle's own cell width, every particle that left its block is handed to
    the neighbour of whatever level holds it (the device searches the 56 neighbour slots, the
    oracle searches the block boxes), positions wrapped across periodic faces bit for bit."""
    ms = _mesh()
    st = refined_state(ms, [0.1], [1.0], 2, seed=9, vel_noise=0.0)
    n = st.npart
    rng = np.random.default_rng(3)
    m = st.pi[0, :n]
    dx = ms.mb_size[m, 6:9]
    dt = 0.01
    for a, r in enumerate((1, 3, 5)):
        st.pr[r, :n] = rng.uniform(-0.9, 0.9, n) * dx[:, a] / dt
    phys = dict(scheme=2, drag_solver=0)
    g = DeviceDust(st, phys)
    o = oracle.Oracle(st, phys)
    for obj in (g, o):
        obj.register_copy()
        obj.push_imex(1.0, 0.0, dt, 0.0)
        obj.route()
    torch.cuda.synchronize()
    assert g.error_word() == 0
    pi = g.t["pi"].cpu().numpy()[:, :n]
    pr = g.t["pr"].cpu().numpy()[:, :n]
    moved = (pi[0] != st.pi[0, :n]).sum()
    assert moved > n // 20
    np.testing.assert_array_equal(pi[0], o.arr["pi"][0, :n])
    np.testing.assert_array_equal(pr, o.arr["pr"][:, :n])
    # every particle inside its new block's box
    mb = ms.mb_size[pi[0]]
    for a, r in enumerate((0, 2, 4)):
        assert ((pr[r] >= mb[:, a]) & (pr[r] < mb[:, 3 + a])).all()
    # and the levels differ where particles changed blocks
    lev = ms.lloc[:, 0]
    assert (lev[pi[0]] != lev[st.pi[0, :n]]).sum() > 0


def test_refined_copy_exchange_is_bit_exact():
    """dustb_ghost_copy_ml (restriction, the 56-slot exchange, coarse-buffer fill, min-mod
    prolongation) equals the oracle's sender-side restatement bit for bit on a random field."""
    ms = _mesh()
    st = refined_state(ms, [0.1], [1.0], 1, seed=2)
    g = DeviceDust(st, dict(scheme=2))
    o = oracle.Oracle(st, dict(scheme=2))
    a = np.random.default_rng(11).standard_normal(ms.field_shape(3))
    g.t["work"].copy_(torch.from_numpy(a))
    o.arr["work"][...] = a
    g.ghost_copy_ml("work", 3)
    o.ghost_copy_ml("work", 3)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(g.t["work"].cpu().numpy(), o.arr["work"])


def _refined_cycle(obj, plan, dt, gpu):
    """One imex2+ cycle of the point-particle drag on a refined mesh, task by task in the order
    of AssembleDustGasDragTasks (src/dust/dust_tasks.cpp:38-120) with the local solver (the
    reference's point particles on a refined 3-D mesh): the deposits exchanged by the general
    remap, u* and the gas state by the multilevel copy exchange."""
    g0, g1, beta, atw22 = oracle.imex2p_coeffs(oracle.GAMMA_DEFAULT)
    a_dt = oracle.GAMMA_DEFAULT * dt

    def add(name, nvar):
        if gpu:
            obj.ghost_add_plan(name, nvar)
        else:
            oracle.dep_apply(plan, obj.arr[name])

    err = 0
    for stage in (1, 2):
        if stage == 1:
            obj.register_copy()
        obj.gas_rk_noflux(g0[stage - 1], g1[stage - 1])
        if stage == 2:
            obj.history_gas(atw22 * dt)
        obj.push_imex(g0[stage - 1], g1[stage - 1], beta[stage - 1] * dt,
                      atw22 * dt if stage == 2 else 0.0)
        r = obj.route()
        err |= 0 if gpu else r
        r = obj.deposit_qp(a_dt)
        err |= 0 if gpu else r
        add("qdep", 5)
        obj.solve_ustar()
        obj.ghost_copy_ml("ustar", 3)
        r = obj.gather_kick_pmbr(a_dt)
        err |= 0 if gpu else r
        add("dmom", 3)
        obj.apply_pmbr(a_dt)
        obj.ghost_copy_ml("u0", 4)
    return err


def _total_momentum(ms, pr, u0, npart):
    vol = ms.mb_size[:, 6] * ms.mb_size[:, 7] * ms.mb_size[:, 8]
    g_ = ms.ng
    n1, n2, n3 = ms.n
    act = u0[:, 1:4, g_:n3 - g_, g_:n2 - g_, g_:n1 - g_].sum(axis=(2, 3, 4))
    gas = (act * vol[:, None]).sum(axis=0)
    m = pr[16, :npart]
    dust = np.array([(m * pr[r, :npart]).sum() for r in (1, 3, 5)])
    return gas + dust


def test_refined_imex_cycles_match_the_oracle():
    """Two imex2+ cycles of the FP64 drag step on a refined mesh (two levels above the root, the
    consistent split, TSC, local solver): the GPU task sequence matches the oracle's (particles
    and gas within 1e-12 of their scale, block ids exact: particles cross between levels),
    and total gas + dust momentum is unchanged to round-off."""
    ms = _mesh()
    plan = build_dep_plan(ms, 0)
    st = refined_state(ms, [0.01, 0.3], [0.5, 1.0], 2, seed=6, vd=[0.8, -0.5],
                       vel_noise=0.2, gas_noise=0.05)
    phys = dict(scheme=2, drag_solver=0, consistent_gas=True)
    g = DeviceDust(st, phys)
    g.set_dep_plan(plan)
    o = oracle.Oracle(st, phys)
    # the smallest cell and the fastest particle set dt (a CFL of 0.3)
    dxmin = ms.mb_size[:, 6].min()
    dt = 0.3 * dxmin / np.abs(st.pr[[1, 3, 5], :st.npart]).max()
    p0 = _total_momentum(ms, st.pr, st.u0, st.npart)
    n = st.npart
    for _ in range(2):
        _refined_cycle(g, plan, dt, True)
        assert _refined_cycle(o, plan, dt, False) == 0
    torch.cuda.synchronize()
    assert g.error_word() == 0
    pr, pi = g.host("pr"), g.host("pi")
    np.testing.assert_array_equal(pi[0], o.arr["pi"][0, :n])
    assert (pi[0] != st.pi[0, :n]).sum() > 0
    for r in range(16):
        sc = max(np.abs(o.arr["pr"][r, :n]).max(), 1e-300)
        assert np.abs(pr[r] - o.arr["pr"][r, :n]).max() <= 1e-12 * sc, r
    u = g.t["u0"].cpu().numpy()
    for v in range(4):
        sc = np.abs(o.arr["u0"][:, v]).max()
        assert np.abs(u[:, v] - o.arr["u0"][:, v]).max() <= 1e-12 * sc, v
    p1 = _total_momentum(ms, pr, u, n)
    absm = np.abs(st.pr[16, :n] * np.abs(st.pr[[1, 3, 5], :n])).sum()
    assert np.abs(p1 - p0).max() <= 1e-12 * absm


@pytest.mark.parametrize("solver", [0, 2])
def test_fused_refined_cycle_equals_the_task_sequence(solver):
    """dustb_refined_imex_cycle (one launch sequence per cycle) gives what the task sequence
    gives, for the local solver and dc1 (its sweeps exchange u* and the operator's deposits
    across levels), and the FP64 dc1 cycle matches the oracle's task sequence with dc1."""
    ms = _mesh()
    plan = build_dep_plan(ms, 0)
    st = refined_state(ms, [0.01, 0.3], [0.5, 1.0], 2, seed=8, vd=[0.8, -0.5],
                       vel_noise=0.2, gas_noise=0.05)
    phys = dict(scheme=2, drag_solver=solver, consistent_gas=True)
    a = DeviceDust(st, phys)
    a.set_dep_plan(plan)
    dxmin = ms.mb_size[:, 6].min()
    dt = 0.3 * dxmin / np.abs(st.pr[[1, 3, 5], :st.npart]).max()
    for _ in range(2):
        a.refined_imex_cycle(dt)
    torch.cuda.synchronize()
    assert a.error_word() == 0
    if solver == 0:
        b = DeviceDust(st, phys)
        b.set_dep_plan(plan)
        for _ in range(2):
            _refined_cycle(b, plan, dt, True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(a.host("pi")[0], b.host("pi")[0])
        for r in range(16):
            sc = max(np.abs(b.host("pr")[r]).max(), 1e-300)
            assert np.abs(a.host("pr")[r] - b.host("pr")[r]).max() <= 1e-12 * sc, r
        return
    # dc1 against the oracle's tasks with the refined exchanges around its operator
    o = oracle.Oracle(st, phys)
    g0, g1, beta, atw22 = oracle.imex2p_coeffs(oracle.GAMMA_DEFAULT)
    a_dt = oracle.GAMMA_DEFAULT * dt
    L = oracle.lib()
    for _ in range(2):
        for stage in (1, 2):
            if stage == 1:
                o.register_copy()
            o.gas_rk_noflux(g0[stage - 1], g1[stage - 1])
            if stage == 2:
                o.history_gas(atw22 * dt)
            o.push_imex(g0[stage - 1], g1[stage - 1], beta[stage - 1] * dt,
                        atw22 * dt if stage == 2 else 0.0)
            assert o.route() == 0
            assert o.deposit_qp(a_dt) == 0
            oracle.dep_apply(plan, o.arr["qdep"])
            o.solve_ustar()
            o.ghost_copy_ml("ustar", 3)
            o.arr["work"][...] = 0.0
            assert L.oracle_operator_particles(C.byref(o.ctx), a_dt) == 0
            oracle.dep_apply(plan, o.arr["work"])
            L.oracle_dc_correct(C.byref(o.ctx))
            o.ghost_copy_ml("ustar", 3)
            assert o.gather_kick_pmbr(a_dt) == 0
            oracle.dep_apply(plan, o.arr["dmom"])
            o.apply_pmbr(a_dt)
            o.ghost_copy_ml("u0", 4)
    n = st.npart
    np.testing.assert_array_equal(a.host("pi")[0], o.arr["pi"][0, :n])
    for r in range(16):
        sc = max(np.abs(o.arr["pr"][r, :n]).max(), 1e-300)
        assert np.abs(a.host("pr")[r] - o.arr["pr"][r, :n]).max() <= 1e-12 * sc, r


def test_mixed_form_on_a_refined_mesh():
    """The mixed-precision imex2+ cycle on a refined mesh (per-level cell sizes, the push carrying
    particles between levels in cell units, the tiles on each block's own ghost cells with the
    general remap and the multilevel copy exchange around them) against the FP64 refined cycle:
    every particle velocity within 1e-5 of the largest, positions within 1e-5 of a cell of the
    particle's level, block ids equal, the gas momentum within 1e-5 of its scale; total gas +
    dust momentum conserved to round-off (the momentum ledgers with per-level volumes)."""
    from athenak_b200.mixed import MixedDust
    ms = _mesh()
    plan = build_dep_plan(ms, 0)
    st = refined_state(ms, [0.01, 0.3], [0.5, 1.0], 2, seed=6, vd=[0.8, -0.5],
                       vel_noise=0.2, gas_noise=0.05)
    phys = dict(scheme=2, drag_solver=0, consistent_gas=True)
    ref = DeviceDust(st, phys)
    ref.set_dep_plan(plan)
    dev = DeviceDust(st, phys)
    dev.set_dep_plan(plan)
    mx = MixedDust(dev=dev)
    mx.export()
    torch.cuda.synchronize()
    n = st.npart
    p0 = _total_momentum(ms, dev.host("pr"), dev.t["u0"].cpu().numpy(), n)
    dxmin = ms.mb_size[:, 6].min()
    dt = 0.3 * dxmin / np.abs(st.pr[[1, 3, 5], :n]).max()
    cycles = 3
    for _ in range(cycles):
        ref.refined_imex_cycle(dt)
        mx.imex_cycle(dt)
    mx.export()
    torch.cuda.synchronize()
    assert ref.error_word() == 0 and dev.error_word() == 0
    a, b = dev.host("pr"), ref.host("pr")
    pa, pb = dev.host("pi"), ref.host("pi")
    np.testing.assert_array_equal(pa[0], pb[0])
    assert (pa[0] != st.pi[0, :n]).sum() > 0
    vscale = np.abs(b[[1, 3, 5]]).max()
    for r in (1, 3, 5):
        assert np.abs(a[r] - b[r]).max() < 1e-5 * vscale, r
    dxp = ms.mb_size[pb[0], 6:9]
    for r, ax in ((0, 0), (2, 1), (4, 2)):
        assert (np.abs(a[r] - b[r]) < 1e-5 * dxp[:, ax]).all(), r
    ua, ub = dev.t["u0"].cpu().numpy(), ref.t["u0"].cpu().numpy()
    for v in range(1, 4):
        sc = np.abs(ub[:, v]).max()
        assert np.abs(ua[:, v] - ub[:, v]).max() < 1e-5 * sc, v
    p1 = _total_momentum(ms, a, ua, n)
    absm = np.abs(st.pr[16, :n] * np.abs(st.pr[[1, 3, 5], :n])).sum()
    assert np.abs(p1 - p0).max() <= 1e-12 * cycles * absm
