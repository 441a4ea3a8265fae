"""Refinable clouds on refined 3-D meshes on the GPU against the oracle.

The leaf traversal (LeafTraversal3D::ForEach over the actual leaves, transition lobes, the
mirrored part at physical x3 faces), the clouds' deposit and gather-kick, the instant switch,
the P1 split and the imex2+ cycle of clouds on a refined mesh (dustb_cloud_*, mesh.leaf set)
must match the oracle's restatement: the gathers and the kicked velocities bit for bit (the
same sums in the same order, FP64 without contraction), the deposits to 1e-12 of their scale
(atomic sums), the split's rows and the switched codes exactly, and two cycles to 1e-12.
"""
import numpy as np
import pytest
import torch

from athenak_b200 import capi
from athenak_b200.amr import leaf_tables, refined_mesh, refined_state, sphere_refine
from athenak_b200.drag import DeviceDust
from oracle import oracle

pytestmark = pytest.mark.gpu


def _mesh(x3bc=0):
    return refined_mesh((4, 4, 4), (8, 8, 8), 2, refine=sphere_refine((0.1, 0.05, -0.02), (0.3, 0.15)),
                        x3bc=x3bc)


def _codes(st, lt, mode, seed=3):
    rng = np.random.default_rng(seed)
    n = st.npart
    if mode == "block":
        code = lt.arrays["blev"][st.pi[0, :n]]
    else:
        code = rng.integers(0, lt.nlev + 1, n)
        lob = rng.integers(0, 4, (3, n)) * (code > 0)
        code = code | (lob[0] << 6) | (lob[1] << 4) | (lob[2] << 9)
    st.pi[3, :n] = code.astype(np.int32)


def _pair(ms, st, phys):
    lt = leaf_tables(ms)
    lo = leaf_tables(ms, builder=oracle.lib().oracle_leaf_tables)
    g = DeviceDust(st, phys)
    g.set_leaf_tables(lt)
    o = oracle.Oracle(st, phys)
    o.set_leaf_tables(lo)
    return g, o


@pytest.mark.parametrize("mode", ["block", "lobed"])
@pytest.mark.parametrize("x3bc", [0, 1])
def test_leaf_deposit_and_gather_kick_match_the_oracle(mode, x3bc):
    ms = _mesh(x3bc)
    st = refined_state(ms, [0.1, 1.0], [0.5, 1.0], 1, seed=5, vel_noise=0.2, gas_noise=0.1)
    _codes(st, leaf_tables(ms), mode)
    phys = dict(scheme=2)
    g, o = _pair(ms, st, phys)
    a_dt = 0.05
    g.cloud_deposit_qp(a_dt)
    assert o.cloud_deposit_qp(a_dt) == 0
    torch.cuda.synchronize()
    assert g.error_word() == 0
    q = g.t["qdep"].cpu().numpy()
    assert np.abs(q - o.arr["qdep"]).max() <= 1e-12 * np.abs(o.arr["qdep"]).max()
    us = st.u0[:, 1:4] / st.u0[:, 0:1]
    g.t["ustar"].copy_(torch.from_numpy(us))
    o.arr["ustar"][:] = us
    gp = g.cloud_gather_kick(a_dt)
    assert o.cloud_gather_kick(a_dt, gp=gp.cpu().numpy().reshape(ms.nmb, *ms.n[::-1], 12)) == 0
    torch.cuda.synchronize()
    assert g.error_word() == 0
    n = st.npart
    pr = g.host("pr")
    for r in (1, 3, 5, 12, 13, 14):
        np.testing.assert_array_equal(pr[r, :n], o.st.pr[r, :n], err_msg=str(r))
    dm = g.t["dmom"].cpu().numpy()
    assert np.abs(dm - o.arr["dmom"]).max() <= 1e-12 * np.abs(o.arr["dmom"]).max()


def test_split_and_instant_switch_match_the_oracle():
    # 2^3 root blocks refined twice (levels 1 and 2), root clouds split pass by pass
    ms = refined_mesh((2, 2, 2), (8, 8, 8), 2, refine=sphere_refine((0.1, 0.05, -0.02), (0.45, 0.2)),
                      x3bc=1)
    st = refined_state(ms, [0.1], [0.5], 1, seed=12, vel_noise=0.2)
    st.pi[3, :st.npart] = 0
    phys = dict(scheme=2)
    g, o = _pair(ms, st, phys)
    sp = capi.split_params(max_level=1)       # the split stops at level 1
    tag = st.npart
    for _ in range(4):
        n_g = g.cloud_split_p1(sp, tag)
        n_o = o.cloud_split_p1(sp, tag)
        assert n_g == n_o
        tag += n_g
        if n_g == 0:
            break
    torch.cuda.synchronize()
    assert g.npart == o.st.npart > st.npart
    n = g.npart
    np.testing.assert_array_equal(g.host("pr")[:, :n], o.st.pr[:, :n])
    np.testing.assert_array_equal(g.host("pi")[:, :n], o.st.pi[:, :n])
    # a switch at level 1 of a state with random plain levels
    rng = np.random.default_rng(8)
    code = rng.integers(0, 3, n).astype(np.int32)
    g.t["pi"][3, :n] = torch.from_numpy(code).to(g.device)
    o.st.pi[3, :n] = code
    assert g.cloud_instant_switch(1) == o.cloud_instant_switch(1) > 0
    np.testing.assert_array_equal(g.host("pi")[3, :n], o.st.pi[3, :n])


@pytest.mark.parametrize("solver", [0, 2])
def test_refined_cloud_cycles_match_the_oracle(solver):
    """Clouds at the level of their leaves, one split pass (lobed transition clouds where a
    support meets finer leaves), then two imex2+ cycles of the clouds on the refined mesh in both
    forms."""
    ms = _mesh()
    st = refined_state(ms, [0.02, 0.5], [1.0, 0.5], 1, seed=21, vel_noise=0.3, gas_noise=0.05,
                       vd=[0.5, -0.3])
    _codes(st, leaf_tables(ms), "block")
    phys = dict(scheme=2, drag_solver=solver, consistent_gas=True)
    g, o = _pair(ms, st, phys)
    sp = capi.split_params(max_level=2)
    n = g.cloud_split_p1(sp, st.npart)
    assert o.cloud_split_p1(sp, st.npart) == n > 0
    dt = 0.2 * ms.mb_size[:, 6].min() / np.abs(st.pr[[1, 3, 5], :st.npart]).max()
    for _ in range(2):
        g.cloud_refined_imex_cycle(dt)
        assert o.cloud_imex_cycle(dt) == 0
    torch.cuda.synchronize()
    assert g.error_word() == 0
    n = g.npart
    assert n == o.st.npart
    a, b = g.host("pr"), o.st.pr
    np.testing.assert_array_equal(g.host("pi")[0, :n], o.st.pi[0, :n])
    for r in (0, 1, 2, 3, 4, 5):
        sc = np.abs(b[r, :n]).max()
        assert np.abs(a[r, :n] - b[r, :n]).max() <= 1e-12 * sc, r
    ua, ub = g.t["u0"].cpu().numpy(), o.arr["u0"]
    for v in range(4):
        sc = np.abs(ub[:, v]).max()
        assert np.abs(ms.active(ua)[:, v] - ms.active(ub)[:, v]).max() <= 1e-12 * sc, v


def test_split_budget_matches_the_oracle():
    ms = _mesh()
    st = refined_state(ms, [0.1], [0.5], 1, seed=14, vel_noise=0.2)
    st.pi[3, :st.npart] = 0
    g, o = _pair(ms, st, dict(scheme=2))
    sp = capi.split_params(max_level=1, budget=5000)
    n_g = g.cloud_split_p1(sp, st.npart)
    assert n_g == o.cloud_split_p1(sp, st.npart) and 5000 <= n_g <= 5026
    torch.cuda.synchronize()
    n = g.npart
    np.testing.assert_array_equal(g.host("pr")[:, :n], o.st.pr[:, :n])
    np.testing.assert_array_equal(g.host("pi")[:, :n], o.st.pi[:, :n])
