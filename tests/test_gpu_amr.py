"""The general deposit remap on refined meshes, on the GPU against the oracle.

dustb_ghost_add_plan (GeneralApply, src/bvals/bvals_dep_general.cpp:1135-1175) applies the plan
of a refined 3-D mesh; it must equal the oracle's apply bit for bit (the same sums in the same
order, FP64 without contraction).  The point-particle deposit on a refined mesh (every block
deposits with its own cell size) followed by the remap must match the oracle's to 1e-12 of the
field's scale (the deposits are atomic sums), and put the particles' whole coupled mass into
active cells.
"""
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
