"""The mixed form on the benchmark's configuration, scaled to fit a test: a 128 x 64 x 64 mesh
as two MeshBlocks of 64^3 (the benchmark's block size), 4 species t_s = {0.01, 0.1, 1, 10},
eps 0.5 each, ppc 4 each (8,388,608 particles), dt from CFL 0.3 with dt / t_s reaching 10
(drag factors up to 0.94), imex2+ with dc1 and TSC, 13 cycles from the rows in cell order.

The stated tolerance (athenak_b200/tolerance.py): with the plain back-reaction the mixed form
holds every particle to 1e-5 of the FP64 form; with the consistent split (the default) the
split's jump at cell faces is the reference algorithm's own, shown by the FP64 form with its
state stored in the mixed layout (the storage twin), and the bounds are those of
tolerance.judge.  The total dust momentum is also checked against the CPU oracle on one
MeshBlock of the same workload."""
import numpy as np
import pytest

from athenak_b200 import tolerance as tol

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CYCLES = 13
CELLS, BLOCK = (128, 64, 64), (64, 64, 64)


def run_forms(consistent, cells=CELLS, cycles=CYCLES, twin=False):
    """FP64 form, mixed form and (twin) the storage twin from the same seeded rows in cell
    order; returns the mixed and twin errors against the FP64 form."""
    from athenak_b200.mixed import MixedDust
    from athenak_b200.workloads import uniform_box
    ref, ms, W = uniform_box(cells, BLOCK, consistent=consistent)
    mxd, _, _ = uniform_box(cells, BLOCK, consistent=consistent)
    ref.sort_by_cell()
    mxd.sort_by_cell()
    mx = MixedDust(dev=mxd)
    tw = None
    if twin:
        tw, _, _ = uniform_box(cells, BLOCK, consistent=consistent)
        tw.sort_by_cell()
        twx = MixedDust(dev=tw, do_import=False)
    for _ in range(cycles):
        ref.imex_cycle(W["dt"])
        mx.imex_cycle(W["dt"])
        if twin:
            tol.storage_twin_cycle(tw, twx, W["dt"])
    mx.export()
    torch.cuda.synchronize()
    assert ref.error_word() == 0 and mx.error_word() == 0
    n = W["npart"]
    v_f = ref.t["pr"][[1, 3, 5], :n]
    u_f = ms.active(ref.t["u0"])[:, 1:4]
    mass = ref.t["pr"][16, :n]

    def errs(d):
        return tol.compare(d.t["pr"][[1, 3, 5], :n], v_f, ms.active(d.t["u0"])[:, 1:4], u_f, mass)
    return errs(mxd), (errs(tw) if twin else None), W, (ref, mxd, ms)


def test_plain_back_reaction_every_particle_within_vtol():
    """Without the split the step is continuous in the positions: every particle and every
    gas cell within 1e-5, positions within 1e-5 cells, integer rows equal."""
    err, _, W, (ref, mxd, ms) = run_forms(consistent=False)
    v = tol.judge(err, split=False)
    assert v["ok"], (err, v)
    n = W["npart"]
    dx = ms.mb_size[0, 6:9]
    for r, ax in ((0, 0), (2, 1), (4, 2)):
        d = (mxd.t["pr"][r, :n] - ref.t["pr"][r, :n]).abs().max()
        assert float(d) < tol.VTOL * dx[ax], r
    assert torch.equal(mxd.t["pi"][:, :n], ref.t["pi"][:, :n])


def test_consistent_split_within_stated_bounds():
    """The mixed form within the stated bounds; the storage twin (FP64 arithmetic, the state
    stored in the mixed layout) has particles beyond 1e-5 too: those outliers are the split's
    response to the storage, not to the mixed form's FP32 arithmetic."""
    err, twin, W, _ = run_forms(consistent=True, twin=True)
    v = tol.judge(err, split=True)
    print("mixed", err, "twin", twin, "verdict", v)
    assert v["ok"], (err, twin, v)
    assert twin["fraction_beyond_vtol"] > 0.0 and twin["velocity_max_rel"] > tol.VTOL, twin


def test_dust_momentum_against_the_oracle():
    """One 64^3 MeshBlock of the workload (4,194,304 particles), 13 cycles: the mixed form's
    total dust momentum within 1e-6 of the CPU oracle's."""
    import os
    from athenak_b200.inputs import DustState
    from athenak_b200.mixed import MixedDust
    from athenak_b200.workloads import uniform_box
    from oracle.oracle import Oracle
    ref, ms, W = uniform_box(BLOCK, BLOCK)
    ref.sort_by_cell()
    torch.cuda.synchronize()
    n = W["npart"]
    st = DustState(ms, ref.host("pr").copy(), ref.host("pi").copy(), n,
                   ref.t["u0"].cpu().numpy().copy(), 4, W["taus"], W["eps"])
    o = Oracle(st, ref.phys, threads=os.cpu_count() or 1)
    mx = MixedDust(dev=ref)
    for _ in range(CYCLES):
        assert o.imex_cycle(W["dt"]) == 0
        mx.imex_cycle(W["dt"])
    mx.export()
    torch.cuda.synchronize()
    assert mx.error_word() == 0
    m = o.st.pr[16, :n]
    p_o = np.array([(m * o.st.pr[r, :n]).sum() for r in (1, 3, 5)])
    pr = ref.host("pr")
    p_m = np.array([(pr[16] * pr[r]).sum() for r in (1, 3, 5)])
    assert np.abs(p_m - p_o).max() <= tol.MOMENTUM_TOL * np.abs(p_o).max(), (p_m, p_o)
