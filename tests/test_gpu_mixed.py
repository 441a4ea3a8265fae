"""Mixed-precision form (FP32 offsets/velocities/weights/kicks, FP64 drag factor, per-cell
accumulators and gas) against the FP64 forms on the same seeded inputs.

Stated tolerance of the mixed form on these small cases (a few cycles, a few thousand
particles): every particle velocity is within 1e-5 of the FP64 result relative to the largest
velocity, every position within 1e-5 cells, the gas momentum field within 1e-5 of its scale;
total gas + dust momentum of the mixed form's own state changes by at most 1e-12 of the
absolute momentum per cycle (the momentum ledgers of the kick tiles and the push return every
FP32 rounding of the exchange to the gas).  The benchmark-shaped case and the
tolerance with the consistent split on large particle counts are in
test_gpu_mixed_config2.py."""
import numpy as np
import pytest

from athenak_b200.mesh import uniform_mesh
from athenak_b200.inputs import make_state
from oracle.oracle import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

VTOL = 1e-5

CASES = {
    "3d_random": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                      st=dict(taus=[0.01, 0.1, 1.0], eps=[0.5, 0.5, 0.5], ppc=2, seed=3,
                              vd=[0.1, -0.2, 0.3], gas_noise=1e-2, vel_noise=0.05),
                      phys=dict(scheme=2, drag_solver=2), dt=2e-3),
    "3d_stiff_64": dict(mesh=((64, 32, 32), (64, 16, 16), 2, (-1.0,) * 3, (1.0,) * 3),
                        st=dict(taus=[0.001, 0.01, 0.1, 1.0], eps=[0.5] * 4, ppc=2, seed=7,
                                shearing_box=True, vel_noise=1e-3, gas_noise=1e-3),
                        phys=dict(scheme=2, drag_solver=2, shearing_box=True), dt=0.01),
    "2d_lattice": dict(mesh=((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3),
                       st=dict(taus=[0.1, 0.03, 1.0], eps=[0.2, 0.5, 0.3], ppc=1,
                               placement="lattice", vd=[0.01 / 3, 0.02 / 3, 0.01],
                               gas_noise=0.0),
                       phys=dict(scheme=2, drag_solver=2), dt=0.0125),
    "cic_dc2_plain": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                          st=dict(taus=[0.001, 1.0], eps=[2.0, 0.3], ppc=3, seed=9,
                                  vel_noise=0.02, gas_noise=1e-2),
                          phys=dict(scheme=1, drag_solver=3, consistent_gas=False), dt=2e-3),
    "ngp_local": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                      st=dict(taus=[0.01, 0.3], eps=[1.0, 0.5], ppc=2, seed=12,
                              vel_noise=0.03, gas_noise=1e-2),
                      phys=dict(scheme=0, drag_solver=0), dt=2e-3),
    "no_back_reaction": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3),
                             st=dict(taus=[0.01, 0.3], eps=[1.0, 0.5], ppc=2, seed=13,
                                     vel_noise=0.03, gas_noise=1e-2),
                             phys=dict(scheme=2, drag_solver=2, back_reaction=False), dt=2e-3),
}


def run_pair(name, cycles=3):
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    c = CASES[name]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    ref = DeviceDust(st, c["phys"])
    mx = MixedDust(st, c["phys"])
    p0 = sum(ref.momentum())
    for _ in range(cycles):
        ref.imex_cycle(c["dt"])
        mx.imex_cycle(c["dt"])
    mx.export()
    torch.cuda.synchronize()
    return st, ref, mx, p0, c


def check(st, ref, mx, c):
    assert ref.error_word() == 0 and mx.error_word() == 0
    a, b = mx.dev.host("pr"), ref.host("pr")
    vscale = np.abs(b[[1, 3, 5]]).max()
    for r in (1, 3, 5, 7, 9, 11):
        assert np.abs(a[r] - b[r]).max() < VTOL * vscale, r
    ms = st.mesh
    dx = ms.mb_size[0, 6:9]
    for r, ax in ((0, 0), (2, 1), (4, 2), (6, 0), (8, 1), (10, 2)):
        if ax == 2 and not ms.three_d:
            continue
        assert np.abs(a[r] - b[r]).max() < VTOL * dx[ax], r
    np.testing.assert_array_equal(mx.dev.host("pi"), ref.host("pi"))
    ua, ub = mx.dev.host("u0"), ref.host("u0")
    for v in range(1, 4):
        sc = np.abs(ub[:, v]).max()
        if sc > 0:
            assert np.abs(ua[:, v] - ub[:, v]).max() < VTOL * sc, v


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_matches_fp64(name):
    st, ref, mx, p0, c = run_pair(name)
    check(st, ref, mx, c)


def absolute_momentum(st):
    """sum of |m v| over particles + sum of |rho u| V over active cells (per component)"""
    n = st.npart
    d = np.array([np.abs(st.pr[16, :n] * st.pr[r, :n]).sum() for r in (1, 3, 5)])
    g = np.abs(st.mesh.active(st.u0)[:, 1:4]).sum(axis=(0, 2, 3, 4)) * st.mesh.cell_volume()
    return (d + g).max()


@pytest.mark.parametrize("name", ["3d_random", "2d_lattice", "cic_dc2_plain", "ngp_local"])
def test_mixed_conserves_momentum(name):
    """Gas + dust momentum of the mixed form is conserved to FP64 round-off: from its own
    initial state (the import rounds m and v to FP32; an export before the first cycle writes
    that state to the rows), every cycle changes the total by at most 1e-12 of the absolute
    momentum.  The kick tiles return the FP32 rounding of their deposits (weights whose sum is 1
    only to FP32 precision, FP32 products and per-cell sums) and of the stored velocities and
    rates to the gas, the push returns the rounding of the FP32 RK combination and of the folded
    consistent kick, and the centre mass is summed in FP64, so that the dust share of a cell
    sums to what the gas gave up.  The FP64 form holds 1e-13."""
    from athenak_b200.mixed import MixedDust
    c = CASES[name]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    absm = absolute_momentum(st)
    mx = MixedDust(st, c["phys"])
    mx.export()
    torch.cuda.synchronize()
    p0 = sum(mx.dev.momentum())
    for cyc in range(1, 5):
        mx.imex_cycle(c["dt"])
        mx.export()
        torch.cuda.synchronize()
        p = sum(mx.dev.momentum())
        assert np.abs(p - p0).max() <= 1e-12 * cyc * absm, (cyc, np.abs(p - p0).max() / absm)
    assert mx.error_word() == 0
    st, ref, mx, p0, c = run_pair(name, cycles=4)
    g, d = ref.momentum()
    assert np.abs(g + d - p0).max() < 1e-13 * absolute_momentum(st)


def test_mixed_matches_oracle():
    c = CASES["3d_random"]
    from athenak_b200.mixed import MixedDust
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    o = Oracle(st, c["phys"])
    mx = MixedDust(st, c["phys"])
    for _ in range(2):
        assert o.imex_cycle(c["dt"]) == 0
        mx.imex_cycle(c["dt"])
    mx.export()
    torch.cuda.synchronize()
    a = mx.dev.host("pr")
    n = st.npart
    vscale = np.abs(o.st.pr[[1, 3, 5], :n]).max()
    for r in (1, 3, 5):
        assert np.abs(a[r] - o.st.pr[r, :n]).max() < VTOL * vscale
    np.testing.assert_array_equal(mx.dev.host("pi")[0], o.st.pi[0, :n])


@pytest.mark.parametrize("variant,rows,chunk", [(0, 1, 64), (0, 2, 128), (0, 4, 2048), (0, 8, 512),
                                                (0, 1, 0), (0, 2, 68), (0, 1, 6144)])
def test_tile_shapes_agree(variant, rows, chunk):
    """The autotuner's knobs (rows per tile, particles per pass) change only the order of the
    FP32 partial sums (64 columns: 56 particles per pass, many passes per tile)."""
    from athenak_b200.mixed import MixedDust
    c = CASES["3d_random"]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    base = MixedDust(st, c["phys"])
    alt = MixedDust(st, c["phys"], rows_per_tile=rows, chunk=chunk, variant=variant)
    for _ in range(2):
        base.imex_cycle(c["dt"])
        alt.imex_cycle(c["dt"])
    base.export(); alt.export()
    torch.cuda.synchronize()
    a, b = alt.dev.host("pr"), base.dev.host("pr")
    vs = np.abs(b[[1, 3, 5]]).max()
    assert np.abs(a[[1, 3, 5]] - b[[1, 3, 5]]).max() < 1e-6 * vs


def test_mixed_sort_keeps_rows():
    from athenak_b200.mixed import MixedDust
    c = CASES["3d_random"]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    mx = MixedDust(st, c["phys"])
    mx.imex_cycle(c["dt"])
    mx.export()
    torch.cuda.synchronize()
    before = mx.dev.host("pr").copy()
    mx.sort()
    mx.export()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(mx.dev.host("pr"), before)


def test_graph_replay_matches_eager():
    """One mixed imex2+ cycle captured as a CUDA graph and replayed: the same state as the
    eager calls (up to the order of the FP32 partial sums' atomic adds)."""
    from athenak_b200.mixed import MixedDust
    c = CASES["3d_random"]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    eager = MixedDust(st, c["phys"])
    graph = MixedDust(st, c["phys"])
    for _ in range(3):
        eager.imex_cycle(c["dt"])
    graph.imex_cycle(c["dt"])
    g = graph.capture(lambda: graph.imex_cycle(c["dt"]))
    for _ in range(2):
        g.replay()
    eager.export(); graph.export()
    torch.cuda.synchronize()
    assert eager.error_word() == 0 and graph.error_word() == 0
    a, b = graph.dev.host("pr"), eager.dev.host("pr")
    vs = np.abs(b[[1, 3, 5]]).max()
    assert np.abs(a[[1, 3, 5]] - b[[1, 3, 5]]).max() < 1e-6 * vs
    np.testing.assert_array_equal(graph.dev.host("pi"), eager.dev.host("pi"))


# boundaries beyond the periodic box: physical x3 faces (reflect, outflow) and shear-periodic
# x1 faces.  Large velocity noise so that particles cross the faces every cycle.
EDGE_MESHES = {
    "strat_reflect": dict(mesh=((16, 16, 32), (8, 8, 16), 2, (-0.05, -0.05, -0.1), (0.05, 0.05, 0.1)),
                          kw=dict(x3bc=1), phys=dict(stratified=True)),
    "strat_outflow": dict(mesh=((16, 16, 32), (8, 8, 16), 2, (-0.05, -0.05, -0.1), (0.05, 0.05, 0.1)),
                          kw=dict(x3bc=2), phys=dict(stratified=True, x3_deposit_drop=True)),
    "shear_x1": dict(mesh=((32, 32, 16), (16, 8, 8), 2, (-0.05, -0.1, -0.05), (0.05, 0.1, 0.05)),
                     kw=dict(shear_x1=True), phys=dict()),
    "shear_strat_outflow": dict(mesh=((16, 32, 32), (8, 8, 16), 2, (-0.05, -0.1, -0.1), (0.05, 0.1, 0.1)),
                                kw=dict(x3bc=2, shear_x1=True), phys=dict(stratified=True)),
}


def edge_pair(name, ts_range=None):
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    e = EDGE_MESHES[name]
    ms = uniform_mesh(*e["mesh"], **e["kw"])
    st = make_state(ms, [0.01, 0.1], [0.5, 0.5], 2, seed=17, shearing_box=True, vel_noise=0.3,
                    gas_noise=1e-2, ts_per_particle=ts_range)
    phys = dict(scheme=2, drag_solver=2, shearing_box=True, **e["phys"])
    return st, DeviceDust(st, phys), MixedDust(st, phys)


def check_edges(st, ref, mx, x1_rows=True):
    assert ref.error_word() == 0 and mx.error_word() == 0
    a, b = mx.dev.host("pr"), ref.host("pr")
    vscale = np.abs(b[[1, 3, 5]]).max()
    for r in (1, 3, 5, 7, 9, 11):
        assert np.abs(a[r] - b[r]).max() < VTOL * vscale, r
    # the rates (imex dv/(a dt), pc2 dv): FP32 velocity differences, 1e-3 of their scale
    rscale = np.abs(b[12:15]).max()
    assert np.abs(a[12:15] - b[12:15]).max() < 1e-3 * rscale
    # masses: kept, or zeroed by an outflow face in both forms
    np.testing.assert_array_equal(a[16] == 0.0, b[16] == 0.0)
    dx = st.mesh.mb_size[0, 6:9]
    for r, ax in ((0, 0), (2, 1), (4, 2)) + (((6, 0), (8, 1), (10, 2)) if x1_rows else ()):
        assert np.abs(a[r] - b[r]).max() < VTOL * dx[ax], r
    np.testing.assert_array_equal(mx.dev.host("pi"), ref.host("pi"))
    ua, ub = mx.dev.host("u0"), ref.host("u0")
    ms = st.mesh
    for v in range(1, 4):
        sa, sb = ms.active(ua)[:, v], ms.active(ub)[:, v]
        sc = np.abs(sb).max()
        assert np.abs(sa - sb).max() < VTOL * sc, v
    ra, rb = mx.dev.host("x3_removed"), ref.host("x3_removed")
    assert ra[1] == rb[1] and abs(ra[0] - rb[0]) <= 1e-6 * abs(rb[0])


@pytest.mark.parametrize("name", list(EDGE_MESHES))
def test_mixed_imex_physical_and_shear_faces(name):
    """The mixed imex2+ cycle on meshes with physical x3 faces or shear-periodic x1 faces (the
    tiles on each block's own ghost cells with the FP64 exchanges around them; the push's
    reflect / outflow / shear crossing) against the FP64 form, to the mixed tolerance."""
    st, ref, mx = edge_pair(name)
    t, dt = 1.7, 2e-3
    for _ in range(3):
        ref.set_time(t); mx.dev.set_time(t)
        ref.imex_cycle(dt)
        mx.imex_cycle(dt)
        t += dt
    mx.export()
    torch.cuda.synchronize()
    check_edges(st, ref, mx)


PC2_CASES = {
    "3d_random": dict(mesh=((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3), kw={},
                      st=dict(taus=[0.01, 0.1, 1.0], eps=[0.5, 0.5, 0.5], ppc=2, seed=3,
                              vd=[0.1, -0.2, 0.3], gas_noise=1e-2, vel_noise=0.05),
                      phys=dict(scheme=2), dt=2e-3),
    "3d_stiff_sbox": dict(mesh=((64, 32, 32), (64, 16, 16), 2, (-1.0,) * 3, (1.0,) * 3), kw={},
                          st=dict(taus=[0.001, 0.01, 0.1, 1.0], eps=[0.5] * 4, ppc=2, seed=7,
                                  shearing_box=True, vel_noise=1e-3, gas_noise=1e-3),
                          phys=dict(scheme=2, shearing_box=True), dt=0.01),
    "2d_xz_sbox_cic": dict(mesh=((32, 32, 1), (16, 16, 1), 2, (-0.5,) * 3, (0.5,) * 3), kw={},
                           st=dict(taus=[0.1, 1.0], eps=[0.5, 0.5], ppc=2, seed=2,
                                   shearing_box=True, vel_noise=0.01),
                           phys=dict(scheme=1, shearing_box=True, const_accel_phi=0.05), dt=0.01),
    "strat_reflect": dict(mesh=((16, 16, 32), (8, 8, 16), 2, (-0.05, -0.05, -0.1), (0.05, 0.05, 0.1)),
                          kw=dict(x3bc=1),
                          st=dict(taus=[0.01, 0.1], eps=[0.5, 0.5], ppc=2, seed=17,
                                  shearing_box=True, vel_noise=0.3, gas_noise=1e-2),
                          phys=dict(scheme=2, shearing_box=True, stratified=True), dt=2e-3),
    # the stratified continuous-distribution workload in small: shear-periodic x1, outflow
    # x3 faces with the deposit fold, per-particle t_s log-uniform over St 1e-3..1
    "strat_shear_continuous": dict(
        mesh=((16, 32, 32), (8, 8, 16), 2, (-0.05, -0.1, -0.1), (0.05, 0.1, 0.1)),
        kw=dict(x3bc=2, shear_x1=True),
        st=dict(taus=[0.1, 0.1], eps=[0.01, 0.01], ppc=2, seed=5, shearing_box=True,
                vel_noise=0.3, gas_noise=1e-2, ts_per_particle=(1e-3, 1.0)),
        phys=dict(scheme=2, shearing_box=True, stratified=True), dt=2e-3),
}


def pc2_pair(name, cycles=3):
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    c = PC2_CASES[name]
    ms = uniform_mesh(*c["mesh"], **c["kw"])
    st = make_state(ms, **c["st"])
    ref, mx = DeviceDust(st, c["phys"]), MixedDust(st, c["phys"])
    # the generator draws every gas cell, ghosts included: the ghost values a step starts from
    ref.init_gas_ghosts()
    mx.dev.init_gas_ghosts()
    p0 = sum(ref.momentum())
    t = 1.7
    for _ in range(cycles):
        ref.set_time(t); mx.dev.set_time(t)
        chi_r = float(ref.pc2_cycle(c["dt"]).item())
        chi_m = float(mx.pc2_cycle(c["dt"]).item())
        assert abs(chi_m - chi_r) <= 1e-5 * chi_r
        t += c["dt"]
    mx.export()
    torch.cuda.synchronize()
    return st, ref, mx, p0


@pytest.mark.parametrize("name", list(PC2_CASES))
def test_mixed_pc2_matches_fp64(name):
    """The mixed pc2 cycle (predictor tiles, half-step sort, advance tiles + the edge kernel,
    the move) against the FP64 pc2 cycle, to the mixed tolerance; X1 is not compared (the
    mixed form does not keep the half-step register)."""
    st, ref, mx, _ = pc2_pair(name)
    check_edges(st, ref, mx, x1_rows=False)


def test_mixed_pc2_conserves_momentum():
    """Without rotation the pc2 impulse handed to the gas is the velocity change the
    particle received, so gas + dust momentum holds to the FP32 rounding of the deposits."""
    cycles = 4
    st, ref, mx, p0 = pc2_pair("3d_random", cycles=cycles)
    g, d = mx.dev.momentum()
    assert np.abs(g + d - p0).max() < 1e-7 * cycles * absolute_momentum(st)


@pytest.mark.parametrize("rows,chunk", [(2, 0), (2, 68), (4, 64), (1, 64)])
def test_clumped_tiles_match_fp64(rows, chunk):
    """A thin dense layer (Gaussian heights of scale 0.4 cells: ~40 particles per cell in the
    midplane) with passes of 60..2340 particles: passes that cover few cells split them into
    slots across threads.  Every shape matches the FP64 form to the mixed tolerance and
    reports no error bit (no bounded copy wait ran out)."""
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1, 1.0], [0.5, 0.5, 0.5], 2, seed=3, vd=[0.1, -0.2, 0.3],
                    gas_noise=1e-2, vel_noise=0.05, hp=0.0025)
    phys = dict(scheme=2, drag_solver=2)
    ref = DeviceDust(st, phys)
    mx = MixedDust(st, phys, rows_per_tile=rows, chunk=chunk)
    for _ in range(3):
        ref.imex_cycle(2e-3)
        mx.imex_cycle(2e-3)
    mx.export()
    torch.cuda.synchronize()
    check(st, ref, mx, None)


@pytest.mark.parametrize("mesh", ["periodic", "shear_x1"])
def test_mixed_imex_shear_shift_matches_fp64(mesh):
    """The 3-D shearing box's implicit shear shift (the imex stages' weights at y + sh x): the
    tiles use the shifted weights, particles whose shifted position lies in the next cell go
    through the per-particle edge kernels; against the FP64 form with the same shift, on a
    periodic box and on the small workload's shear-periodic box (time advancing)."""
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    ms = uniform_mesh((32, 32, 32), (16, 16, 16), 2, (-0.05,) * 3, (0.05,) * 3,
                      shear_x1=(mesh == "shear_x1"))
    st = make_state(ms, [0.1], [1.0], 1, seed=1, shearing_box=True, gas_noise=1e-3,
                    vel_noise=0.02)
    phys = dict(scheme=2, drag_solver=2, shearing_box=True)
    ref, mx = DeviceDust(st, phys), MixedDust(st, phys)
    dt, t, sh = 2e-3, 1.7, (1.5e-3 * 4, 1.5e-3 * 4)
    for _ in range(3):
        ref.set_time(t); mx.dev.set_time(t)
        ref.imex_cycle(dt, sh=sh)
        mx.imex_cycle(dt, sh=sh)
        t += dt
    mx.export()
    torch.cuda.synchronize()
    check(st, ref, mx, None)


def test_copy_wait_timeout_is_reported_and_recoverable():
    """Failure detection without a fault: the test hook makes the first tile of every deposit
    launch skip its first bulk copy, so that tile's bounded wait runs out.  The kernels
    return, the error word carries DUSTB_ERR_TIMEOUT, and the context stays usable: a
    fresh shadow on the same device runs a clean cycle afterwards."""
    from athenak_b200.mixed import MixedDust
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1], [1.0], 2, seed=2)
    phys = dict(scheme=2, drag_solver=1)
    probe = MixedDust(st, phys, variant=7)      # DUSTB_MIXED_PROBE_COPY_TIMEOUT
    probe.imex_cycle(2e-3)
    torch.cuda.synchronize()
    assert probe.error_word() & 0x40             # DUSTB_ERR_TIMEOUT
    clean = MixedDust(st, phys)
    clean.imex_cycle(2e-3)
    clean.export()
    torch.cuda.synchronize()
    assert clean.error_word() == 0


def test_uneven_blocks_from_the_work_queue():
    """Four MeshBlocks stacked in x3 around a Gaussian particle layer (scale 0.009 of a box
    of 0.1): the inner blocks hold more than 100 times the particles of the outer ones and
    the midplane cells ~70 each (tiles of several passes, split cells).  The persistent
    tile launches taking the tiles heaviest first from the device work queue match the FP64
    form to the per-particle tolerance (the plain back-reaction: a step continuous in the
    positions, so the bar holds for every one of the 1,048,576 particles), and the
    one-CTA-per-tile launches to FP32 rounding."""
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mixed import MixedDust
    ms = uniform_mesh((32, 32, 64), (32, 32, 16), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.3], [1.0, 0.5], 8, seed=21, hp=0.009, vel_noise=0.03,
                    gas_noise=1e-2)
    counts = np.bincount(st.pi[0, :st.npart], minlength=ms.nmb)
    assert counts.min() > 0 and counts.max() > 100 * counts.min(), counts
    phys = dict(scheme=2, drag_solver=2, consistent_gas=False)
    ref = DeviceDust(st, phys)
    mq = MixedDust(st, phys)                    # the work queue (default)
    mg = MixedDust(st, phys, variant=8)         # DUSTB_MIXED_GRID_TILES: one CTA per tile
    dt = 2e-3
    for _ in range(3):
        ref.imex_cycle(dt)
        mq.imex_cycle(dt)
        mg.imex_cycle(dt)
    mq.export()
    mg.export()
    torch.cuda.synchronize()
    check(st, ref, mq, None)
    a, b = mq.dev.host("pr"), mg.dev.host("pr")
    vscale = np.abs(b[[1, 3, 5]]).max()
    for r in (1, 3, 5):
        assert np.abs(a[r] - b[r]).max() < 1e-6 * vscale, r
    assert mg.error_word() == 0


def test_library_autotuner_keeps_the_results():
    """dustb_mixed_tune picks a tile shape and launch form on the caller's workspace without
    changing the state: cycles after tuning match cycles with the default shape to FP32
    rounding of the sums' order, and match the FP64 form."""
    from athenak_b200.mixed import MixedDust
    c = CASES["3d_random"]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    a = MixedDust(st, c["phys"])
    b = MixedDust(st, c["phys"])
    rows, chunk, grid, tms = a.tune(1.7 * c["dt"])
    assert rows in (1, 2, 4, 8) and tms > 0.0
    from athenak_b200.drag import DeviceDust
    ref = DeviceDust(st, c["phys"])
    for _ in range(3):
        a.imex_cycle(c["dt"])
        b.imex_cycle(c["dt"])
        ref.imex_cycle(c["dt"])
    a.export()
    b.export()
    torch.cuda.synchronize()
    assert a.error_word() == 0 and b.error_word() == 0
    pa, pb = a.dev.host("pr"), b.dev.host("pr")
    vscale = np.abs(pb[[1, 3, 5]]).max()
    for r in (1, 3, 5):
        assert np.abs(pa[r] - pb[r]).max() < 1e-6 * vscale, r
    check(st, ref, a, c)


def _window_pair(st, phys, variant, cycles, pc2=False, dt=None, **kw):
    from athenak_b200.mixed import MixedDust
    a = MixedDust(st, phys, variant=32 | variant, **kw)
    b = MixedDust(st, phys, variant=variant, **kw)
    for _ in range(cycles):
        for mx in (a, b):
            if pc2:
                mx.pc2_cycle(dt)
            else:
                mx.imex_cycle(dt)
    a.export()
    b.export()
    torch.cuda.synchronize()
    assert a.error_word() == 0 and b.error_word() == 0
    pa, pb = a.dev.host("pr"), b.dev.host("pr")
    vscale = np.abs(pb[[1, 3, 5]]).max()
    for r in (1, 3, 5):
        assert np.abs(pa[r] - pb[r]).max() < 1e-6 * vscale, (variant, r)
    np.testing.assert_array_equal(a.dev.host("pi")[0], b.dev.host("pi")[0])


@pytest.mark.parametrize("case", ["3d_random", "cic_dc2_plain"])
def test_window_staged_by_tensor_copy_keeps_the_results(case):
    """DUSTB_MIXED_WINDOW_TMA: the gathering tiles take their gas window from shared memory,
    staged by one tensor copy per tile, instead of loading it per thread: the same window
    values in the same order, so the cycles match the default form to the FP32 rounding of
    the deposits' order -- imex2+ with one CTA per tile and on the work queue, pc2 (predictor
    and advance tiles), and tiles of several passes (the window kept across them)."""
    c = CASES[case]
    ms = uniform_mesh(*c["mesh"])
    st = make_state(ms, **c["st"])
    for grid in (0, 8):
        _window_pair(st, c["phys"], grid, 3, dt=c["dt"])
    _window_pair(st, c["phys"], 0, 2, pc2=True, dt=c["dt"])
    _window_pair(st, c["phys"], 0, 2, dt=c["dt"], rows_per_tile=2, chunk=68)
