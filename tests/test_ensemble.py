"""The batched ensemble of independent damping boxes: the box mesh, the seeded box draws and
the exact damping solution (CPU); the ensemble on the GPU against the FP64 form and the exact
solution."""
import numpy as np
import pytest

from athenak_b200.mesh import box_ensemble_mesh, dir_index


def rk4(taus, eps, v0, t, n=20000):
    """The damping ODE (src/pgen/tests/dust_damping.cpp:9-16) integrated by fine RK4."""
    taus, eps = np.asarray(taus), np.asarray(eps)

    def f(y):
        u, v = y[0], y[1:]
        return np.concatenate([[np.sum(eps * (v - u) / taus)], -(v - u) / taus])
    y = np.concatenate([[0.0], np.full(len(taus), v0)])
    h = t / n
    for _ in range(n):
        k1 = f(y); k2 = f(y + 0.5 * h * k1); k3 = f(y + 0.5 * h * k2); k4 = f(y + h * k3)
        y = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
    return y


def test_damping_solution_matches_rk4():
    pytest.importorskip("torch")
    from athenak_b200.ensemble import damping_solution
    for taus, eps in (((0.5,), (1.0,)), ((0.2, 1.0, 3.0), (0.3, 2.0, 5.0)), ((0.05, 10.0), (10.0, 0.1))):
        ex = damping_solution(taus, eps, 0.1, 0.7)
        assert np.abs(ex - rk4(taus, eps, 0.1, 0.7)).max() < 1e-12
        # momentum: u + sum eps_s v_s is constant
        assert abs(ex[0] + np.dot(eps, ex[1:]) - 0.1 * sum(eps)) < 1e-14


def test_box_mesh_blocks_are_their_own_neighbours():
    ms = box_ensemble_mesh(12, 5)
    assert ms.nmb == 5 and ms.nx == (12, 12, 12)
    for m in range(5):
        for d in range(27):
            assert ms.nghbr[m, d] == (-1 if d == dir_index(0, 0, 0) else m)
    assert np.allclose(ms.mb_size[:, 6:9], 1.0 / 12)


def test_draw_boxes_ranges():
    pytest.importorskip("torch")
    from athenak_b200.ensemble import draw_boxes
    bs = draw_boxes(300, seed=2)
    assert bs == draw_boxes(300, seed=2)
    assert all(16 <= b.side <= 64 and 1 <= len(b.taus) <= 4 and 1 <= b.ppc <= 8 for b in bs)
    assert all(1e-3 <= t <= 10 for b in bs for t in b.taus)
    assert all(0.1 <= e <= 10 for b in bs for e in b.eps)


@pytest.mark.gpu
def test_ensemble_matches_fp64_and_exact():
    """Twelve boxes of 8..12 cells per side in packs by side: after 30 cycles every box's
    species and gas velocities match the FP64 form run on the same pack (mixed tolerance),
    the exact damping solution to 2e-3 of v0 (the imex2+ scheme's own error), and momentum
    holds to 1e-7 per cycle."""
    import torch
    from athenak_b200.ensemble import EnsemblePack, draw_boxes
    boxes = draw_boxes(12, seed=5, sides=(8, 12))
    by_side = {}
    for b in boxes:
        by_side.setdefault(b.side, []).append(b)
    cycles = 30
    for side, bs in by_side.items():
        mixed = EnsemblePack(side, bs)
        fp64 = EnsemblePack(side, bs)
        mixed.step(cycles)
        for _ in range(cycles):
            fp64.dev.imex_cycle(fp64.dt)
        torch.cuda.synchronize()
        assert mixed.mx.error_word() == 0 and fp64.dev.error_word() == 0
        for c in mixed.check():
            assert c["err_vs_exact"] < 2e-3, c
            assert c["momentum_change"] < 1e-7 * cycles, c
        mixed.mx.export()
        torch.cuda.synchronize()
        a, b = mixed.dev.host("pr"), fp64.dev.host("pr")
        assert np.abs(a[1] - b[1]).max() < 1e-5 * 0.1
        np.testing.assert_array_equal(mixed.dev.host("pi"), fp64.dev.host("pi"))


@pytest.mark.gpu
def test_ensemble_one_launch_matches_pack_by_pack():
    """The whole ensemble as one CUDA-graph launch per substep (every pack resident, its rows
    detached, each pack's cycle on a branch of its own) gives every box the result of the
    pack-by-pack replays up to FP32 rounding (the FP64 atomics sum in another order): the
    per-box errors against the exact damping solution agree to 1e-6 of v0 and momentum holds
    as before."""
    from athenak_b200.ensemble import draw_boxes, run_ensemble, run_ensemble_one_launch
    boxes = draw_boxes(12, seed=5, sides=(8, 12))
    cycles = 20
    _, ps_a, ch_a = run_ensemble(boxes, cycles)
    _, ps_b, ch_b, npacks = run_ensemble_one_launch(boxes, cycles)
    assert npacks == len({b.side for b in boxes}) and ps_a == ps_b
    key = lambda c: (c["side"], c["nspecies"], c["ppc"], c["dt_over_tau_min"])
    for a, b in zip(sorted(ch_a, key=key), sorted(ch_b, key=key)):
        assert key(a) == key(b)
        assert abs(a["err_vs_exact"] - b["err_vs_exact"]) < 1e-6, (a, b)
        assert b["err_vs_exact"] < 2e-3 and b["momentum_change"] < 1e-7 * cycles, b
