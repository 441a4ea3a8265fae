"""Batched ensemble of independent periodic dust_damping boxes.

The reference runs one box per job (the dust_damping problem generator,
src/pgen/tests/dust_damping.cpp:115-125, :323-511): gas at rest, dust species moving through
it, every cell alike on the particle lattice, so the discrete system is the damping ODE
    du/dt = sum_s eps_s (v_s - u) / t_s,   dv_s/dt = -(v_s - u) / t_s
(src/pgen/tests/dust_damping.cpp:9-16).  Here the boxes that have the same number of cells
per side form one MeshBlock pack in which every block is a box periodic onto itself
(mesh.box_ensemble_mesh), so one call of the drag step advances every box of the pack, and
one cycle of a pack is captured as a CUDA graph and replayed.  Each box is checked against
the exact solution of its ODE (a matrix exponential) and for momentum conservation.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .drag import DeviceDust, GAMMA_DEFAULT
from .mesh import box_ensemble_mesh
from .mixed import MixedDust
from .inputs import IPX, IPVX, IPY, IPZ, IPX1, IPY1, IPZ1, IPVX1, IPTS, IPM, PGID, PTAG, PSP

__all__ = ["Box", "draw_boxes", "damping_solution", "EnsemblePack", "run_ensemble",
           "run_ensemble_one_launch"]


@dataclass
class Box:
    side: int            # cells per side (the box is [0, 1]^3)
    taus: tuple          # stopping time of each species
    eps: tuple           # dust-to-gas density ratio of each species
    ppc: int             # particles per cell of each species


def draw_boxes(n, seed=1, sides=(16, 64), taus=(1e-3, 10.0), eps=(0.1, 10.0), ppc=(1, 8),
               nspecies=(1, 4)):
    """n boxes with sides log-uniform in `sides`, 1..4 species, t_s and eps log-uniform,
    ppc uniform in `ppc` (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        side = int(round(math.exp(rng.uniform(math.log(sides[0]), math.log(sides[1])))))
        ns = int(rng.integers(nspecies[0], nspecies[1] + 1))
        ts = tuple(float(x) for x in np.exp(rng.uniform(math.log(taus[0]), math.log(taus[1]), ns)))
        ep = tuple(float(x) for x in np.exp(rng.uniform(math.log(eps[0]), math.log(eps[1]), ns)))
        out.append(Box(side, ts, ep, int(rng.integers(ppc[0], ppc[1] + 1))))
    return out


def damping_solution(taus, eps, v0, t):
    """Exact (u, v_1..v_S) at time t of the damping ODE from u = 0, v_s = v0."""
    ns = len(taus)
    A = np.zeros((ns + 1, ns + 1))
    for s, (ts, e) in enumerate(zip(taus, eps)):
        A[0, 0] -= e / ts
        A[0, 1 + s] += e / ts
        A[1 + s, 0] += 1.0 / ts
        A[1 + s, 1 + s] -= 1.0 / ts
    y0 = np.concatenate([[0.0], np.full(ns, v0)])
    # exp(A t) y0 through the eigen-decomposition of A (diagonalisable: A is similar to a
    # symmetric matrix under the weights (1, eps_s))
    w = np.sqrt(np.concatenate([[1.0], np.asarray(eps, float)]))
    S = (A * w[:, None]) / w[None, :]
    lam, Q = np.linalg.eigh(0.5 * (S + S.T))
    z0 = Q.T @ (w * y0)
    return (Q @ (np.exp(lam * t) * z0)) / w


class EnsemblePack:
    """The boxes of one side as one MeshBlock pack on the device, in the reference layout,
    advanced by the mixed-precision imex2+ cycle."""

    def __init__(self, side, boxes, v0=0.1, device="cuda", detach=False, mixed=True):
        """detach: free the reference rows after the import (the cycles advance the shadow
        alone; check() rebuilds the rows before its export).  mixed False: no mixed-precision
        shadow (the FP64 form advances the reference rows)."""
        self.side, self.boxes, self.v0 = side, list(boxes), v0
        self.ms = box_ensemble_mesh(side, len(self.boxes))
        ncell = side ** 3
        counts = [ncell * b.ppc * len(b.taus) for b in self.boxes]
        self.npart = int(sum(counts))
        phys = dict(scheme=2, drag_solver=2, consistent_gas=True, back_reaction=True)
        self.dev = DeviceDust.empty(self.ms, self.npart, phys, device=device, nspecies=4)
        self._fill_rows()
        u0 = self.dev.t["u0"]
        u0.zero_()
        u0[:, 0] = 1.0                               # gas at rest, density 1
        dx = 1.0 / side
        self.dt = 0.3 * dx / (1.0 + v0)
        self.mx = None
        if mixed:
            self.mx = MixedDust(dev=self.dev, do_import=False)
            self.mx.import_()
            if detach:
                self.dev.detach_rows()
        self.cycles = 0
        self.graph = None

    def _fill_rows(self):
        """The initial reference rows: ppc particles of every species at every cell centre
        of every box (the damping test's lattice), moving at v0 through gas at rest."""
        side, v0 = self.side, self.v0
        ncell = side ** 3
        if self.dev.t.get("pr") is None:
            self.dev.attach_rows(
                torch.zeros((17, self.npart), dtype=torch.float64, device=self.dev.device),
                torch.zeros((5, self.npart), dtype=torch.int32, device=self.dev.device))
        pr, pi = self.dev.t["pr"], self.dev.t["pi"]
        f64 = dict(dtype=torch.float64, device=self.dev.device)
        dx = 1.0 / side
        c = torch.arange(ncell, device=self.dev.device)
        cx = ((c % side).to(torch.float64) + 0.5) * dx
        cy = (((c // side) % side).to(torch.float64) + 0.5) * dx
        cz = ((c // (side * side)).to(torch.float64) + 0.5) * dx
        p0 = 0
        for m, b in enumerate(self.boxes):
            for s, (ts, e) in enumerate(zip(b.taus, b.eps)):
                n = ncell * b.ppc
                sl = slice(p0, p0 + n)
                # ppc particles at every cell centre (the damping test's lattice)
                pr[IPX, sl] = cx.repeat(b.ppc); pr[IPY, sl] = cy.repeat(b.ppc); pr[IPZ, sl] = cz.repeat(b.ppc)
                pr[IPX1, sl] = pr[IPX, sl]; pr[IPY1, sl] = pr[IPY, sl]; pr[IPZ1, sl] = pr[IPZ, sl]
                pr[IPVX, sl] = v0; pr[IPVX1, sl] = v0
                pr[IPTS, sl] = ts
                pr[IPM, sl] = e * 1.0 / n            # eps_s rho V_box over the particles
                pi[PGID, sl] = m
                pi[PSP, sl] = s
                pi[PTAG, sl] = torch.arange(p0, p0 + n, dtype=torch.int32, device=self.dev.device)
                p0 += n

    def step(self, n, stream=None):
        """n imex2+ cycles of every box (the first call runs one eager cycle and captures
        one; the rest replay the capture)."""
        for _ in range(n):
            if self.graph is None:
                self.mx.imex_cycle(self.dt, GAMMA_DEFAULT)
                self.graph = self.mx.capture(lambda: self.mx.imex_cycle(self.dt, GAMMA_DEFAULT))
            else:
                self.graph.replay()
            self.cycles += 1

    def check(self):
        """Per box: the largest deviation of the gas and species mean velocities from the
        exact damping solution, relative to v0, and the change of total momentum relative
        to the initial dust momentum (per-box sums formed on the device).  Detached rows are
        rebuilt first (the export writes positions, velocities, registers and rates; species,
        tags and masses are the initial ones)."""
        if self.dev.t.get("pr") is None:
            self._fill_rows()
        self.mx.export()
        pr, pi = self.dev.t["pr"], self.dev.t["pi"]
        nb = len(self.boxes)
        key = (pi[PGID].long() * 4 + pi[PSP].long())
        f64 = dict(dtype=torch.float64, device=pr.device)
        vs = torch.zeros(nb * 4, **f64).index_add_(0, key, pr[IPVX])
        cnt = torch.zeros(nb * 4, **f64).index_add_(0, key, torch.ones_like(pr[IPVX]))
        pd = torch.zeros(nb * 4, **f64).index_add_(0, key, pr[IPM] * pr[IPVX])
        gas = self.ms.active(self.dev.t["u0"])[:, 1].sum(dim=(1, 2, 3)) * (1.0 / self.side) ** 3
        vs, cnt, pd, gas = (x.cpu().numpy() for x in (vs, cnt, pd, gas))
        t = self.cycles * self.dt
        out = []
        for k, b in enumerate(self.boxes):
            ex = damping_solution(b.taus, b.eps, self.v0, t)
            err = abs(gas[k] - ex[0])
            ptot = gas[k]
            for s in range(len(b.taus)):
                err = max(err, abs(vs[4 * k + s] / cnt[4 * k + s] - ex[1 + s]))
                ptot += pd[4 * k + s]
            p0 = sum(b.eps) * self.v0
            out.append({"side": b.side, "nspecies": len(b.taus), "ppc": b.ppc,
                        "dt_over_tau_min": self.dt / min(b.taus), "t": t,
                        "err_vs_exact": float(err / self.v0),
                        "momentum_change": float(abs(ptot - p0) / p0)})
        return out

    def free(self):
        self.graph = None
        del self.mx, self.dev
        torch.cuda.empty_cache()


def run_ensemble_one_launch(boxes, cycles, v0=0.1):
    """Every box resident at once, one pack per side with its reference rows detached after
    the import, and one substep of the whole ensemble as ONE CUDA-graph launch: the cycle of
    every pack captured on a stream of its own, forked from and joined to the capture stream,
    so the packs' kernels run side by side (the small packs fill the GPU together).  Returns
    the device time of cycles 2..cycles (graph replays), the particle-cycles done in them,
    the per-box checks and the number of packs."""
    by_side = {}
    for b in boxes:
        by_side.setdefault(b.side, []).append(b)
    packs = [EnsemblePack(side, by_side[side], v0, detach=True) for side in sorted(by_side)]
    # one eager cycle of every pack: it sets the kernels' shared-memory limits (a capture
    # does not) and is the untimed first cycle
    for p in packs:
        p.mx.imex_cycle(p.dt, GAMMA_DEFAULT)
        p.cycles += 1
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in packs]
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cap = torch.cuda.current_stream()
        for p, st in zip(packs, streams):
            st.wait_stream(cap)
            p.mx.imex_cycle(p.dt, GAMMA_DEFAULT, stream=st)
        for st in streams:
            cap.wait_stream(st)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(cycles - 1):
        g.replay()
    t1.record()
    torch.cuda.synchronize()
    for p in packs:
        p.cycles += cycles - 1
    ms = t0.elapsed_time(t1)
    psteps = sum(p.npart for p in packs) * (cycles - 1)
    del g
    checks = []
    for p in packs:
        assert p.mx.error_word() == 0, "device error word set"
        checks += p.check()
        p.free()
    return ms, psteps, checks, len(packs)


def run_ensemble_fp64(boxes, cycles=3, v0=0.1):
    """The FP64 per-task form (dustb_imex_cycle on the reference rows, the comparator of the
    mixed form) on the same boxes, every pack resident and one substep of the whole ensemble
    as one CUDA-graph launch whose branches are the packs' cycles, as the mixed arm runs.
    Returns the device time of cycles 2..cycles, the particle-cycles done in them and the
    largest relative deviation of any box from its exact damping solution."""
    by_side = {}
    for b in boxes:
        by_side.setdefault(b.side, []).append(b)
    packs = [EnsemblePack(side, by_side[side], v0, mixed=False) for side in sorted(by_side)]
    for p in packs:
        p.dev.imex_cycle(p.dt, GAMMA_DEFAULT)
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in packs]
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cap = torch.cuda.current_stream()
        for p, st in zip(packs, streams):
            st.wait_stream(cap)
            p.dev.imex_cycle(p.dt, GAMMA_DEFAULT, stream=st)
        for st in streams:
            cap.wait_stream(st)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(cycles - 1):
        g.replay()
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    del g, streams
    psteps = sum(p.npart for p in packs) * (cycles - 1)
    worst = 0.0
    for p in packs:
        assert p.dev.error_word() == 0, "device error word set"
        pr, pi = p.dev.t["pr"], p.dev.t["pi"]
        key = pi[PGID].long() * 4 + pi[PSP].long()
        f64 = dict(dtype=torch.float64, device=pr.device)
        nb = len(p.boxes)
        vs = torch.zeros(nb * 4, **f64).index_add_(0, key, pr[IPVX]).cpu().numpy()
        cnt = torch.zeros(nb * 4, **f64).index_add_(0, key, torch.ones_like(pr[IPVX])).cpu().numpy()
        t = cycles * p.dt
        for k, b in enumerate(p.boxes):
            ex = damping_solution(b.taus, b.eps, v0, t)
            for s_ in range(len(b.taus)):
                worst = max(worst, abs(vs[4 * k + s_] / cnt[4 * k + s_] - ex[1 + s_]) / v0)
        del p.dev
    torch.cuda.empty_cache()
    return ms, psteps, worst


def run_ensemble(boxes, cycles, v0=0.1, stream=None):
    """Every box advanced `cycles` imex2+ cycles, one pack per side; returns the device time
    of the timed cycles (all but the first of each pack), the particle-cycles they did and
    the per-box checks."""
    by_side = {}
    for b in boxes:
        by_side.setdefault(b.side, []).append(b)
    ms_tot, psteps, checks = 0.0, 0, []
    for side in sorted(by_side):
        pack = EnsemblePack(side, by_side[side], v0)
        pack.step(1)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        pack.step(cycles - 1)
        t1.record()
        torch.cuda.synchronize()
        ms_tot += t0.elapsed_time(t1)
        psteps += pack.npart * (cycles - 1)
        assert pack.mx.error_word() == 0, "device error word set"
        checks += pack.check()
        pack.free()
    return ms_tot, psteps, checks
