#!/usr/bin/env python
"""Benchmark of the dust drag step: particle-steps/s, mixed precision vs FP64, on one B200.

Workload (the metric's configuration): uniform periodic 256^3 mesh as 64 MeshBlocks of 64^3
(ng = 2), 4 species tau_s = {0.01, 0.1, 1, 10}/Omega, epsilon 0.5 each, ppc 4 per species
(268,435,456 particles), uniform-random positions (seeded hash; the rows then put in cell
order once, as the reference's SortParticles keeps them), NSH-drift velocities plus
Gaussian 1e-3 c_s noise, gas NSH drift plus 1e-3 uniform noise, imex2+ with dc1, TSC,
consistent point split, dt from CFL 0.3 with the cell width set so that dt/tau_s spans
0.01..10 over the species (athenak_b200/workloads.py).  A step is one imex2+ cycle (two
working stages) of every particle; inputs (~20-46 GB) are far larger than L2, so no flush is
needed between timed steps.

Arms: --impl ours (default) times the mixed form and the FP64 per-task form on the GPU;
--impl reference times the CPU oracle port (OpenMP, all host threads) on a bounded sample.
N > 1 GPUs run independent replicas (the step does not shard across GPUs here).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dust particle-steps/s (gather+kick+deposit), mixed vs FP64 on 1 B200 at err<=1e-6"
UNIT = "particle-steps/s"
GAMMA = 1.707106781186547

# Algorithmic bytes of one launch of each mixed-form kernel: (bytes per particle, bytes per
# cell), the minimum each must read and write (4-byte particle words, FP64 cells).  Averages
# over the two launches of a cycle (stage 1, stage 2):
#   count: stage 1 reads the cell, offsets, velocity, drag factor and mass and writes the key
#          (40 B; the mass and drag factor for the pending consistent kick), stage 2 also the
#          register displacement (52 B); the histogram counter, 8 B per cell
#   move:  stage 1 reads key, cell, row, offsets, velocity, t_s, mass, drag factor (48 B),
#          stage 2 also the velocity register, displacement and rates (84 B); both write cell,
#          row, offsets, velocity, velocity register, displacement, t_s, mass, drag factor
#          (68 B): (116 + 152) / 2
#   deposit_qp: offsets, drag factor, mass, velocity in (32 B); Q, P out and the centre mass
#          (40 B per cell)
#   operator: offsets, drag factor, mass in (20 B); u* in, work out (48 B per cell)
#   kick:  offsets, drag factor, mass, velocity in, velocity and rate out (56 B); u* in, dmom
#          out (48 B per cell)
#   window: the FP64 u* of every active cell and of the one-cell layer around each block in,
#          the FP32 window out: (24 + 16) B times (66/64)^3
MIXED_BYTES = {
    "window": (0.0, 44.0),
    "count": (46.0, 8.0),
    "move": (134.0, 0.0),
    "fill": (0.0, 16.0),
    "deposit_qp": (32.0, 40.0),
    "operator": (20.0, 48.0),
    "kick": (56.0, 48.0),
}
# The whole step's algorithmic bytes (the minimum passes the reference's data dependencies
# force, each field read and written once per pass): per particle-step in the mixed layout
# and per active cell per cycle (imex2+ / dc1, FP64 mesh fields).
STEP_BYTES_PARTICLE = 468.0
STEP_BYTES_CELL = 1112.0


def peaks():
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            d = json.load(f)
        if "hbm_gbs" in d:
            return d["hbm_gbs"], "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return 6650.0, "fallback 6650 GB/s"


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def timed_cycles(fn, steps, stream):
    import torch
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(steps):
        fn()
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps


def cpu_baseline(threads=None, cycles=2):
    """The oracle port (OpenMP, atomics: the reference's Kokkos OpenMP form) on a bounded
    sample of the workload: one 64^3 MeshBlock (the benchmark's block, periodic onto itself)
    with the same species, ppc, cell width and dt (4,194,304 particles, far larger than the
    host caches), the rows put in cell order (the oracle's SortParticles), one warm-up cycle
    and `cycles` timed cycles."""
    from athenak_b200.inputs import make_state
    from athenak_b200.mesh import uniform_mesh
    from athenak_b200.workloads import TAUS4, uniform_box_geometry
    from oracle.oracle import Oracle
    threads = threads or os.cpu_count() or 1
    g = uniform_box_geometry((64, 64, 64))
    ms = uniform_mesh((64, 64, 64), (64, 64, 64), 2, tuple(-x / 2 for x in g["L"]),
                      tuple(x / 2 for x in g["L"]))
    st = make_state(ms, TAUS4, [0.5] * 4, 4, seed=1, shearing_box=True, vel_noise=1e-3,
                    gas_noise=1e-3)
    o = Oracle(st, dict(scheme=2, drag_solver=2), threads=threads)
    o.sort_particles()                        # the rows in cell order, as the GPU arms
    dt = g["dt"]
    o.imex_cycle(dt)
    t = time.perf_counter()
    for _ in range(cycles):
        o.imex_cycle(dt)
    el = time.perf_counter() - t
    return {"value": st.npart * cycles / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one 64^3 MeshBlock periodic onto itself, 4 species ppc 4 each "
                      f"({st.npart} particles, in cell order), the benchmark's cell width and dt, "
                      f"{cycles} imex2+/dc1 cycles after 1 warm-up, FP64, OpenMP atomics"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, args.steps)
    cb = cpu_baseline(cycles=min(steps, 3))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": min(steps, 3), "warmup": 1,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded hash)",
            "config": {"workload": "uniform 256^3 mesh, 64 MeshBlocks of 64^3, 4 species ppc 4 "
                                   "each (268,435,456 particles), imex2+/dc1 TSC",
                       "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def load_traffic():
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def restore(dev, snap):
    pr0, pi0, u00 = snap
    dev.t["pr"].copy_(pr0)
    dev.t["pi"].copy_(pi0)
    dev.t["u0"].copy_(u00)
    for k in ("u1", "qdep", "ustar", "dmom", "resid", "work"):
        dev.t[k].zero_()


def roofline(ktimes, nk, npart, ncell, ms_step):
    """The dominant single kernel (largest time per cycle) against HBM: its algorithmic bytes
    per launch (MIXED_BYTES) over its mean CUDA-event launch time; and the whole step's
    algorithmic bytes (STEP_BYTES_*) over the timed step."""
    peak, src = peaks()
    meas = {k: v for k, v in ktimes.items() if k in MIXED_BYTES and v[1] > 0}
    out = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_source": src}
    if meas:
        dom = max(meas, key=lambda k: meas[k][0])
        bp, bc = MIXED_BYTES[dom]
        per_launch = bp * npart + bc * ncell
        avg_ms = meas[dom][0] / meas[dom][1]
        ach = per_launch / (avg_ms * 1e-3) / 1e9
        tr = load_traffic().get(dom)
        out.update({"kernel": dom, "achieved": round(ach, 1), "frac": round(ach / peak, 3),
                    "traffic": tr, "traffic_source": "profiles/roofline_traffic.json: ncu "
                    "dram__bytes of a 64^3 capture scaled to one launch of this workload"
                    if tr is not None else None,
                    "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": round(avg_ms, 4),
                    "bytes_per_particle": bp, "bytes_per_cell": bc})
        out["kernels"] = {}
        for k, (t, n) in meas.items():
            bp, bc = MIXED_BYTES[k]
            a = (bp * npart + bc * ncell) / (t / n * 1e-3) / 1e9
            out["kernels"][k] = {"avg_launch_ms": round(t / n, 4), "achieved": round(a, 1),
                                 "frac": round(a / peak, 3)}
    step_bytes = STEP_BYTES_PARTICLE * npart + STEP_BYTES_CELL * ncell
    out["step_bytes"] = step_bytes
    out["step_achieved"] = round(step_bytes / (ms_step * 1e-3) / 1e9, 1)
    out["step_frac"] = round(out["step_achieved"] / peak, 3)
    return out


def run_ours(args, rep):
    import torch
    from athenak_b200 import tolerance as tol
    from athenak_b200.mixed import MixedDust
    from athenak_b200.workloads import uniform_box
    rank, world = rep.rank, rep.world
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    stream = torch.cuda.current_stream()
    if args.refined_only:
        out = measure_refined(args)
        if rank == 0:
            print(json.dumps(dict(out, note="refined-mesh workload only")), flush=True)
        return
    if args.clouds_only:
        out = measure_clouds(args)
        if rank == 0:
            print(json.dumps(dict(out, note="refinable-cloud workload only (profiling case)")),
                  flush=True)
        return
    if args.pc2_only:
        out = measure_pc2_strat(args, stream, lambda x: x, lambda: None)
        if rank == 0:
            print(json.dumps(dict(out, note="stratified pc2 workload only (profiling case)")), flush=True)
        return
    cells = (args.cells,) * 3 if args.cells else ((64, 64, 64) if args.small else (256, 256, 256))
    block = tuple(min(64, c) for c in cells) if not args.small else (32, 32, 32)
    ppc = (1, 1, 1, 1) if args.small else (4, 4, 4, 4)
    dev, ms, W = uniform_box(cells, block, ppc)
    npart, ncell, dt = W["npart"], W["ncell"], W["dt"]
    # the rows in cell order (SortParticles, which the reference runs every sort interval so
    # that its particles stay close to cell order), as both forms find them in a run
    dev.sort_by_cell()
    torch.cuda.synchronize()
    res = {}
    barrier, maxall = rep.barrier, rep.max_over_ranks
    # snapshot of the initial state (every run below starts from it)
    snap = (dev.t["pr"].clone(), dev.t["pi"].clone(), dev.t["u0"].clone())
    ncyc = args.warmup + args.steps
    # ---- mixed form ----
    mx = MixedDust(dev=dev, do_import=False)
    mx.import_()
    # the mixed form's own initial state (the rows rounded to its FP32 storage): the reference
    # of its momentum conservation
    mx.export()
    mom0_mixed = [float(x) for x in sum(dev.momentum())]
    if args.grid_tiles:
        mx.set_tiles(0, 0, 8)                   # DUSTB_MIXED_GRID_TILES
    if args.window_tma:
        mx.mp.variant |= 32                     # DUSTB_MIXED_WINDOW_TMA
    if args.tune:
        # the library's autotuner (dustb_mixed_tune) on this workspace: rows per tile,
        # particles per pass, persistent work-queue CTAs or one CTA per tile
        rows, chunk, grid, tms = mx.tune(GAMMA * dt)
        res["tuned"] = {"rows_per_tile": rows, "chunk": chunk,
                        "launch": "one CTA per tile" if grid else "persistent CTAs, work queue",
                        "qp_plus_operator_ms": round(tms, 3), "by": "dustb_mixed_tune"}
    for _ in range(args.warmup):
        mx.imex_cycle(dt)
    # the timed steps replay one captured cycle (a CUDA graph of its kernel launches)
    graph = mx.capture(lambda: mx.imex_cycle(dt))
    barrier()
    clk = Clocks(int(os.environ.get("LOCAL_RANK", 0)))
    clk.start()
    ms_mixed = timed_cycles(graph.replay, args.steps, stream)
    clocks = clk.stop()
    ms_mixed = maxall(ms_mixed)
    mx.export()
    torch.cuda.synchronize()
    err_mixed = dev.error_word()
    v_mixed = dev.t["pr"][[1, 3, 5], :npart].clone()
    u_mixed = ms.active(dev.t["u0"])[:, 1:4].clone()
    mom_mixed = [float(x) for x in sum(dev.momentum())]
    # the per-kernel breakdown: eager cycles with CUDA events around every launch (after the
    # state above was taken)
    nk = 3
    mx.timing(True)
    ms_eager = timed_cycles(lambda: mx.imex_cycle(dt), nk, stream)
    ktimes = mx.kernel_times()
    mx.timing(False)
    # device-resident round trip: import + cycle + export per step (the rows in the reference
    # layout before and after every step, no host copies)
    ms_dev_rt = timed_cycles(lambda: (mx.import_(), mx.imex_cycle(dt), mx.export()),
                             min(args.steps, 3), stream)
    del graph
    # the cost of the momentum ledgers (exact conservation): the same cycle with them off
    # (DUSTB_MIXED_NO_LEDGER), timed the same way
    ms_no_ledger = None
    if args.ledger_timing:
        mx.mp.variant |= 16
        mx.imex_cycle(dt)
        graph = mx.capture(lambda: mx.imex_cycle(dt))
        ms_no_ledger = maxall(timed_cycles(graph.replay, args.steps, stream))
        del graph
        mx.mp.variant &= ~16
    if args.mixed_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": rep.throughput(npart, ms_mixed),
                              "unit": UNIT, "ms_per_step": ms_mixed, "steps": args.steps,
                              "config": {"cells": ncell, "particles": npart},
                              "kernels": {k: v for k, v in ktimes.items()},
                              "roofline": roofline(ktimes, nk, npart, ncell, ms_mixed),
                              "ms_per_step_without_momentum_ledger": ms_no_ledger,
                              "note": "mixed form only (profiling case)"}), flush=True)
        return
    # ---- the storage twin: FP64 cycles with the state rounded to the mixed form's layout
    # before each (an import and an export): the reference algorithm's own response to the
    # mixed form's FP32 storage ----
    restore(dev, snap)
    for _ in range(ncyc):
        tol.storage_twin_cycle(dev, mx, dt)
    del mx
    torch.cuda.empty_cache()
    torch.cuda.synchronize()
    v_twin = dev.t["pr"][[1, 3, 5], :npart].clone()
    u_twin = ms.active(dev.t["u0"])[:, 1:4].clone()
    # ---- FP64 per-task form from the same initial state ----
    restore(dev, snap)
    mom0 = [float(x) for x in sum(dev.momentum())]
    del snap
    torch.cuda.empty_cache()
    for _ in range(args.warmup):
        dev.imex_cycle(dt)
    barrier()
    ms_fp64 = timed_cycles(lambda: dev.imex_cycle(dt), args.steps, stream)
    ms_fp64 = maxall(ms_fp64)
    torch.cuda.synchronize()
    err_fp64 = dev.error_word()
    v64 = dev.t["pr"][[1, 3, 5], :npart]
    u64 = ms.active(dev.t["u0"])[:, 1:4]
    mass = dev.t["pr"][16, :npart]
    errors = tol.compare(v_mixed, v64, u_mixed, u64, mass)
    mom64 = [float(x) for x in sum(dev.momentum())]
    ptot = max(abs(x) for x in mom0)
    errors["total_momentum_change_mixed_rel"] = max(abs(a - b) for a, b in zip(mom_mixed, mom0_mixed)) / ptot
    errors["total_momentum_change_fp64_rel"] = max(abs(a - b) for a, b in zip(mom64, mom0)) / ptot
    errors["error_words"] = [err_mixed, err_fp64]
    twin = tol.compare(v_twin, v64, u_twin, u64, mass)
    verdict = tol.judge(errors, split=True)
    del v64, u64, mass, v_mixed, u_mixed, v_twin, u_twin
    # ---- end to end through the C ABI with host buffers (mixed form) ----
    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(dev, dt, args, stream)
    roof = roofline(ktimes, nk, npart, ncell, ms_mixed)
    total_ms = sum(v[0] for v in ktimes.values()) or 1.0
    shares = {k: {"ms_per_step": round(v[0] / nk, 3), "launches_per_step": v[1] / nk,
                  "share": round(v[0] / total_ms, 3)} for k, v in ktimes.items() if v[1]}
    steps_per_s = rep.throughput(npart, ms_mixed)
    del dev
    torch.cuda.empty_cache()
    # ---- the FP64 form in the seeded (unsorted) order of the rows ----
    fp64_seeded = None
    if not args.no_seeded:
        d2, _, _ = uniform_box(cells, block, ppc)
        d2.imex_cycle(dt)
        barrier()
        ms_seed = maxall(timed_cycles(lambda: d2.imex_cycle(dt), 2, stream))
        fp64_seeded = {"ms_per_step": ms_seed, "value": rep.throughput(npart, ms_seed),
                       "steps": 2, "warmup": 1}
        del d2
        torch.cuda.empty_cache()
    fp64_best = min(ms_fp64, fp64_seeded["ms_per_step"]) if fp64_seeded else ms_fp64
    # kernels of ours per mixed cycle (dc1, consistent split): per stage gas update, count,
    # scan (3), move, Q/P tile, solve, operator tile, correction, kick tile, consistent gas
    # = 12, stage 2 adds the history term, and one ghost exchange of u0 closes the cycle:
    # 12 + 13 + 1 (the consistent dust kicks are folded into the next stage's push)
    launches_mixed = 26 * args.steps
    # ---- the stratified pc2 workload (mixed pc2 vs FP64 pc2) ----
    strat = None
    if not args.no_pc2:
        strat = measure_pc2_strat(args, stream, maxall, barrier)
    # ---- the batched ensemble of damping boxes ----
    ens = None
    if not args.no_ensemble:
        ens = measure_ensemble(args)
    # ---- refinable clouds on the uniform root mesh of config 4 ----
    clouds = None
    if not args.no_clouds:
        clouds = measure_clouds(args)
    # ---- point particles on the refined mesh of config 4 ----
    refined = None
    if not args.no_refined:
        refined = measure_refined(args)
    if rank == 0:
        cb = None if args.no_cpu else cpu_baseline()
        line = {
            "metric": METRIC, "value": steps_per_s, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed (f32 particles/weights/kicks, f64 drag factor, accumulators, gas)",
            "data": "synthetic (seeded hash)",
            "config": {"workload": f"uniform periodic {cells[0]}^3 mesh, {ms.nmb} MeshBlocks of "
                                   f"{block[0]}^3, 4 species tau_s={{0.01,0.1,1,10}}, eps 0.5, "
                                   f"ppc {ppc[0]} each, imex2+/dc1 TSC, consistent split",
                       "particles": npart, "cells": ncell, "dt": dt,
                       "dt_over_tau_s": list(W["dt_over_ts"]),
                       "rotation": "off: a uniform periodic box (config 2 names no shearing "
                                   "box); the NSH drift velocities are the initial state",
                       "l2": "inputs far larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}"},
            "fp64": {"value": rep.throughput(npart, ms_fp64), "ms_per_step": ms_fp64,
                     "order": "rows in cell order",
                     "form": "per-task FP64 kernels (reference layout, FP64 atomics), built "
                             "--fmad=false for bit parity with the oracle"},
            "fp64_seeded_order": fp64_seeded,
            "timing": {"timed": "CUDA-graph replay of one captured cycle",
                       "eager_ms_per_step": ms_eager,
                       "device_import_cycle_export_ms_per_step": ms_dev_rt,
                       "momentum_ledger": "on (gas + dust momentum to FP64 round-off)",
                       "ms_per_step_without_momentum_ledger": ms_no_ledger},
            "speedup_mixed_vs_fp64": fp64_best / ms_mixed,
            "speedup_basis": "the faster of the FP64 form's two row orders",
            "errors_mixed_vs_fp64": errors,
            "errors_storage_twin_vs_fp64": dict(twin, form="FP64 cycles with the state "
                                                "rounded to the mixed layout before each"),
            "tolerance": verdict,
            "tolerance_ok": verdict["ok"],
            "roofline": roof,
            "kernels": shares,
            "clocks": clocks,
            "gpu_launches": launches_mixed,
            "cpu_baseline": cb,
            "e2e": e2e,
            "pc2_stratified": strat,
            "ensemble": ens,
            "clouds": clouds,
            "refined": refined,
        }
        if res.get("tuned"):
            line["config"]["tuned"] = res["tuned"]
        line["config"]["gather_window"] = ("staged in shared memory by one tensor copy per tile"
                                           if args.window_tma else "loaded per thread (L1)")
        print(json.dumps(line), flush=True)


def measure_pc2_strat(args, stream, maxall, barrier):
    """Mixed pc2 cycles (CUDA-graph replay) and FP64 pc2 cycles from the same initial state of
    the stratified workload (rows in cell order), the FP64 form also in the seeded order, and
    the mixed result's errors against the FP64 one."""
    import torch
    from athenak_b200.mixed import MixedDust
    from athenak_b200.workloads import stratified_box
    dev, ms, W = stratified_box(args.small)
    npart, dt = W["npart"], W["dt"]
    steps = args.steps
    # the FP64 form in the seeded order of the rows first
    for _ in range(args.warmup):
        dev.pc2_cycle(dt)
    barrier()
    ms_seed = maxall(timed_cycles(lambda: dev.pc2_cycle(dt), steps, stream))
    del dev
    torch.cuda.empty_cache()
    dev, ms, W = stratified_box(args.small)
    dev.sort_by_cell()                        # the rows in cell order (SortParticles)
    pr0, pi0, u00 = dev.t["pr"].clone(), dev.t["pi"].clone(), dev.t["u0"].clone()
    mx = MixedDust(dev=dev, do_import=False)
    mx.import_()
    for _ in range(args.warmup):
        mx.pc2_cycle(dt)
    graph = mx.capture(lambda: mx.pc2_cycle(dt))
    barrier()
    ms_mixed = maxall(timed_cycles(graph.replay, steps, stream))
    mx.export()
    torch.cuda.synchronize()
    err_m = dev.error_word()
    v_m = dev.t["pr"][[1, 3, 5]].clone()
    rem_m = dev.t["x3_removed"].clone()
    # per-kernel breakdown (eager cycles with CUDA events; after the state above was taken)
    nk = 3
    mx.timing(True)
    timed_cycles(lambda: mx.pc2_cycle(dt), nk, stream)
    kt = mx.kernel_times()
    mx.timing(False)
    names = {"deposit_qp": "predictor", "kick": "advance"}
    tot = sum(v[0] for v in kt.values()) or 1.0
    shares = {names.get(k, k): {"ms_per_step": round(v[0] / nk, 3), "launches_per_step": v[1] / nk,
                                "share": round(v[0] / tot, 3)} for k, v in kt.items() if v[1]}
    del graph, mx
    torch.cuda.empty_cache()
    dev.t["pr"].copy_(pr0); dev.t["pi"].copy_(pi0); dev.t["u0"].copy_(u00)
    dev.t["x3_removed"].zero_()
    del pr0, pi0, u00
    for _ in range(args.warmup):
        dev.pc2_cycle(dt)
    barrier()
    ms_64 = maxall(timed_cycles(lambda: dev.pc2_cycle(dt), steps, stream))
    torch.cuda.synchronize()
    err_64 = dev.error_word()
    v64 = dev.t["pr"][[1, 3, 5]]
    mass = dev.t["pr"][16]
    dv = v_m - v64
    pd_m, pd_64 = (mass * v_m).sum(dim=1), (mass * v64).sum(dim=1)
    rem_64 = dev.t["x3_removed"]
    out = {
        "workload": "stratified shearing box 128x128x256 (16 MeshBlocks of 64^3), shear-periodic x1, "
                    "outflow x3, 7 bins St 1e-3..1 ppc 1 each, mass ~ St^0.5, Z 0.01, H_p 0.02, "
                    "pc2 TSC" if not args.small else "small 32x32x64 stratified test",
        "particles": npart, "cells": W["ncell"], "dt": dt, "mesh_time": W["t"],
        "value": npart / (ms_mixed * 1e-3), "unit": UNIT, "ms_per_step": ms_mixed,
        "steps": steps, "warmup": args.warmup, "timed": "CUDA-graph replay of one captured cycle",
        "fp64": {"value": npart / (ms_64 * 1e-3), "ms_per_step": ms_64, "order": "rows in cell order",
                 "form": "per-task FP64 kernels (reference layout, FP64 atomics)"},
        "fp64_seeded_order": {"value": npart / (ms_seed * 1e-3), "ms_per_step": ms_seed},
        "speedup_mixed_vs_fp64": min(ms_64, ms_seed) / ms_mixed,
        "speedup_basis": "the faster of the FP64 form's two row orders",
        "kernels": shares,
        "errors_mixed_vs_fp64": {
            "velocity_max_rel": float(dv.abs().max() / v64.abs().max()),
            "velocity_rms_rel": float(torch.sqrt((dv * dv).mean() / (v64 * v64).mean())),
            "dust_momentum_rel": float((pd_m - pd_64).abs().max() / pd_64.abs().max()),
            "x3_removed_mass_rel": float((rem_m[0] - rem_64[0]).abs() / rem_64[0].abs().clamp_min(1e-300)),
            "x3_removed_count": [float(rem_m[1]), float(rem_64[1])],
            "error_words": [err_m, err_64]},
    }
    out["tolerance_ok"] = (out["errors_mixed_vs_fp64"]["velocity_max_rel"] <= 1e-5 and
                           out["errors_mixed_vs_fp64"]["dust_momentum_rel"] <= 1e-6)
    del dev
    torch.cuda.empty_cache()
    return out


def measure_ensemble(args):
    """1024 independent periodic dust_damping boxes (sides log-uniform in 16..64 cells, 1-4
    species, t_s log-uniform in 1e-3..10, eps log-uniform in 0.1..10, ppc 1..8), one
    MeshBlock pack per side, each pack's cycle a replayed CUDA graph; every box checked
    against the exact solution of its damping ODE."""
    import torch
    from athenak_b200.ensemble import draw_boxes, run_ensemble, run_ensemble_one_launch
    n = 32 if args.small else 1024
    boxes = draw_boxes(n, seed=1, sides=(8, 16) if args.small else (16, 64))
    cycles = args.ensemble_cycles
    try:
        # every box resident, one CUDA-graph launch per substep
        ms, ps, ch, npk = run_ensemble_one_launch(boxes, cycles)
        timed = (f"cycles 2..{cycles}: one CUDA-graph launch per substep over all {n} boxes "
                 f"({npk} packs by side as parallel branches, reference rows detached)")
    except torch.cuda.OutOfMemoryError:
        torch.cuda.empty_cache()
        ms, ps, ch = run_ensemble(boxes, cycles)
        timed = (f"cycles 2..{cycles} of every pack (CUDA-graph replays pack by pack; the "
                 f"resident ensemble did not fit), device time summed over packs")
    worst = max(ch, key=lambda c: c["err_vs_exact"])
    # the FP64 per-task form on the same boxes, launched the same way (3 cycles: it is slow)
    from athenak_b200.ensemble import run_ensemble_fp64
    torch.cuda.empty_cache()
    try:
        ms64, ps64, err64 = run_ensemble_fp64(boxes, 3)
        fp64 = {"device_ms": ms64, "value": ps64 / (ms64 * 1e-3), "cycles": 3,
                "max_err_vs_exact_rel_v0": err64,
                "timed": "cycles 2..3: one CUDA-graph launch per substep over all boxes, the "
                         "packs' FP64 dustb_imex_cycle as parallel branches (rows in the "
                         "lattice order they are built in)"}
    except torch.cuda.OutOfMemoryError:
        torch.cuda.empty_cache()
        fp64 = {"unavailable": "the FP64 reference rows of every pack do not fit at once"}
    except RuntimeError as e:          # (a failed capture of the FP64 cycles)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        fp64 = {"unavailable": f"the FP64 arm failed: {str(e)[:200]}"}
    return {"workload": f"{n} periodic dust_damping boxes, sides log-uniform {boxes and min(b.side for b in boxes)}.."
                        f"{max(b.side for b in boxes)} cells, 1-4 species, t_s 1e-3..10, eps 0.1..10, ppc 1..8, "
                        f"imex2+/dc1 TSC, one pack per side ({len(set(b.side for b in boxes))} packs)",
            "boxes": n, "particles": int(sum(b.side ** 3 * b.ppc * len(b.taus) for b in boxes)),
            "cells": int(sum(b.side ** 3 for b in boxes)), "cycles": cycles,
            "value": ps / (ms * 1e-3), "unit": UNIT, "device_ms": ms,
            "timed": timed,
            "max_err_vs_exact_rel_v0": max(c["err_vs_exact"] for c in ch),
            "max_momentum_change_rel": max(c["momentum_change"] for c in ch),
            "worst_box": worst, "fp64": fp64,
            "speedup_mixed_vs_fp64": (ps / (ms * 1e-3)) / fp64["value"] if "value" in fp64 else None}


def measure_clouds(args):
    """Refinable clouds on config 4's root mesh without its refinement: 128^3 cells as 512
    MeshBlocks of 16^3, 2 species tau_s = {0.1, 1}, eps 0.5 each, 8 clouds per cell each
    (33.5 M level-0 P1 hat clouds), imex2+/dc1 with the overlap split, FP64 (the clouds' reference
    layout kernels); the point-particle TSC cycle of the same particles beside it, and the
    total momentum change of the cloud cycles."""
    import numpy as np
    import torch
    from athenak_b200 import capi
    from athenak_b200.drag import DeviceDust
    from athenak_b200.mesh import uniform_mesh
    cells = (32, 32, 32) if args.small else (128, 128, 128)
    ms = uniform_mesh(cells, (16, 16, 16), 2, (-0.5,) * 3, (0.5,) * 3)
    ppc, taus, eps = 8, [0.1, 1.0], [0.5, 0.5]
    ncell = ms.ncell_active
    npart = ncell * ppc * len(taus)
    phys = dict(scheme=2, drag_solver=2, back_reaction=True)
    dev = DeviceDust.empty(ms, npart, phys, nspecies=len(taus))
    d = capi.DustbSeedDesc()
    d.seed, d.nspecies = 4, len(taus)
    for s_, (t, e) in enumerate(zip(taus, eps)):
        d.ppc[s_], d.taus[s_], d.mass[s_] = ppc, t, e / (ncell * ppc)
        d.vx[s_], d.vy[s_], d.vz[s_] = 0.01 * (s_ + 1), -0.02, 0.005
    d.vel_noise, d.rho0, d.gas_noise = 1e-2, 1.0, 1e-3
    d.nb1, d.nb2, d.nb3 = ms.nblocks
    dev.seed_uniform(d)
    dev.init_gas_ghosts()
    dev.sort_by_cell()                        # the rows in cell order (SortParticles)
    dt = 0.3 / cells[0]
    pr0, pi0, u00 = dev.t["pr"].clone(), dev.t["pi"].clone(), dev.t["u0"].clone()
    steps = max(1, min(args.steps, 3))

    def timed(cycle):
        cycle()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            cycle()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    def scale():
        pr = dev.t["pr"][:, :npart]
        m = pr[16]
        dsum = torch.stack([(m * pr[r]).abs().sum() for r in (1, 3, 5)])
        u0 = ms.active(dev.t["u0"])
        gsum = u0[:, 1:4].abs().sum(dim=(0, 2, 3, 4)) * ms.cell_volume()
        return float((dsum + gsum).max())

    p0 = sum(dev.momentum())
    sc = scale()
    ms_cloud = timed(lambda: dev.cloud_imex_cycle(dt))
    p1 = sum(dev.momentum())
    err_cloud = dev.error_word()
    dev.t["pr"].copy_(pr0); dev.t["pi"].copy_(pi0); dev.t["u0"].copy_(u00)
    ms_point = timed(lambda: dev.imex_cycle(dt))
    err_point = dev.error_word()
    # the same clouds through the leaf traversal of refined meshes (the mesh as one level)
    from athenak_b200.amr import leaf_tables, uniform_leaf_spec
    dev.t["pr"].copy_(pr0); dev.t["pi"].copy_(pi0); dev.t["u0"].copy_(u00)
    dev.set_leaf_tables(leaf_tables(uniform_leaf_spec(ms)))
    ms_leaf = timed(lambda: dev.cloud_imex_cycle(dt))
    err_leaf = dev.error_word()
    out = {"workload": f"{cells[0]}^3 uniform mesh (config 4's root mesh, no refinement), "
                       f"{ms.nmb} MeshBlocks of 16^3, 2 species tau_s 0.1, 1, eps 0.5 each, "
                       f"8 level-0 P1 hat clouds per cell each, imex2+/dc1, overlap split, FP64",
           "particles": npart, "cells": ncell, "dt": dt, "steps": steps,
           "value": npart / (ms_cloud * 1e-3), "unit": UNIT, "ms_per_step": ms_cloud,
           "timed": "CUDA events around eager cycles after one warm-up cycle",
           "fp64_points_tsc": {"ms_per_step": ms_point, "value": npart / (ms_point * 1e-3)},
           "leaf_traversal": {"ms_per_step": ms_leaf, "value": npart / (ms_leaf * 1e-3),
                              "note": "the same clouds through the refined-mesh leaf traversal "
                                      "(the mesh as one level of leaf tables)"},
           "momentum_change_rel": float(np.abs(p1 - p0).max() / sc),
           "error_words": [err_cloud, err_point, err_leaf]}
    del dev, pr0, pi0, u00
    torch.cuda.empty_cache()
    return out


def measure_refined(args):
    """The SMR/AMR configuration's mesh with point particles (athenak_b200/workloads.py
    clump_refined): a 128^3 root with two more levels around a Gaussian clump, 1520 MeshBlocks
    of 16^3, per-block particle counts over 100 times apart, the FP64 imex2+ cycle on the
    refined mesh (dustb_refined_imex_cycle: the general deposit remap, the multilevel copy
    exchange, particles routed across levels, local solver, consistent split), eager cycles
    after one warm-up cycle, and the total momentum change (per-block cell volumes)."""
    import numpy as np
    import torch
    from athenak_b200.workloads import clump_refined
    dev, ms, info = clump_refined(small=args.small)
    npart, dt = info["npart"], info["dt"]
    vol = torch.from_numpy(ms.mb_size[:, 6] * ms.mb_size[:, 7] * ms.mb_size[:, 8]).to(dev.device)
    g_ = ms.ng
    n1, n2, n3 = ms.n

    def momentum():
        return momentum_n(npart)

    def momentum_n(npart):
        u0 = dev.t["u0"][:, 1:4, g_:n3 - g_, g_:n2 - g_, g_:n1 - g_].sum(dim=(2, 3, 4))
        gas = (u0 * vol[:, None]).sum(0)
        pr = dev.t["pr"][:, :npart]
        m = pr[16]
        dust = torch.stack([(m * pr[r]).sum() for r in (1, 3, 5)])
        absm = float(torch.stack([(m * pr[r]).abs().sum() for r in (1, 3, 5)]).max())
        return (gas + dust).cpu().numpy(), absm

    p0, absm = momentum()
    steps = max(1, min(args.steps, 3))
    snap = (dev.t["pr"].clone(), dev.t["pi"].clone(), dev.t["u0"].clone())

    def timed(cycle):
        cycle()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            cycle()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    ms_cyc = timed(lambda: dev.refined_imex_cycle(dt))
    p1, _ = momentum()
    err_fp64 = dev.error_word()
    v64 = dev.t["pr"][[1, 3, 5], :npart].clone()
    gid64 = dev.t["pi"][0, :npart].clone()
    # the mixed form on the same mesh from the same state (its tiles from the device work queue,
    # heaviest first: the blocks' particle counts are 125x apart)
    from athenak_b200.mixed import MixedDust
    dev.t["pr"].copy_(snap[0]); dev.t["pi"].copy_(snap[1]); dev.t["u0"].copy_(snap[2])
    mx = MixedDust(dev=dev)
    mx.export()
    pm0, _ = momentum()
    ms_mixed = timed(lambda: mx.imex_cycle(dt))
    mx.export()
    torch.cuda.synchronize()
    pm1, _ = momentum()
    vm = dev.t["pr"][[1, 3, 5], :npart]
    vscale = float(v64.abs().max())
    dvp = (vm - v64).abs().amax(dim=0)
    dv = float(dvp.max()) / vscale
    # where the largest deviations sit: particles whose block differs between the two forms
    # (a position within FP32 round-off of a block face), and the worst particle's block level
    gidm = dev.t["pi"][0, :npart]
    nmis = int((gidm != gid64).sum())
    pw = int(dvp.argmax())
    lev_w = int(ms.lloc[int(gid64[pw]), 0] - ms.root_level)
    same = gidm == gid64
    dv_same = float(dvp[same].max()) / vscale if bool(same.any()) else 0.0
    del gidm, same, dvp
    err_mixed = dev.error_word()
    del mx, v64, gid64
    torch.cuda.empty_cache()
    # refinable clouds on the same mesh from the same state: every cloud takes the level of its
    # leaf (the instant switch at level 0), one P1 split pass turns the clouds whose support
    # meets finer leaves into lobed transition clouds and their separated pieces, then imex2+
    # cycles of the clouds over the actual leaves (dustb_cloud_refined_imex_cycle)
    from athenak_b200 import capi
    from athenak_b200.amr import leaf_tables
    dev.t["pr"].copy_(snap[0]); dev.t["pi"].copy_(snap[1]); dev.t["u0"].copy_(snap[2])
    del snap
    torch.cuda.empty_cache()
    lt = leaf_tables(ms)
    dev.set_leaf_tables(lt)
    nsw = dev.cloud_instant_switch(0)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    nsplit = dev.cloud_split_p1(capi.split_params(max_level=lt.nlev), int(npart))
    b.record()
    torch.cuda.synchronize()
    ms_split = a.elapsed_time(b)
    ncl = dev.npart
    pc0, absc = momentum_n(ncl)
    ms_cloud = timed(lambda: dev.cloud_refined_imex_cycle(dt))
    pc1, _ = momentum_n(ncl)
    err_cloud = dev.error_word()
    out = {"workload": "128^3 root mesh of 16^3 MeshBlocks with two more levels around a Gaussian "
                       "dust clump (peak eps 100, sigma 0.05 L): point particles, 2 species "
                       "tau_s 0.1, 1, 1 + floor(150 exp(-r^2/2 sigma^2)) per species per cell, "
                       "imex2+ / local solver, consistent split, TSC, FP64",
           "meshblocks": info["nmb"], "blocks_per_level": info["levels"],
           "block_particles_max_over_min": info["block_particles_max_over_min"],
           "particles": npart, "cells": info["ncell"], "dt": dt, "steps": steps,
           "value": npart / (ms_cyc * 1e-3), "unit": UNIT, "ms_per_step": ms_cyc,
           "timed": "CUDA events around eager dustb_refined_imex_cycle calls after one warm-up",
           "deposit_remap_entries": info["plan_entries"],
           "momentum_change_rel": float(np.abs(p1 - p0).max() / absm),
           "mixed": {"ms_per_step": ms_mixed, "value": npart / (ms_mixed * 1e-3),
                     "speedup_vs_fp64": ms_cyc / ms_mixed,
                     "momentum_change_rel": float(np.abs(pm1 - pm0).max() / absm),
                     "velocity_max_rel_vs_fp64_after_same_cycles": dv,
                     "velocity_max_rel_same_block": dv_same,
                     "particles_in_another_block": nmis,
                     "worst_particle_level": lev_w,
                     "note": "the FP64 form ran 1 + steps cycles, the mixed form the same number "
                             "from the same state"},
           "clouds": {"ms_per_step": ms_cloud, "value": ncl / (ms_cloud * 1e-3),
                      "clouds": ncl, "switched_to_leaf_level": nsw,
                      "split_pieces_appended": nsplit, "split_pass_ms": ms_split,
                      "momentum_change_rel": float(np.abs(pc1 - pc0).max() / absc),
                      "timed": "CUDA events around eager dustb_cloud_refined_imex_cycle calls "
                               "after one warm-up (FP64 refinable clouds over the actual leaves)"},
           "error_words": [err_fp64, err_mixed, err_cloud]}
    del dev
    torch.cuda.empty_cache()
    return out


E2E_ROWS_IN = [0, 1, 2, 3, 4, 5, 15, 16]     # X, V, t_s, m
E2E_ROWS_OUT = [0, 1, 2, 3, 4, 5]            # X, V


class HostRoundTrip:
    """Steps of the mixed cycle through the C ABI with the particle rows and u0 held in pinned
    host memory: every step copies in the FP64 rows it reads (X, V, t_s, m, PGID) and u0,
    imports, runs one mixed cycle, exports, and copies out the state the next step reads
    (X, V, PGID, u0).  X1, V1 and R are the integrator's stage registers: the export writes
    them on the device, but the next cycle sets X1, V1 from X, V at its first stage and its
    first stage does not read R, so they are not copied back.

    serial: the copies in, the cycle and the copies out on one stream, one after the other.
    pipelined: the copies out run on a second stream after the export, and the next step's
    copies in on a third: each output row goes back to the device as soon as its copy to the
    host has landed (an event per row), t_s and m (inputs only, but the export may zero m)
    between them, so the two directions of the bus overlap; the cycle waits for the last copy
    in.  A step then costs the cycle plus the copies in, the copies out hidden behind them.
    K steps of either form hold K copies in, K cycles and K copies out (the pipelined form's
    copies in of step s + 1 run inside step s)."""

    def __init__(self, dev, mx, pipelined=True):
        import torch
        self.dev, self.mx, self.pipelined = dev, mx, pipelined
        n = dev.npart
        self.h_pr = torch.empty((17, n), dtype=torch.float64, pin_memory=True)
        self.h_pi = torch.empty((1, n), dtype=torch.int32, pin_memory=True)
        self.h_u0 = torch.empty_like(dev.t["u0"], device="cpu").pin_memory()
        self.h_pr.copy_(dev.t["pr"])
        # the mass as the mixed form carries it (FP32, exact in FP64), which its export writes
        # back: the host's inputs then equal what every export leaves on the device
        self.h_pr[16].copy_(self.h_pr[16].float().double())
        self.h_pi.copy_(dev.t["pi"][:1])
        self.h_u0.copy_(dev.t["u0"])
        self.bytes_in = (len(E2E_ROWS_IN) * 8 + 4) * n + self.h_u0.numel() * 8
        self.bytes_out = (len(E2E_ROWS_OUT) * 8 + 4) * n + self.h_u0.numel() * 8
        self.comp = torch.cuda.current_stream()
        self.down, self.up = torch.cuda.Stream(), torch.cuda.Stream()
        self.ready = None

    # (device tensor, host tensor) of every item a step copies
    def _outputs(self):
        d, t = self.dev.t, self
        return ([(d["pr"][r], t.h_pr[r]) for r in E2E_ROWS_OUT] +
                [(d["pi"][0], t.h_pi[0]), (d["u0"], t.h_u0)])

    def _inputs_only(self):
        return [(self.dev.t["pr"][r], self.h_pr[r]) for r in E2E_ROWS_IN if r not in E2E_ROWS_OUT]

    def _cycle(self, dt):
        self.mx.import_()
        self.mx.imex_cycle(dt)
        self.mx.export()

    def step(self, dt):
        import torch
        if not self.pipelined:
            for dv, hv in self._inputs_only() + self._outputs():
                dv.copy_(hv, non_blocking=True)
            self._cycle(dt)
            for dv, hv in self._outputs():
                hv.copy_(dv, non_blocking=True)
            return
        if self.ready is None:                       # the first step's copies in
            with torch.cuda.stream(self.up):
                self.up.wait_stream(self.comp)
                for dv, hv in self._inputs_only() + self._outputs():
                    dv.copy_(hv, non_blocking=True)
            self.ready = torch.cuda.Event()
            self.ready.record(self.up)
        self.comp.wait_event(self.ready)
        self._cycle(dt)
        exported = torch.cuda.Event()
        exported.record(self.comp)
        landed = []
        with torch.cuda.stream(self.down):
            self.down.wait_event(exported)
            for dv, hv in self._outputs():
                hv.copy_(dv, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.down)
                landed.append(ev)
        only = self._inputs_only()
        with torch.cuda.stream(self.up):
            self.up.wait_event(exported)
            for q, ((dv, hv), ev) in enumerate(zip(self._outputs(), landed)):
                if q < len(only):                    # t_s, m while row q comes back
                    only[q][0].copy_(only[q][1], non_blocking=True)
                self.up.wait_event(ev)
                dv.copy_(hv, non_blocking=True)
            for dv, hv in only[len(landed):]:
                dv.copy_(hv, non_blocking=True)
        self.ready = torch.cuda.Event()
        self.ready.record(self.up)

    def drain(self):
        """Makes the compute stream wait for every copy issued so far."""
        if self.ready is not None:
            self.comp.wait_event(self.ready)

    def timed(self, dt, steps):
        import torch
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record(self.comp)
        for _ in range(steps):
            self.step(dt)
        self.drain()
        t1.record(self.comp)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / steps


def measure_e2e(dev, dt, args, stream):
    """The metric end to end (HostRoundTrip, pipelined).  The host rows are first put in cell
    order once (dustb_sort_by_cell, the reference's SortParticles), the order a host code that
    sorts its particles keeps them in; each step's export writes every particle back to its
    own row."""
    import torch
    from athenak_b200.mixed import MixedDust
    dev.sort_by_cell()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    n = dev.npart
    mx = MixedDust(dev=dev, do_import=False)
    try:
        rt = HostRoundTrip(dev, mx, pipelined=True)
    except RuntimeError as e:
        return {"value": None, "unit": UNIT, "note": f"pinned host buffers unavailable: {e}"[:200]}
    steps = min(args.steps, 3)
    rt.step(dt)
    rt.drain()
    ms = rt.timed(dt, steps)
    out = {"value": n / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": rt.bytes_in,
           "d2h_bytes_per_step": rt.bytes_out, "ms_per_step": ms, "steps": steps,
           "path": "dustb_mixed_import + dustb_mixed_imex_cycle + dustb_mixed_export, pinned "
                   "host rows; copies out and the next step's copies in overlapped row by row"}
    del rt, mx
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="a 64^3 test workload")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the tile-shape autotuner (rows per tile, particles per pass)")
    ap.add_argument("--grid-tiles", action="store_true",
                    help="one CTA per tile instead of the work queue (profiling cases)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cells", type=int, default=0,
                    help="a cubic mesh of this many cells per side (profiling cases)")
    ap.add_argument("--mixed-only", action="store_true", help="time the mixed form only")
    ap.add_argument("--no-refined", action="store_true",
                    help="skip the refined-mesh (SMR/AMR) point-particle workload")
    ap.add_argument("--refined-only", action="store_true",
                    help="run the refined-mesh workload alone and print its object")
    ap.add_argument("--no-ledger-timing", dest="ledger_timing", action="store_false",
                    help="skip the timing of the cycle without the momentum ledgers")
    ap.add_argument("--no-pc2", action="store_true",
                    help="skip the stratified pc2 workload (128x128x256, 29.4 M particles)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the batched ensemble of 1024 damping boxes")
    ap.add_argument("--ensemble-cycles", type=int, default=20,
                    help="imex2+ cycles of every ensemble box")
    ap.add_argument("--no-clouds", action="store_true",
                    help="skip the refinable-cloud workload (128^3, 33.5 M clouds, FP64)")
    ap.add_argument("--no-seeded", action="store_true",
                    help="skip the FP64 form's timing in the seeded row order")
    ap.add_argument("--window-tma", action="store_true",
                    help="the gathering tiles stage their gas window by a tensor copy per tile")
    ap.add_argument("--clouds-only", action="store_true",
                    help="time the uniform refinable-cloud workload only (profiling case)")
    ap.add_argument("--pc2-only", action="store_true",
                    help="time the stratified pc2 workload only (profiling case)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    from athenak_b200.replicas import Replicas
    rep = Replicas(world, rank, backend="nccl", timeout_s=600)
    try:
        run_ours(args, rep)
    finally:
        rep.close()


if __name__ == "__main__":
    main()
