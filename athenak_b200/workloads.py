"""Seeded synthetic workloads of the drag step, generated on the device (dustb_seed_uniform).

uniform_box: the FP64-vs-mixed workload on a uniform periodic mesh of MeshBlocks (at full size
256^3 cells in 64 MeshBlocks of 64^3, 4 species t_s = {0.01, 0.1, 1, 10}/Omega, eps 0.5 each,
ppc 4 each: 268,435,456 particles).  Positions are the reference's hash draws keyed on tag +
seed (src/pgen/dust_amr/dust_setup.hpp:36-50); velocities the NSH drift of each species
(dust_setup.hpp:58-65) plus Gaussian 1e-3 c_s noise; the gas the NSH drift plus 1e-3 uniform
noise.  The time step is the CFL step dt = 0.3 dx / (c_s + |v|_max) with the cell width chosen
so that dt / t_s reaches `stiffness` for the shortest stopping time (10: dt/t_s spans 0.01..10
over the four species).  The rotation terms are off: the mesh is a uniform periodic box, not a
shearing box, and the NSH drift is the initial state.

stratified_box: the stratified streaming-instability set-up with a continuous size
distribution (inputs/dust_amr/si3d_strat_continuous.athinput at 128x128x256), pc2 coupling.
"""
from __future__ import annotations

import math

import numpy as np

GAMMA = 1.707106781186547          # 1 + 1/sqrt(2), the imex2+ gamma (src/driver/driver.cpp:201)
TAUS4 = [0.01, 0.1, 1.0, 10.0]


def uniform_box_geometry(cells, taus=TAUS4, eps=(0.5, 0.5, 0.5, 0.5), stiffness=10.0):
    """Cell width, box size and dt of the uniform-mesh workload: dt = stiffness * min(t_s),
    the CFL step 0.3 dx / (c_s + |v|_max) of the cell width dx."""
    from .inputs import nsh_gas
    om, q, etavk = 1.0, 1.5, 0.05
    ugx, ugp = nsh_gas(om, q, 2 * om * etavk, list(eps), list(taus))
    vmax = max(abs(ugx), abs(ugp)) + 3e-3
    dt = stiffness * min(taus)
    dx = dt * (1.0 + vmax) / 0.3
    return dict(dt=dt, dx=dx, L=[dx * c for c in cells], ug=(ugx, ugp))


def uniform_box(cells=(256, 256, 256), block=(64, 64, 64), ppc=(4, 4, 4, 4), taus=TAUS4,
                eps=(0.5, 0.5, 0.5, 0.5), stiffness=10.0, seed=1, consistent=True,
                device="cuda"):
    """The uniform-mesh workload; returns (DeviceDust, MeshSpec, info).  info: npart, ncell,
    dt, dx, L, taus, c_max (the largest drag factor a dt / (t_s + a dt) of the imex2+ stage)."""
    from . import capi
    from .drag import DeviceDust
    from .inputs import nsh_dust
    from .mesh import uniform_mesh
    om, q = 1.0, 1.5
    g = uniform_box_geometry(cells, taus, eps, stiffness)
    dt, dx, L = g["dt"], g["dx"], g["L"]
    ugx, ugp = g["ug"]
    ms = uniform_mesh(tuple(cells), tuple(block), 2, tuple(-x / 2 for x in L),
                      tuple(x / 2 for x in L))
    ncell = ms.ncell_active
    npart = ncell * sum(ppc)
    phys = dict(scheme=2, drag_solver=2, consistent_gas=bool(consistent), back_reaction=True)
    dev = DeviceDust.empty(ms, npart, phys, device=device, nspecies=len(taus))
    d = capi.DustbSeedDesc()
    d.seed = seed
    d.nspecies = len(taus)
    vol = float(np.prod(L))
    for s in range(len(taus)):
        d.ppc[s] = ppc[s]
        d.taus[s] = taus[s]
        d.mass[s] = eps[s] * 1.0 * vol / (ncell * ppc[s])
        vx, vp = nsh_dust(om, q, taus[s], ugx, ugp)
        d.vx[s], d.vy[s], d.vz[s] = vx, vp, 0.0
    d.vel_noise = 1e-3
    d.rho0 = 1.0
    d.ug[0], d.ug[1], d.ug[2] = ugx, ugp, 0.0
    d.gas_noise = 1e-3
    d.nb1, d.nb2, d.nb3 = ms.nblocks
    dev.seed_uniform(d)
    a_dt = GAMMA * dt
    info = dict(npart=npart, ncell=ncell, dt=dt, dx=dx, L=L, taus=list(taus), eps=list(eps),
                cells=tuple(cells), block=tuple(block), ppc=tuple(ppc),
                c_max=a_dt / (min(taus) + a_dt),
                dt_over_ts=(dt / max(taus), dt / min(taus)))
    return dev, ms, info


def stratified_box(small=False, device="cuda"):
    """The stratified set-up: a 3-D shearing box with shear-periodic x1 faces, vertical gravity
    and outflow x3 faces, cells of 0.00625 H, MeshBlocks of 64^3; 7 bins of equal width in
    ln St over St 1e-3..1, 1 particle per bin per cell, each with its own St inside its bin
    and mass ~ St^0.5, total Z = 0.01 of the gas; Gaussian heights of scale H_p = 0.02 H; NSH
    drift of each particle's own St plus 1e-3 Gaussian noise; gas rho = 1 with the NSH drift
    of the bins plus 1e-3 noise (the hydro's own stratified gas is outside the drag step);
    pc2 coupling, TSC.  Returns (DeviceDust, MeshSpec, info)."""
    from . import capi
    from .drag import DeviceDust
    from .inputs import nsh_gas
    from .mesh import uniform_mesh
    cells = (32, 32, 64) if small else (128, 128, 256)
    nblock = (16, 16, 32) if small else (64, 64, 64)
    dxc = 0.00625
    hi = tuple(0.5 * dxc * c for c in cells)
    ms = uniform_mesh(cells, nblock, 2, tuple(-h for h in hi), hi, x3bc=2, shear_x1=True)
    nspec, slope, Z, hp = 7, 0.5, 0.01, 0.02
    lo_t, hi_t = 1e-3, 1.0
    w = (math.log(hi_t) - math.log(lo_t)) / nspec
    tmid = [math.exp(math.log(lo_t) + (s + 0.5) * w) for s in range(nspec)]
    share = np.array([t ** slope for t in tmid])
    share /= share.sum()
    ncell = ms.ncell_active
    npart = ncell * nspec
    vol = float(np.prod([2 * h for h in hi]))
    # mean of (t/t_mid)^slope over a log-uniform bin of width w
    mean_w = math.sinh(slope * w / 2) / (slope * w / 2)
    om, q, etavk = 1.0, 1.5, 0.05
    ugx, ugp = nsh_gas(om, q, 2 * om * etavk, list(Z * share), tmid)
    phys = dict(scheme=2, drag_solver=2, shearing_box=True, stratified=True, back_reaction=True,
                qshear=q, omega0=om)
    dev = DeviceDust.empty(ms, npart, phys, device=device, nspecies=nspec)
    d = capi.DustbSeedDesc()
    d.seed = 3
    d.nspecies = nspec
    for s in range(nspec):
        d.ppc[s] = 1
        d.taus[s] = tmid[s]
        d.mass[s] = Z * vol * share[s] / (ncell * mean_w)
    d.ts_lo, d.ts_hi, d.mass_slope, d.hp = lo_t, hi_t, slope, hp
    d.nsh, d.omega0, d.qshear = 1, om, q
    d.vel_noise = 1e-3
    d.rho0 = 1.0
    d.ug[0], d.ug[1], d.ug[2] = ugx, ugp, 0.0
    d.gas_noise = 1e-3
    d.nb1, d.nb2, d.nb3 = ms.nblocks
    dev.seed_uniform(d)
    t0 = 3.7                                   # a mesh time with a non-zero shear offset
    dev.set_time(t0)
    dev.init_gas_ghosts()
    dt = 0.3 * dxc / (1.0 + q * om * hi[0])
    return dev, ms, dict(npart=npart, ncell=ncell, dt=dt, t=t0, cells=cells)


def clump_refined(small=False, peak_ppc=150, seed=4, device="cuda"):
    """The refined-mesh workload of the SMR/AMR configuration with point particles: a 128^3 root
    mesh (8^3 MeshBlocks of 16^3) with two more levels around a Gaussian dust clump at the
    centre (peak eps = 100, sigma = 0.05 L; the root blocks within 0.33 L of the clump refined
    once, the level-1 blocks within 0.16 L once more: 1520 blocks, 424 / 648 / 448 per level),
    2 species t_s = {0.1, 1}/Omega.  Every cell of every block holds 1 + floor(peak_ppc *
    exp(-r^2 / 2 sigma^2)) particles of each species (in the clump's centre blocks more than 100
    times as many per block as far from it), placed uniformly in the cell, of mass
    eps(x) rho V / n / 2 with eps = 0.01 + 100 exp(-r^2 / 2 sigma^2); velocities 1e-2 Gaussian
    noise, gas rho = 1 at rest plus 1e-3 noise; the rows in cell order (as the sort keeps
    them); dt from a CFL of 0.3 on the finest cells.  Generated on the device (torch's
    seeded Philox stream: the placement only sets where the work lies).  small: a 32^3 root of
    16^3 blocks refined the same way.  Returns (DeviceDust, MeshSpec, info)."""
    import torch
    from .amr import refined_mesh, build_dep_plan
    from .drag import DeviceDust
    L, sigma, peak_eps, eps_bg = 1.0, 0.05, 100.0, 0.01
    taus = [0.1, 1.0]
    nroot = (2, 2, 2) if small else (8, 8, 8)

    def refine(e, c):
        r = math.sqrt(sum(x * x for x in c))
        return r < (0.33 * L if e == 0 else 0.16 * L)

    ms = refined_mesh(nroot, (16, 16, 16), 2, (-L / 2,) * 3, (L / 2,) * 3, refine=refine)
    dev_ = torch.device(device)
    gen = torch.Generator(device=dev_)
    gen.manual_seed(seed)
    nx = 16
    mb = torch.from_numpy(ms.mb_size).to(dev_)
    nmb = ms.nmb
    # every active cell: block, (k, j, i), centre, volume
    kk, jj, ii = torch.meshgrid(torch.arange(nx, device=dev_), torch.arange(nx, device=dev_),
                                torch.arange(nx, device=dev_), indexing="ij")
    cm = torch.arange(nmb, device=dev_).repeat_interleave(nx ** 3)
    ck, cj, ci = (t.reshape(-1).repeat(nmb) for t in (kk, jj, ii))
    dx = mb[cm, 6:9]
    cen = mb[cm, 0:3] + (torch.stack([ci, cj, ck], 1).double() + 0.5) * dx
    r2 = (cen ** 2).sum(1)
    g = torch.exp(-r2 / (2.0 * sigma ** 2))
    ncell_p = 1 + torch.floor(peak_ppc * g).long()            # per species
    vol = dx.prod(1)
    eps = eps_bg + peak_eps * g
    nper = int(ncell_p.sum().item())
    npart = 2 * nper
    phys = dict(scheme=2, drag_solver=0, consistent_gas=True, back_reaction=True)
    dev = DeviceDust.empty(ms, npart, phys, device=device, nspecies=2)
    pr, pi = dev.t["pr"], dev.t["pi"]
    # cell of every particle of one species (cell order), then the two species cell by cell
    cid = torch.repeat_interleave(torch.arange(cm.numel(), device=dev_), ncell_p)
    cell2 = torch.repeat_interleave(torch.arange(cm.numel() * 2, device=dev_),
                                    ncell_p.repeat_interleave(2))
    c = cell2 // 2
    sp = (cell2 % 2).int()
    u = torch.rand((npart, 3), generator=gen, device=dev_, dtype=torch.float64)
    lo = mb[cm[c], 0:3] + torch.stack([ci[c], cj[c], ck[c]], 1).double() * dx[c]
    pos = lo + u * dx[c]
    for a, (rx, rx1) in enumerate(((0, 6), (2, 8), (4, 10))):
        pr[rx] = pos[:, a]
        pr[rx1] = pos[:, a]
    vel = 1e-2 * torch.randn((npart, 3), generator=gen, device=dev_, dtype=torch.float64)
    for a, (rv, rv1) in enumerate(((1, 7), (3, 9), (5, 11))):
        pr[rv] = vel[:, a]
        pr[rv1] = vel[:, a]
    pr[15] = torch.tensor(taus, device=dev_, dtype=torch.float64)[sp.long()]
    pr[16] = 0.5 * eps[c] * vol[c] / ncell_p[c].double()
    pi[0] = cm[c].int()
    tag = torch.arange(npart, device=dev_, dtype=torch.int64)
    pi[1] = (tag & 0xFFFFFFFF).int()            # PTAG the low word, PTAGH the high
    pi[2] = sp
    pi[4] = (tag >> 32).int()
    u0 = dev.t["u0"]
    u0[:, 0] = 1.0
    u0[:, 1:4] = 1e-3 * (2.0 * torch.rand(u0[:, 1:4].shape, generator=gen, device=dev_,
                                           dtype=torch.float64) - 1.0)
    del cid, cell2, u, lo, pos, vel, c, sp
    torch.cuda.synchronize()
    plan = build_dep_plan(ms, 0)
    dev.set_dep_plan(plan)
    counts = torch.zeros(nmb, device=dev_, dtype=torch.long)
    counts.index_add_(0, cm, 2 * ncell_p)
    counts = counts.cpu().numpy()
    dxmin = float(ms.mb_size[:, 6].min())
    dt = 0.3 * dxmin / (1.0 + 0.05)
    info = dict(npart=npart, ncell=int(cm.numel()), nmb=nmb, dt=dt,
                levels=np.bincount(ms.lloc[:, 0])[ms.root_level:].tolist(),
                block_particles_max_over_min=float(counts.max() / counts.min()),
                plan_entries=int(plan.ent_src.size))
    return dev, ms, info
