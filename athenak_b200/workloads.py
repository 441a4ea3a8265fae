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
