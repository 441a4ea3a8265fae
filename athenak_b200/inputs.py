"""Seeded synthetic inputs of the drag step in the reference's SoA layout.

Placement and draws follow the reference's stateless hash initial conditions
(src/pgen/dust_amr/dust_setup.hpp:36-50 HashUniform01, a SplitMix64 finaliser keyed on
particle tag + seed*0x9e3779b97f4a7c15; positions dust_setup.hpp:114-118, :159-175), the
multi-species NSH equilibrium (SolveNSHGas dust_setup.cpp:186-200, NSHDustDrift
dust_setup.hpp:58-65) and the damping test's lattice placement
(src/pgen/tests/dust_damping.cpp:115-125).  Arrays are numpy (host); the device copies are
made by the caller.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import MeshSpec, X1MIN, X2MIN, X3MIN, DX1, DX2, DX3

NREAL, NINT = 17, 5
IPX, IPVX, IPY, IPVY, IPZ, IPVZ = 0, 1, 2, 3, 4, 5
IPX1, IPVX1, IPY1, IPVY1, IPZ1, IPVZ1 = 6, 7, 8, 9, 10, 11
IPRX, IPRY, IPRZ, IPTS, IPM = 12, 13, 14, 15, 16
PGID, PTAG, PSP, PLEV, PTAGH = 0, 1, 2, 3, 4

GOLDEN64 = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
# per-coordinate key offsets of the position draws (dust_setup.hpp:116-117, :164)
KX = np.uint64(0x632BE59BD9B4E019)
KY = np.uint64(0x8CB92BAA3F3D8DD7)
KZ = np.uint64(0x58F38DED6F7C55B5)
KG = np.uint64(0x1D8E4E27C47D124F)


def seed_key(seed: int):
    """seed * 0x9e3779b97f4a7c15 modulo 2^64 (the key offset of a seed)."""
    return np.uint64((int(seed) * 0x9E3779B97F4A7C15) % (1 << 64))


def hash_uniform01(key):
    """SplitMix64 finaliser -> double in [0, 1) from the top 53 bits."""
    with np.errstate(over="ignore"):
        z = np.asarray(key, dtype=np.uint64) + GOLDEN64
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def nsh_gas(omega0, qshear, ax, eps, taus):
    """Gas (u_x, u_phi) of the multi-species NSH equilibrium with radial forcing ax."""
    b = 2.0 - qshear
    sa = sb = 0.0
    for e, t in zip(eps, taus):
        T = omega0 * t
        dd = 1.0 + 2.0 * b * T * T
        sa += e / dd
        sb += e * T / dd
    den = (1.0 + sa) ** 2 + 2.0 * b * sb * sb
    return (ax / omega0) * sb / den, -(ax / (2.0 * omega0)) * (1.0 + sa) / den


def nsh_dust(omega0, qshear, ts, ux, uphi):
    """Steady drift (v_x, v_phi) of a particle with stopping time ts."""
    T = omega0 * ts
    b = 2.0 - qshear
    vx = (ux + 2.0 * T * uphi) / (1.0 + 2.0 * b * T * T)
    return vx, uphi - b * T * vx


@dataclass
class DustState:
    mesh: MeshSpec
    pr: np.ndarray          # (17, stride) float64
    pi: np.ndarray          # (5, stride) int32
    npart: int
    u0: np.ndarray          # (nmb, 4, n3, n2, n1)
    nspecies: int
    taus: list
    eps: list
    omega0: float = 1.0
    qshear: float = 1.5
    shearing_box: bool = False

    @property
    def stride(self) -> int:
        return int(self.pr.shape[1])

    def copy(self) -> "DustState":
        return DustState(self.mesh, self.pr.copy(), self.pi.copy(), self.npart, self.u0.copy(),
                         self.nspecies, list(self.taus), list(self.eps), self.omega0,
                         self.qshear, self.shearing_box)


def _block_of(mesh: MeshSpec, x, y, z):
    """PGID of positions inside the mesh (lexicographic blocks)."""
    nb = mesh.nblocks
    L = [mesh.hi[a] - mesh.lo[a] for a in range(3)]
    bi = np.clip(((x - mesh.lo[0]) / L[0] * nb[0]).astype(np.int64), 0, nb[0] - 1)
    bj = np.clip(((y - mesh.lo[1]) / L[1] * nb[1]).astype(np.int64), 0, nb[1] - 1)
    if mesh.three_d:
        bk = np.clip(((z - mesh.lo[2]) / L[2] * nb[2]).astype(np.int64), 0, nb[2] - 1)
    else:
        bk = np.zeros_like(bi)
    m = (bk * nb[1] + bj) * nb[0] + bi
    # the block's own half-open box decides (positions on a block face)
    mb = mesh.mb_size
    for a, (c, lo_i, hi_i) in enumerate(((x, 0, 3), (y, 1, 4), (z, 2, 5))):
        if a == 2 and not mesh.three_d:
            break
        below = c < mb[m, lo_i]
        above = c >= mb[m, hi_i]
        step = [1, nb[0], nb[0] * nb[1]][a]
        m = np.where(below, m - step, np.where(above, m + step, m))
    return m.astype(np.int32)


def make_state(mesh: MeshSpec, taus, eps, ppc, seed=1, placement="random", rho0=1.0,
               shearing_box=False, omega0=1.0, qshear=1.5, etavk=0.05, gas_noise=1e-3,
               vel_noise=0.0, vd=None, vgas=(0.0, 0.0, 0.0), hp=None, capacity=None,
               ts_per_particle=None) -> DustState:
    """Seeded particles and gas.

    taus/eps/ppc: per-species stopping time, dust-to-gas ratio and particles per cell.
    placement: "random" (hash of tag + seed) or "lattice" (ppc particles at every cell
    centre, every species on every cell: the damping test's exact discrete system).
    shearing_box: NSH equilibrium velocities (gas drift + per-species dust drift) with
    radial forcing 2 Omega etavk; otherwise dust species s moves at vd[s] in x1.
    vel_noise: Gaussian (Box-Muller on two hash draws) velocity noise; gas_noise: uniform.
    hp: Gaussian heights of scale hp (stratified layer), redrawn while outside the box.
    ts_per_particle: None, or (lo, hi) -- each particle draws t_s log-uniform in [lo, hi]
    from a hash of its tag.
    """
    nspec = len(taus)
    ppc = list(ppc) if np.ndim(ppc) else [int(ppc)] * nspec
    ncells = mesh.ncell_active
    counts = [ncells * p for p in ppc]
    npart = int(sum(counts))
    stride = int(capacity or npart)
    pr = np.zeros((NREAL, stride), np.float64)
    pi = np.zeros((NINT, stride), np.int32)
    lo, hi = mesh.lo, mesh.hi
    L = [hi[a] - lo[a] for a in range(3)]
    sp = np.concatenate([np.full(c, s, np.int32) for s, c in enumerate(counts)])
    tag = np.arange(npart, dtype=np.uint64)
    if placement == "lattice":
        # every cell holds ppc_s particles of species s at its centre (dust_damping lattice)
        x = np.empty(npart); y = np.empty(npart); z = np.empty(npart)
        off = 0
        cx, cy, cz = _cell_centres(mesh)
        for s, p in enumerate(ppc):
            for r in range(p):
                sl = slice(off, off + ncells)
                x[sl], y[sl], z[sl] = cx, cy, cz
                off += ncells
    else:
        key = tag + seed_key(seed)
        x = lo[0] + hash_uniform01(key + KX) * L[0]
        y = lo[1] + hash_uniform01(key + KY) * L[1]
        if mesh.three_d:
            if hp is None:
                z = lo[2] + hash_uniform01(key + KZ) * L[2]
            else:
                z = np.zeros(npart)
                todo = np.ones(npart, bool)
                for t in range(64):
                    kz = key + KZ + np.uint64(t) * np.uint64(0x2545F4914F6CDD1D)
                    u1 = np.maximum(hash_uniform01(kz), 1e-300)
                    u2 = hash_uniform01(kz + KG)
                    zz = hp * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
                    ok = todo & (zz >= lo[2]) & (zz < hi[2])
                    z[ok] = zz[ok]
                    todo &= ~ok
                    if not todo.any():
                        break
        else:
            z = np.full(npart, 0.5 * (lo[2] + hi[2]))
    # stopping times and masses
    ts = np.asarray(taus, np.float64)[sp]
    if ts_per_particle is not None:
        tlo, thi = ts_per_particle
        u = hash_uniform01(tag + seed_key(seed) + np.uint64(0xD6E8FEB86659FD93))
        ts = np.exp(np.log(tlo) + u * (np.log(thi) - np.log(tlo)))
    vol_tot = L[0] * L[1] * (L[2] if mesh.three_d else 1.0)
    mass = np.asarray([eps[s] * rho0 * vol_tot / counts[s] for s in range(nspec)])[sp]
    # velocities
    vx = np.zeros(npart); vy = np.zeros(npart); vz = np.zeros(npart)
    ug = np.array(vgas, np.float64)
    if shearing_box:
        ax = 2.0 * omega0 * etavk
        ugx, ugp = nsh_gas(omega0, qshear, ax, eps, taus)
        ug = np.array([ugx, ugp, 0.0]) if mesh.three_d else np.array([ugx, 0.0, ugp])
        dvx, dvp = nsh_dust(omega0, qshear, ts, ugx, ugp)
        vx[:] = dvx
        if mesh.three_d:
            vy[:] = dvp
        else:
            vz[:] = dvp
    elif vd is not None:
        vx[:] = np.asarray(vd, np.float64)[sp]
    if vel_noise > 0.0:
        key = tag + seed_key(seed)
        for a, arr in enumerate((vx, vy, vz)):
            u1 = np.maximum(hash_uniform01(key + np.uint64(0x1111 * (a + 1)) + KG), 1e-300)
            u2 = hash_uniform01(key + np.uint64(0x2222 * (a + 1)) + KG)
            arr += vel_noise * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    m = _block_of(mesh, x, y, z)
    pr[IPX, :npart] = x; pr[IPY, :npart] = y; pr[IPZ, :npart] = z
    pr[IPVX, :npart] = vx; pr[IPVY, :npart] = vy; pr[IPVZ, :npart] = vz
    pr[IPX1, :npart] = x; pr[IPY1, :npart] = y; pr[IPZ1, :npart] = z
    pr[IPVX1, :npart] = vx; pr[IPVY1, :npart] = vy; pr[IPVZ1, :npart] = vz
    pr[IPTS, :npart] = ts
    pr[IPM, :npart] = mass
    pi[PGID, :npart] = m
    pi[PTAG, :npart] = (tag & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    pi[PTAGH, :npart] = (tag >> np.uint64(32)).astype(np.uint32).view(np.int32)
    pi[PSP, :npart] = sp
    # gas: rho0 everywhere (ghosts included), momentum rho0*(u + noise)
    u0 = np.zeros(mesh.field_shape(4), np.float64)
    u0[:, 0] = rho0
    for a in range(3):
        u0[:, 1 + a] = rho0 * ug[a]
    if gas_noise > 0.0:
        shp = u0[:, 1].shape
        cid = np.arange(np.prod(shp), dtype=np.uint64).reshape(shp)
        for a in range(3):
            k = cid * np.uint64(3) + np.uint64(a) + seed_key(seed) + KG
            u0[:, 1 + a] += rho0 * gas_noise * (2.0 * hash_uniform01(k) - 1.0)
    return DustState(mesh, pr, pi, npart, u0, nspec, list(taus), list(eps), omega0, qshear,
                     shearing_box)


def _cell_centres(mesh: MeshSpec):
    """Cell-centre coordinates of every active cell, block by block (k, j, i order)."""
    nx1, nx2, nx3 = mesh.nx
    mb = mesh.mb_size
    i = np.arange(nx1) + 0.5
    j = np.arange(nx2) + 0.5
    k = np.arange(nx3) + 0.5
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    xs, ys, zs = [], [], []
    for m in range(mesh.nmb):
        xs.append((mb[m, X1MIN] + I * mb[m, DX1]).ravel())
        ys.append((mb[m, X2MIN] + J * mb[m, DX2]).ravel())
        if mesh.three_d:
            zs.append((mb[m, X3MIN] + K * mb[m, DX3]).ravel())
        else:
            zs.append(np.full(I.size, 0.5 * (mb[m, X3MIN] + mb[m, 5])))
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(zs)
