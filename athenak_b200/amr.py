"""Multi-level (SMR/AMR) MeshBlock meshes in the layout of the C ABI, and the general deposit
remap plan built over them.

A mesh is a tree of MeshBlocks as AthenaK builds it (src/mesh/meshblock_tree.cpp): the root
grid of nmb_root blocks sits at root_level = ceil(log2(max nmb_root)) of a tree whose node
(level, lx1, lx2, lx3) has the children (level + 1, 2 lx + c1, 2 ly + c2, 2 lz + c3), child
number c1 + 2 c2 + 4 c3.  The leaves are the MeshBlocks, numbered (gid) in the depth-first
order of that child numbering (CreateZOrderedLLList).  Refinement keeps every leaf's 26
neighbours within one level of it (the tree's 2:1 balance, corners included).

Per block it gives what the dust module reads from the Mesh: ``mb_size`` (RegionSize at the
block's logical location, src/mesh/mesh.hpp:25-29), its LogicalLocation and level, and the 56
neighbour slots of ``pmb->nghbr`` (gid and level per NeighborIndex slot, filled by the rules of
MeshBlock::SetNeighbors, src/mesh/meshblock.cpp:142-420: four sub-slots per face and two per
edge for finer neighbours, the slot of this block's own sub-face for a coarser neighbour, and a
coarser neighbour of an edge or corner stored only where that edge or corner lies on the
outside of this block's parent).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .mesh import MeshSpec, dir_index

X1MIN, X2MIN, X3MIN, X1MAX, X2MAX, X3MAX, DX1, DX2, DX3 = range(9)


def neighbor_index(ix: int, iy: int, iz: int, n1: int = 0, n2: int = 0) -> int:
    """Slot of direction (ix, iy, iz), sub-slot (n1, n2), in the 56-entry neighbour table
    (NeighborIndex, src/mesh/nghbr_index.hpp:29-60)."""
    if abs(ix) + abs(iy) + abs(iz) == 0 or abs(ix * iy * iz) > 1:
        return -1
    if iz == 0:
        if ix * iy == 0:
            return abs(ix) * 2 * (ix + 1) + abs(iy) * 2 * (iy + 5) + n1 + 2 * n2
        return 16 + (ix + 1) + 2 * (iy + 1) + n1
    if ix * iy == 0:
        return 24 + abs(ix) * (ix + 9) + abs(iy) * (iy + 17) + 2 * (iz + 1) + n1 + 2 * n2
    return 48 + (ix + 1) // 2 + (iy + 1) + 2 * (iz + 1)


class _Tree:
    """The nodes of a block tree: every node that exists (leaf or refined), and the leaves."""

    def __init__(self, nmbroot, root_level, x3_periodic):
        self.nmbroot = tuple(nmbroot)
        self.root_level = root_level
        self.x3_periodic = x3_periodic
        self.nodes = set()
        self.leaves = set()
        for lz in range(nmbroot[2]):
            for ly in range(nmbroot[1]):
                for lx in range(nmbroot[0]):
                    self.leaves.add((root_level, lx, ly, lz))
        # the coarser nodes above the root grid (the nodes of the tree's upper levels)
        for lev in range(root_level + 1):
            s = root_level - lev
            for lz in range(-(-nmbroot[2] // (1 << s))):
                for ly in range(-(-nmbroot[1] // (1 << s))):
                    for lx in range(-(-nmbroot[0] // (1 << s))):
                        self.nodes.add((lev, lx, ly, lz))

    def nb(self, lev, a):
        return self.nmbroot[a] << (lev - self.root_level)

    def refine(self, node):
        lev, lx, ly, lz = node
        self.leaves.discard(node)
        for n in range(8):
            ch = (lev + 1, 2 * lx + (n & 1), 2 * ly + ((n >> 1) & 1), 2 * lz + ((n >> 2) & 1))
            self.nodes.add(ch)
            self.leaves.add(ch)

    def wrap(self, lev, lx, ly, lz):
        """The location wrapped across periodic faces; None beyond a non-periodic x3 face."""
        t = [lx, ly, lz]
        for a in range(3):
            n = self.nb(lev, a)
            if t[a] < 0 or t[a] >= n:
                if a == 2 and not self.x3_periodic:
                    return None
                t[a] %= n
        return (lev, t[0], t[1], t[2])

    def find_neighbor(self, loc, o1, o2, o3):
        """FindNeighbor (src/mesh/meshblock_tree.cpp:374-460): the node at loc's level and
        offset (o1, o2, o3) if it exists (a leaf, or a refined node whose children are the
        finer neighbours), else the coarser leaf that covers it; None beyond the mesh."""
        lev = loc[0]
        w = self.wrap(lev, loc[1] + o1, loc[2] + o2, loc[3] + o3)
        if w is None:
            return None
        if w in self.nodes:
            return w
        c = (lev - 1, w[1] >> 1, w[2] >> 1, w[3] >> 1)
        if c in self.leaves:
            return c
        raise RuntimeError("the block tree is not balanced")

    def balance(self):
        """Refines until every leaf's neighbours (26 directions) lie within one level."""
        changed = True
        while changed:
            changed = False
            for leaf in sorted(self.leaves, key=lambda t: -t[0]):
                lev = leaf[0]
                if lev <= self.root_level:
                    continue
                for o3 in (-1, 0, 1):
                    for o2 in (-1, 0, 1):
                        for o1 in (-1, 0, 1):
                            if (o1, o2, o3) == (0, 0, 0):
                                continue
                            w = self.wrap(lev, leaf[1] + o1, leaf[2] + o2, leaf[3] + o3)
                            if w is None or w in self.nodes:
                                continue
                            c = (lev - 1, w[1] >> 1, w[2] >> 1, w[3] >> 1)
                            if c in self.nodes:
                                continue
                            # two or more levels coarser: refine the covering leaf
                            g = (lev - 2, w[1] >> 2, w[2] >> 2, w[3] >> 2)
                            if g in self.leaves:
                                self.refine(g)
                                changed = True
                if changed:
                    break

    def zorder(self):
        out = []

        def walk(n):
            if n in self.leaves:
                out.append(n)
                return
            lev, lx, ly, lz = n
            for c in range(8):
                ch = (lev + 1, 2 * lx + (c & 1), 2 * ly + ((c >> 1) & 1), 2 * lz + ((c >> 2) & 1))
                if ch in self.nodes:
                    walk(ch)
        walk((0, 0, 0, 0))
        return out


def refined_mesh(nmbroot=(4, 4, 4), nx=(8, 8, 8), ng=2, lo=(-0.5,) * 3, hi=(0.5,) * 3,
                 refine=None, extra_levels=2, x3bc=0) -> MeshSpec:
    """A 3-D mesh of nmbroot root blocks of nx cells, refined by refine(level, centre) (a
    predicate on a leaf's level above the root, 0-based, and its centre) up to extra_levels
    levels above the root, then balanced.  Periodic in x1 and x2 and, unless x3bc != 0, in x3.

    The returned MeshSpec carries, besides the single-level fields: lloc (nmb, 4: level, lx1,
    lx2, lx3), nghbr56 / nlev56 (nmb, 56: gid and level per slot, -1 for none), nmbroot,
    root_level and max_level.  Its 27-slot nghbr holds the first sub-slot of each direction."""
    if ng < 2:
        raise ValueError("the dust module requires nghost >= 2")
    if min(nx) < 2 * ng:
        raise ValueError("refined meshes need blocks of at least 2 nghost cells per direction")
    root_level = max(int(np.ceil(np.log2(n))) if n > 1 else 0 for n in nmbroot)
    tree = _Tree(nmbroot, root_level, x3bc == 0)
    L = [hi[a] - lo[a] for a in range(3)]

    def centre(n):
        lev = n[0]
        return tuple(lo[a] + (n[1 + a] + 0.5) * L[a] / tree.nb(lev, a) for a in range(3))

    if refine is not None:
        for e in range(extra_levels):
            lev = root_level + e
            for leaf in sorted(tree.leaves):
                if leaf[0] == lev and refine(e, centre(leaf)):
                    tree.refine(leaf)
            tree.balance()
    leaves = tree.zorder()
    nmb = len(leaves)
    gid = {n: i for i, n in enumerate(leaves)}
    max_level = max(n[0] for n in leaves)
    mb = np.zeros((nmb, 9), np.float64)
    lloc = np.zeros((nmb, 4), np.int32)
    for m, n in enumerate(leaves):
        lloc[m] = n
        for a in range(3):
            nb = tree.nb(n[0], a)
            b = n[1 + a]
            # block edges as AthenaK forms them: a linear interpolation of the mesh extent
            f0, f1 = b / nb, (b + 1) / nb
            x0 = lo[a] * (1.0 - f0) + hi[a] * f0 if b > 0 else lo[a]
            x1 = lo[a] * (1.0 - f1) + hi[a] * f1 if b < nb - 1 else hi[a]
            mb[m, a] = x0
            mb[m, 3 + a] = x1
            mb[m, 6 + a] = (x1 - x0) / nx[a]
    ng56 = np.full((nmb, 56), -1, np.int32)
    nl56 = np.full((nmb, 56), -1, np.int32)
    for m, me in enumerate(leaves):
        lev = me[0]
        myf = [me[1 + a] & 1 for a in range(3)]
        myo = [2 * f - 1 for f in myf]

        def put(slot, node):
            ng56[m, slot] = gid[node]
            nl56[m, slot] = node[0]

        def leaf_of(node, c1, c2, c3):
            return (node[0] + 1, 2 * node[1] + c1, 2 * node[2] + c2, 2 * node[3] + c3)

        for o3 in (-1, 0, 1):
            for o2 in (-1, 0, 1):
                for o1 in (-1, 0, 1):
                    o = (o1, o2, o3)
                    nd = abs(o1) + abs(o2) + abs(o3)
                    if nd == 0:
                        continue
                    nt = tree.find_neighbor(me, o1, o2, o3)
                    if nt is None:
                        continue
                    # the child index along a crossed direction: the near half
                    ff = [1 - (o[a] + 1) // 2 if o[a] != 0 else None for a in range(3)]
                    free = [a for a in range(3) if o[a] == 0]
                    if nt not in tree.leaves:
                        # finer: the children touching this block, one sub-slot each
                        if nd == 1:
                            for fb in (0, 1):
                                for fa in (0, 1):
                                    c = list(ff)
                                    c[free[0]] = fa
                                    c[free[1]] = fb
                                    put(neighbor_index(o1, o2, o3, fa, fb), leaf_of(nt, *c))
                        elif nd == 2:
                            for fa in (0, 1):
                                c = list(ff)
                                c[free[0]] = fa
                                put(neighbor_index(o1, o2, o3, fa, 0), leaf_of(nt, *c))
                        else:
                            put(neighbor_index(o1, o2, o3), leaf_of(nt, *ff))
                        continue
                    if nt[0] == lev:
                        put(neighbor_index(o1, o2, o3), nt)
                        continue
                    # coarser: the sub-slot of this block's position on the shared face; on an
                    # edge or corner only where it lies on the outside of this block's parent
                    if nd == 1:
                        put(neighbor_index(o1, o2, o3, myf[free[0]], myf[free[1]]), nt)
                    elif nd == 2:
                        crossed = [a for a in range(3) if o[a] != 0]
                        if all(myo[a] == o[a] for a in crossed):
                            put(neighbor_index(o1, o2, o3, myf[free[0]], 0), nt)
                    else:
                        if all(myo[a] == o[a] for a in range(3)):
                            put(neighbor_index(o1, o2, o3), nt)
    ng27 = np.full((nmb, 27), -1, np.int32)
    for m in range(nmb):
        for o3 in (-1, 0, 1):
            for o2 in (-1, 0, 1):
                for o1 in (-1, 0, 1):
                    if (o1, o2, o3) != (0, 0, 0):
                        ng27[m, dir_index(o1, o2, o3)] = ng56[m, neighbor_index(o1, o2, o3)]
    spec = MeshSpec(nx=tuple(nx), nblocks=tuple(nmbroot), ng=ng, lo=tuple(lo), hi=tuple(hi),
                    three_d=True, multi_d=True, x3bc=x3bc, mb_size=mb, nghbr=ng27)
    spec.lloc = lloc
    spec.nghbr56 = ng56
    spec.nlev56 = nl56
    spec.nmbroot = tuple(nmbroot)
    spec.root_level = root_level
    spec.max_level = max_level
    return spec


def sphere_refine(centre=(0.0, 0.0, 0.0), radii=(0.3, 0.15)):
    """A refinement predicate: a leaf whose centre lies within radii[e] of centre is refined
    to the next level (e = levels above the root)."""
    def f(e, c):
        r = np.sqrt(sum((c[a] - centre[a]) ** 2 for a in range(3)))
        return e < len(radii) and r < radii[e]
    return f


def refined_state(ms: MeshSpec, taus, eps, ppc, seed=1, rho0=1.0, vel_noise=1e-3,
                  gas_noise=1e-3, vd=None):
    """Seeded particles on a refined mesh: ppc particles of each species per cell of every
    block (a finer block holds more per unit volume, as refinable clouds split into finer
    ones), uniform hash positions inside the block (keyed on tag + seed, as
    athenak_b200.inputs), the mass of a particle eps rho0 V_cell / ppc of its own block, dust
    velocity vd[s] in x1 plus Gaussian noise, gas rho0 with uniform momentum noise."""
    from .inputs import (DustState, hash_uniform01, seed_key, KX, KY, KZ, KG, NREAL, NINT,
                         IPX, IPY, IPZ, IPVX, IPVY, IPVZ, IPX1, IPY1, IPZ1, IPVX1, IPVY1,
                         IPVZ1, IPTS, IPM, PGID, PTAG, PSP, PTAGH)
    nspec = len(taus)
    ncb = ms.nx[0] * ms.nx[1] * ms.nx[2]
    per = ncb * int(ppc)
    npart = ms.nmb * nspec * per
    pr = np.zeros((NREAL, npart), np.float64)
    pi = np.zeros((NINT, npart), np.int32)
    tag = np.arange(npart, dtype=np.uint64)
    key = tag + seed_key(seed)
    blk = (np.arange(npart) // (nspec * per)).astype(np.int32)
    sp = ((np.arange(npart) // per) % nspec).astype(np.int32)
    mb = ms.mb_size
    for a, (kk, r, r1) in enumerate(((KX, IPX, IPX1), (KY, IPY, IPY1), (KZ, IPZ, IPZ1))):
        lo_, hi_ = mb[blk, a], mb[blk, 3 + a]
        x = lo_ + hash_uniform01(key + kk) * (hi_ - lo_)
        x = np.minimum(x, np.nextafter(hi_, lo_))
        pr[r] = x
        pr[r1] = x
    vol = mb[blk, 6] * mb[blk, 7] * mb[blk, 8]
    pr[IPM] = np.asarray(eps, np.float64)[sp] * rho0 * vol / int(ppc)
    pr[IPTS] = np.asarray(taus, np.float64)[sp]
    vel = [np.zeros(npart), np.zeros(npart), np.zeros(npart)]
    if vd is not None:
        vel[0] += np.asarray(vd, np.float64)[sp]
    if vel_noise > 0.0:
        for a in range(3):
            u1 = np.maximum(hash_uniform01(key + np.uint64(0x1111 * (a + 1)) + KG), 1e-300)
            u2 = hash_uniform01(key + np.uint64(0x2222 * (a + 1)) + KG)
            vel[a] += vel_noise * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    for r, r1, v in ((IPVX, IPVX1, vel[0]), (IPVY, IPVY1, vel[1]), (IPVZ, IPVZ1, vel[2])):
        pr[r] = v
        pr[r1] = v
    pi[PGID] = blk
    pi[PTAG] = (tag & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    pi[PTAGH] = (tag >> np.uint64(32)).astype(np.uint32).view(np.int32)
    pi[PSP] = sp
    u0 = np.zeros(ms.field_shape(4), np.float64)
    u0[:, 0] = rho0
    if gas_noise > 0.0:
        shp = u0[:, 1].shape
        cid = np.arange(np.prod(shp), dtype=np.uint64).reshape(shp)
        for a in range(3):
            k = cid * np.uint64(3) + np.uint64(a) + seed_key(seed) + KG
            u0[:, 1 + a] += rho0 * gas_noise * (2.0 * hash_uniform01(k) - 1.0)
    return DustState(ms, pr, pi, npart, u0, nspec, list(taus), list(eps))


# ---- the general deposit remap plan (built by the C++ host layer) ----------------------------

X3_FOLD, X3_DROP = 1, 2


def plan_geometry(ms: MeshSpec, x3mode: int = 0) -> np.ndarray:
    """The geometry ints of dustb_host_dep_plan: nx1..3, ng, nmb_root1..3, root_level,
    max_level, x3mode (0 periodic, 1 fold, 2 drop)."""
    return np.array([*ms.nx, ms.ng, *ms.nmbroot, ms.root_level, ms.max_level, x3mode], np.int32)


def _host_lib():
    from . import build
    lib = C.CDLL(build.build_host())
    f = lib.dustb_host_dep_plan
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong]
    f.restype = C.c_int
    f = lib.dustb_host_leaf_tables
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_void_p] * 9
    f.restype = C.c_int
    return lib


def leaf_geometry(ms: MeshSpec) -> np.ndarray:
    """The geometry vector of dustb_host_leaf_tables: nx1..3, nmb_root1..3, root_level,
    max_level, x3per."""
    return np.array([*ms.nx, *ms.nmbroot, ms.root_level, ms.max_level, int(ms.x3bc == 0)],
                    np.int32)


class LeafTables:
    """The leaf traversal's block geometry of a refined 3-D mesh (dustb_leaf_tables): host
    arrays, the finest grid's levels and extent, the root cell size."""

    KEYS = ("fbox", "blev", "nnb", "nb", "nbs", "nbmax", "safe", "lockey", "locblk")

    def __init__(self, arrays: dict, nlev: int, nfine, root_dx, nunsafe: int = 0):
        self.arrays = arrays
        self.nlev = int(nlev)
        self.nfine = tuple(int(v) for v in nfine)
        self.root_dx = tuple(float(v) for v in root_dx)
        self.nunsafe = int(nunsafe)


def empty_leaf_arrays(nmb: int) -> dict:
    mx = 64
    return dict(fbox=np.zeros((nmb, 6), np.int32), blev=np.zeros(nmb, np.int32),
                nnb=np.zeros(nmb, np.int32), nb=np.full((nmb, mx), -1, np.int32),
                nbs=np.zeros((nmb, mx, 3), np.int32), nbmax=np.zeros(nmb, np.int32),
                safe=np.zeros((nmb, 3), np.int32), lockey=np.zeros(nmb, np.int64),
                locblk=np.zeros(nmb, np.int32))


def root_cell_size(ms: MeshSpec):
    return tuple((ms.hi[a] - ms.lo[a]) / (ms.nmbroot[a] * ms.nx[a]) for a in range(3))


def uniform_leaf_spec(ms: MeshSpec):
    """A uniform 3-D mesh (blocks numbered (b3 nb2 + b2) nb1 + b1) in the terms of the leaf
    tables: every block at the root level, its same-level neighbours in the first sub-slot of
    each NeighborIndex direction."""
    from types import SimpleNamespace
    nb1, nb2, nb3 = ms.nblocks
    root = max(int(np.ceil(np.log2(n))) if n > 1 else 0 for n in ms.nblocks)
    lloc = np.zeros((ms.nmb, 4), np.int32)
    ng56 = np.full((ms.nmb, 56), -1, np.int32)
    for m in range(ms.nmb):
        b1, b2, b3 = m % nb1, (m // nb1) % nb2, m // (nb1 * nb2)
        lloc[m] = (root, b1, b2, b3)
        for o3 in (-1, 0, 1):
            for o2 in (-1, 0, 1):
                for o1 in (-1, 0, 1):
                    if o1 or o2 or o3:
                        ng56[m, neighbor_index(o1, o2, o3, 0, 0)] = ms.nghbr[m, dir_index(o1, o2, o3)]
    return SimpleNamespace(nx=ms.nx, nmbroot=tuple(ms.nblocks), root_level=root, max_level=root,
                           x3bc=ms.x3bc, lloc=lloc, nghbr56=ng56, nmb=ms.nmb, lo=ms.lo, hi=ms.hi)


def leaf_tables(ms: MeshSpec, builder=None) -> LeafTables:
    """The tables of a refined 3-D mesh from the C++ host layer (dustb_host_leaf_tables), or
    from builder (a function of the same signature: the oracle's own build in the tests)."""
    if builder is None:
        lib = _host_lib()
        builder = lib.dustb_host_leaf_tables
    geo = leaf_geometry(ms)
    lloc = np.ascontiguousarray(ms.lloc, np.int32)
    ng56 = np.ascontiguousarray(ms.nghbr56, np.int32)
    arr = empty_leaf_arrays(ms.nmb)
    info = np.zeros(5, np.int32)
    rc = builder(geo.ctypes.data, ms.nmb, lloc.ctypes.data, ng56.ctypes.data, info.ctypes.data,
                 *(arr[k].ctypes.data for k in LeafTables.KEYS))
    if rc != 0:
        raise RuntimeError(f"leaf tables: the build failed ({rc})")
    return LeafTables(arr, info[0], info[1:4], root_cell_size(ms), info[4])


class DepPlan:
    """Host arrays of a general deposit remap: per target cell (flat index m ncell + cell of the
    padded block arrays) its source ghost cells (same flat index) and weights (overlap volume
    over target cell volume), targets ascending and each target's sources by (source gid,
    source cell).  nbad: source ghost cells not covered exactly once (0 on a valid mesh)."""

    def __init__(self, seg_tgt, seg_ptr, ent_src, ent_w, nbad=0):
        self.seg_tgt = np.ascontiguousarray(seg_tgt, np.int32)
        self.seg_ptr = np.ascontiguousarray(seg_ptr, np.int32)
        self.ent_src = np.ascontiguousarray(ent_src, np.int32)
        self.ent_w = np.ascontiguousarray(ent_w, np.float64)
        self.nbad = int(nbad)

    @property
    def nseg(self) -> int:
        return int(self.seg_tgt.size)


def build_dep_plan(ms: MeshSpec, x3mode: int = 0) -> DepPlan:
    """The plan of a refined 3-D mesh from the C++ host layer (dustb_host_dep_plan)."""
    lib = _host_lib()
    geo = plan_geometry(ms, x3mode)
    lloc = np.ascontiguousarray(ms.lloc, np.int32)
    ng56 = np.ascontiguousarray(ms.nghbr56, np.int32)
    counts = np.zeros(3, np.int32)
    rc = lib.dustb_host_dep_plan(geo.ctypes.data, ms.nmb, lloc.ctypes.data, ng56.ctypes.data,
                                 counts.ctypes.data, None, None, None, None, 0, 0)
    if rc != 0:
        raise RuntimeError(f"dustb_host_dep_plan failed ({rc})")
    nseg, nent = int(counts[0]), int(counts[1])
    seg_tgt = np.zeros(max(nseg, 1), np.int32)
    seg_ptr = np.zeros(nseg + 1, np.int32)
    ent_src = np.zeros(max(nent, 1), np.int32)
    ent_w = np.zeros(max(nent, 1), np.float64)
    rc = lib.dustb_host_dep_plan(geo.ctypes.data, ms.nmb, lloc.ctypes.data, ng56.ctypes.data,
                                 counts.ctypes.data, seg_tgt.ctypes.data, seg_ptr.ctypes.data,
                                 ent_src.ctypes.data, ent_w.ctypes.data, nseg, nent)
    if rc != 0:
        raise RuntimeError(f"dustb_host_dep_plan failed ({rc})")
    return DepPlan(seg_tgt[:nseg], seg_ptr, ent_src[:nent], ent_w[:nent], counts[2])


def host_lib_path() -> str:
    from . import build
    return os.path.abspath(build.HOST_LIB)
