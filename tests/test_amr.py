"""Refined (multi-level) 3-D meshes and the general deposit remap, on the CPU.

The block tree and its 56 neighbour slots follow MeshBlock::SetNeighbors
(src/mesh/meshblock.cpp:142-420); the remap plan built by the C++ host layer
(dustb_host_dep_plan: interval overlaps over each target's neighbour list, as
DepRemapPlan does, src/bvals/bvals_dep_general.cpp:62-545) must equal the oracle's
brute-force plan (finest-level unit cubes looked up in an ownership grid) entry for entry,
and applying it must conserve the deposit exactly.
"""
import numpy as np
import pytest

from athenak_b200.amr import (build_dep_plan, neighbor_index, refined_mesh, refined_state,
                              sphere_refine, X3_FOLD, X3_DROP)
from oracle import oracle

MESHES = {
    "sphere_2lev": dict(nmbroot=(4, 4, 4), nx=(8, 8, 8), refine=sphere_refine((0.1, 0.05, -0.02),
                                                                             (0.3, 0.15))),
    "offcentre_4x2x2": dict(nmbroot=(4, 2, 2), nx=(8, 8, 8), lo=(-1.0, -0.5, -0.5),
                            hi=(1.0, 0.5, 0.5), refine=sphere_refine((0.9, 0.4, 0.45), (0.4, 0.2))),
}


def mesh(name, x3bc=0):
    return refined_mesh(x3bc=x3bc, **MESHES[name])


@pytest.mark.parametrize("name", sorted(MESHES))
def test_tree_is_balanced_and_neighbour_slots_symmetric(name):
    ms = mesh(name)
    assert ms.max_level == ms.root_level + 2
    lev = ms.lloc[:, 0]
    for m in range(ms.nmb):
        nb = ms.nghbr56[m]
        for s in range(56):
            g = nb[s]
            if g < 0:
                continue
            assert ms.nlev56[m, s] == lev[g]
            assert abs(int(lev[g]) - int(lev[m])) <= 1
            # adjacency is symmetric: the neighbour lists this block in one of its slots
            assert m in set(ms.nghbr56[g]), (m, s, g)
    # every face of every block is covered: the same-level slot, or four finer ones, or the
    # coarser neighbour in this block's own sub-slot
    for m in range(ms.nmb):
        for o in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            slots = [neighbor_index(*o, a, b) for b in (0, 1) for a in (0, 1)]
            assert (ms.nghbr56[m, slots] >= 0).any()


@pytest.mark.parametrize("x3mode", [0, X3_FOLD, X3_DROP])
@pytest.mark.parametrize("name", sorted(MESHES))
def test_plan_equals_the_bruteforce_oracle(name, x3mode):
    ms = mesh(name, x3bc=0 if x3mode == 0 else 1)
    p = build_dep_plan(ms, x3mode)
    q = oracle.dep_plan(ms, x3mode)
    assert p.nbad == 0
    assert p.nseg > 0
    for f in ("seg_tgt", "seg_ptr", "ent_src"):
        np.testing.assert_array_equal(getattr(p, f), getattr(q, f), err_msg=f)
    np.testing.assert_array_equal(p.ent_w, q.ent_w)


def _field(ms, nvar, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(ms.field_shape(nvar))


def _integrals(ms, a):
    """(active, ghost) integrals of every variable: sum of value times cell volume."""
    n1, n2, n3 = ms.n
    g = ms.ng
    vol = (ms.mb_size[:, 6] * ms.mb_size[:, 7] * ms.mb_size[:, 8])[:, None, None, None, None]
    act = np.zeros(a.shape, bool)
    act[:, :, g:n3 - g, g:n2 - g, g:n1 - g] = True
    w = a * vol
    return (w * act).sum(axis=(0, 2, 3, 4)), (w * ~act).sum(axis=(0, 2, 3, 4))


@pytest.mark.parametrize("x3mode", [0, X3_FOLD, X3_DROP])
def test_remap_conserves_the_deposit(x3mode):
    ms = mesh("sphere_2lev", x3bc=0 if x3mode == 0 else 1)
    p = build_dep_plan(ms, x3mode)
    a = _field(ms, 3, 5)
    if x3mode == X3_DROP:
        # the ghost cells beyond the physical x3 faces carry nothing (they would be dropped)
        g, n3 = ms.ng, ms.n[2]
        lo_face = ms.mb_size[:, 2] == ms.lo[2]
        hi_face = ms.mb_size[:, 5] == ms.hi[2]
        a[lo_face, :, :g] = 0.0
        a[hi_face, :, n3 - g:] = 0.0
    act0, gh0 = _integrals(ms, a)
    b = oracle.dep_apply(p, a.copy())
    act1, _ = _integrals(ms, b)
    scale = np.abs(a).max() * ms.mb_size[:, 6:9].prod(axis=1).max() * a[0, 0].size * ms.nmb
    np.testing.assert_allclose(act1, act0 + gh0, rtol=0, atol=1e-12 * scale)


def test_plan_on_a_mesh_without_refinement_is_the_same_level_exchange():
    """One level, 2x2x2 root blocks (their Z order is the lexicographic order): the general
    remap adds the same ghost deposits as the same-level exchange, in another order."""
    ms = refined_mesh((2, 2, 2), (8, 8, 8), 2, refine=None)
    p = build_dep_plan(ms, 0)
    st = refined_state(ms, [0.1], [1.0], 1, seed=3)
    o = oracle.Oracle(st, dict(scheme=2))
    a = _field(ms, 3, 11)
    o.arr["work"][...] = a
    o.ghost_add("work", 3)
    b = oracle.dep_apply(p, a.copy())
    g = ms.ng
    n1, n2, n3 = ms.n
    sl = (slice(None), slice(None), slice(g, n3 - g), slice(g, n2 - g), slice(g, n1 - g))
    np.testing.assert_allclose(b[sl], o.arr["work"][sl], rtol=0, atol=1e-13 * np.abs(a).max())


def _slot_search(ms, m, ix, iy, iz, fx, fy, fz):
    """The neighbour-slot search of SetNewPrtclGID on a refined mesh
    (src/bvals/bvals_part.cpp:312-394), restated as the device kernel route_slot_ml does it."""
    nb = ms.nghbr56[m]
    lev = ms.lloc[:, 0]
    mylevel = lev[m]

    def lev_of(s):
        return lev[nb[s]] if nb[s] >= 0 else -1

    def filled(jx, jy, jz, k):
        nd = abs(jx) + abs(jy) + abs(jz)
        end = neighbor_index(jx, jy, jz) + (4 if nd == 1 else (2 if nd == 2 else 1))
        for q in range(k, end):
            if nb[q] >= 0:
                return q
        return -1

    def coarse_cover(jx, jy, jz):
        mb = ms.mb_size[m]
        lx, ly, lz = mb[3] - mb[0], mb[4] - mb[1], mb[5] - mb[2]
        l1 = int(np.floor((mb[0] - ms.lo[0]) / lx + 0.5))
        l2 = int(np.floor((mb[1] - ms.lo[1]) / ly + 0.5))
        l3 = int(np.floor((mb[2] - ms.lo[2]) / lz + 0.5))
        kx = jx if (jx == 0 or (l1 & 1) == (1 if jx > 0 else 0)) else 0
        ky = jy if (jy == 0 or (l2 & 1) == (1 if jy > 0 else 0)) else 0
        kz = jz if (jz == 0 or (l3 & 1) == (1 if jz > 0 else 0)) else 0
        if abs(kx) + abs(ky) + abs(kz) == 0 or (kx, ky, kz) == (jx, jy, jz):
            return -1
        return filled(kx, ky, kz, neighbor_index(kx, ky, kz))

    nd = abs(ix) + abs(iy) + abs(iz)
    s = neighbor_index(ix, iy, iz)
    if nd == 1:
        if lev_of(s) > mylevel:
            sub = {0: (fy, fz), 1: (fx, fz), 2: (fx, fy)}[[ix, iy, iz].index(next(v for v in (ix, iy, iz) if v))]
            s = neighbor_index(ix, iy, iz, *sub)
        return filled(ix, iy, iz, s)
    if nd == 2:
        if lev_of(s) > mylevel:
            free = [a for a, v in enumerate((ix, iy, iz)) if v == 0][0]
            s = neighbor_index(ix, iy, iz, (fx, fy, fz)[free], 0)
        s = filled(ix, iy, iz, s)
        return s if s >= 0 else coarse_cover(ix, iy, iz)
    s = filled(ix, iy, iz, s)
    return s if s >= 0 else coarse_cover(ix, iy, iz)


def test_slot_search_finds_the_block_that_holds_the_position():
    """For points just beyond every face, edge and corner of every block (both halves of each
    transverse direction), the slot search of the route lands in the block whose box holds the
    point (periodic wrap), at every level difference."""
    ms = mesh("sphere_2lev")
    mb = ms.mb_size
    L = [ms.hi[a] - ms.lo[a] for a in range(3)]
    rng = np.random.default_rng(1)
    checked = 0
    for m in range(ms.nmb):
        lo, hi = mb[m, :3], mb[m, 3:6]
        dx = mb[m, 6:9]
        for o in [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)
                  if (a, b, c) != (0, 0, 0)]:
            for _ in range(4):
                x = np.empty(3)
                for a in range(3):
                    if o[a] < 0:
                        x[a] = lo[a] - rng.uniform(0.05, 0.9) * dx[a]
                    elif o[a] > 0:
                        x[a] = hi[a] + rng.uniform(0.05, 0.9) * dx[a]
                    else:
                        x[a] = lo[a] + rng.uniform(0.02, 0.98) * (hi[a] - lo[a])
                ix, iy, iz = [int((x[a] - lo[a] + (hi[a] - lo[a])) // (hi[a] - lo[a])) - 1
                              for a in range(3)]
                assert (ix, iy, iz) == o
                f = [0 if x[a] < 0.5 * (lo[a] + hi[a]) else 1 for a in range(3)]
                s = _slot_search(ms, m, ix, iy, iz, *f)
                assert s >= 0, (m, o)
                g = ms.nghbr56[m, s]
                w = [(x[a] - ms.lo[a]) % L[a] + ms.lo[a] for a in range(3)]
                own = np.nonzero(np.all((mb[:, :3] <= w) & (w < mb[:, 3:6]), axis=1))[0]
                assert own.tolist() == [g], (m, o, s, g, own)
                checked += 1
    assert checked == ms.nmb * 26 * 4


def _linear_field(ms, nvar, sentinel):
    """A field linear in the position of every cell centre (f_v = 1 + v + 0.3 x - 0.7 y + 1.1 z),
    with the ghost cells set to sentinel."""
    n1, n2, n3 = ms.n
    g = ms.ng
    a = np.full(ms.field_shape(nvar), sentinel)
    cen = []
    for m in range(ms.nmb):
        mb = ms.mb_size[m]
        xs = [mb[d] + (np.arange(ms.n[d]) - g + 0.5) * mb[6 + d] for d in range(3)]
        Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        cen.append((X, Y, Z))
        for v in range(nvar):
            f = 1.0 + v + 0.3 * X - 0.7 * Y + 1.1 * Z
            a[m, v, g:n3 - g, g:n2 - g, g:n1 - g] = f[g:n3 - g, g:n2 - g, g:n1 - g]
    return a, cen


def test_refined_copy_exchange_is_exact_for_a_linear_field():
    """The oracle's copy exchange of a refined mesh fills every ghost cell of a block away from
    the domain faces with the value of a linear field there: same-level copies, restrictions
    (the mean of 8 cells is the centre value) and min-mod prolongation (equal one-sided
    slopes) are all exact for it, at every level difference."""
    ms = mesh("sphere_2lev")
    st = refined_state(ms, [0.1], [1.0], 1, seed=3)
    o = oracle.Oracle(st, dict(scheme=2))
    a, cen = _linear_field(ms, 3, 1e30)
    o.arr["work"][...] = a
    o.ghost_copy_ml("work", 3)
    b = o.arr["work"]
    span = [ms.hi[d] - ms.lo[d] for d in range(3)]
    checked = 0
    for m in range(ms.nmb):
        mb = ms.mb_size[m]
        # (blocks whose ghost zone stays inside the domain: no periodic image)
        if any(mb[d] - 3 * ms.ng * mb[6 + d] < ms.lo[d] or mb[3 + d] + 3 * ms.ng * mb[6 + d] > ms.hi[d]
               for d in range(3)):
            continue
        X, Y, Z = cen[m]
        for v in range(3):
            f = 1.0 + v + 0.3 * X - 0.7 * Y + 1.1 * Z
            assert np.abs(b[m, v] - f).max() < 1e-12 * max(span), (m, v)
        checked += 1
    assert checked > 20
    assert not np.any(b >= 1e29)


def test_refined_copy_exchange_keeps_a_constant():
    ms = mesh("offcentre_4x2x2")
    st = refined_state(ms, [0.1], [1.0], 1, seed=3)
    o = oracle.Oracle(st, dict(scheme=2))
    a = np.full(ms.field_shape(3), np.nan)
    g = ms.ng
    n1, n2, n3 = ms.n
    a[:, :, g:n3 - g, g:n2 - g, g:n1 - g] = 2.5
    o.arr["work"][...] = a
    o.ghost_copy_ml("work", 3)
    np.testing.assert_array_equal(o.arr["work"], np.full(a.shape, 2.5))
