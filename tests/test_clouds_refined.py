"""Refinable clouds on refined 3-D meshes: the leaf tables and the oracle's leaf traversal,
instant switch and P1 split (CPU).

The leaf tables of the C++ host layer (dustb_host_leaf_tables, BuildLeafTraversal3D) must
equal the oracle's own build integer for integer.  The oracle's traversal
(LeafTraversal3D::ForEach with the transition lobes of CloudShape1D) is pinned by properties
the reference states: every cloud's weights over the actual leaves sum to one (the deposit
puts the coupled mass into active cells exactly, at physical x3 faces too through the mirrored
part); on a uniform mesh the leaf traversal equals the uniform-mesh traversal; the P1 split
conserves mass and momentum and leaves every piece's support on leaves no coarser than its
level; the instant switch gives every plain cloud of level >= L the level max(L, its leaf's).
"""
import numpy as np
import pytest

from athenak_b200 import capi
from athenak_b200.amr import (leaf_tables, refined_mesh, refined_state, sphere_refine,
                              LeafTables)
from oracle import oracle


def _mesh(x3bc=0, nmbroot=(4, 4, 4)):
    return refined_mesh(nmbroot, (8, 8, 8), 2, refine=sphere_refine((0.1, 0.05, -0.02), (0.3, 0.15)),
                        x3bc=x3bc)


def _oracle_tables(ms):
    return leaf_tables(ms, builder=oracle.lib().oracle_leaf_tables)


def _set_codes(st, lt, mode, seed=3):
    """PLEV of every particle: its block's level ("block"), random levels 0..nlev ("random"), or
    random levels with random transition lobes ("lobed")."""
    rng = np.random.default_rng(seed)
    n = st.npart
    blev = lt.arrays["blev"][st.pi[0, :n]]
    if mode == "block":
        code = blev
    else:
        code = rng.integers(0, lt.nlev + 1, n)
        if mode == "lobed":
            lob = rng.integers(0, 4, (3, n)) * (code > 0)
            code = code | (lob[0] << 6) | (lob[1] << 4) | (lob[2] << 9)
    st.pi[3, :n] = code.astype(np.int32)


@pytest.mark.parametrize("x3bc,nmbroot", [(0, (4, 4, 4)), (1, (4, 4, 4)), (0, (2, 1, 2))])
def test_leaf_tables_match_the_oracle(x3bc, nmbroot):
    ms = _mesh(x3bc, nmbroot)
    a, b = leaf_tables(ms), _oracle_tables(ms)
    assert (a.nlev, a.nfine, a.nunsafe) == (b.nlev, b.nfine, b.nunsafe)
    assert a.nlev >= 1
    for k in LeafTables.KEYS:
        np.testing.assert_array_equal(a.arrays[k], b.arrays[k], err_msg=k)
    # every block's neighbours are distinct images, and the anchor is never its own
    # unshifted neighbour
    nn = a.arrays["nnb"]
    assert nn.min() >= 6 and nn.max() <= 64
    for m in range(ms.nmb):
        pairs = {(int(a.arrays["nb"][m, k]), *map(int, a.arrays["nbs"][m, k])) for k in range(nn[m])}
        assert len(pairs) == nn[m] and (m, 0, 0, 0) not in pairs


def _deposited_mass(o, ms):
    q = ms.active(o.arr["qdep"])[:, 0]
    vol = ms.mb_size[:, 6] * ms.mb_size[:, 7] * ms.mb_size[:, 8]
    return (q.sum(axis=(1, 2, 3)) * vol).sum()


@pytest.mark.parametrize("mode", ["block", "random", "lobed"])
@pytest.mark.parametrize("x3bc", [0, 1])
def test_leaf_weights_deposit_the_whole_mass(mode, x3bc):
    ms = _mesh(x3bc)
    st = refined_state(ms, [0.1, 1.0], [0.5, 1.0], 1, seed=5)
    lt = _oracle_tables(ms)
    _set_codes(st, lt, mode)
    o = oracle.Oracle(st, dict(scheme=2))
    o.set_leaf_tables(lt)
    a_dt = 0.05
    err = o.cloud_deposit_qp(a_dt)
    assert err == 0
    n = st.npart
    m, ts = st.pr[16, :n], st.pr[15, :n]
    want = (m * a_dt / (ts + a_dt)).sum()
    assert abs(_deposited_mass(o, ms) - want) <= 1e-13 * want


def test_leaf_traversal_equals_the_uniform_traversal():
    """On a uniform mesh the leaf traversal (every block level 0) and the uniform-mesh one
    visit the same cells with the same weights: deposits and gathers agree to round-off."""
    ms = refined_mesh((2, 2, 2), (8, 8, 8), 2, refine=None)
    st = refined_state(ms, [0.1, 1.0], [0.5, 1.0], 1, seed=9, vel_noise=0.3, gas_noise=0.2)
    lt = _oracle_tables(ms)
    st.pi[3, :st.npart] = np.random.default_rng(2).integers(0, 3, st.npart)
    uni = ms.copy() if hasattr(ms, "copy") else ms
    a = oracle.Oracle(st, dict(scheme=2))
    a.ctx.mesh.nghbr_ml = None           # the uniform-mesh traversal
    b = oracle.Oracle(st, dict(scheme=2))
    b.ctx.mesh.nghbr_ml = None
    b.set_leaf_tables(lt)
    assert a.cloud_deposit_qp(0.05) == 0 and b.cloud_deposit_qp(0.05) == 0
    scale = np.abs(a.arr["qdep"]).max()
    assert np.abs(a.arr["qdep"] - b.arr["qdep"]).max() <= 1e-13 * scale
    for o in (a, b):
        o.arr["ustar"][:] = o.arr["u0"][:, 1:4] / o.arr["u0"][:, 0:1]
        assert o.cloud_gather_kick(0.05) == 0
    n = st.npart
    for r in (1, 3, 5):
        va, vb = a.st.pr[r, :n], b.st.pr[r, :n]
        assert np.abs(va - vb).max() <= 1e-13 * np.abs(va).max()
    del uni


def test_instant_switch_takes_the_leaf_level():
    ms = _mesh()
    st = refined_state(ms, [0.1], [1.0], 1, seed=11)
    lt = _oracle_tables(ms)
    _set_codes(st, lt, "random", seed=4)
    o = oracle.Oracle(st, dict(scheme=2))
    o.set_leaf_tables(lt)
    n = st.npart
    before = o.st.pi[3, :n].copy()
    L = 1
    nch = o.cloud_instant_switch(L)
    after = o.st.pi[3, :n]
    blev = lt.arrays["blev"][st.pi[0, :n]]    # every particle lies inside its own block
    want = np.where(before >= L, np.maximum(L, blev), before)
    np.testing.assert_array_equal(after, want)
    assert nch == int((want != before).sum()) > 0


@pytest.mark.parametrize("x3bc", [0, 1])
def test_split_conserves_mass_and_momentum(x3bc):
    """Root clouds split pass by pass until no cloud is eligible: the pieces carry the parents'
    mass and momentum exactly (to round-off), keep their parents' species and stopping times,
    get fresh tags, and sit in the blocks that hold them."""
    ms = _mesh(x3bc)
    st = refined_state(ms, [0.1, 1.0], [0.5, 1.0], 1, seed=12, vel_noise=0.2)
    lt = _oracle_tables(ms)
    st.pi[3, :st.npart] = 0                  # root clouds
    o = oracle.Oracle(st, dict(scheme=2))
    o.set_leaf_tables(lt)
    sp = capi.split_params(max_level=lt.nlev)
    n0 = o.st.npart
    m0 = o.st.pr[16, :n0].sum()
    p0 = np.array([(o.st.pr[16, :n0] * o.st.pr[r, :n0]).sum() for r in (1, 3, 5)])
    tag = n0
    passes = 0
    while True:
        n = o.cloud_split_p1(sp, tag)
        tag += n
        passes += 1
        if n == 0 or passes > 6:
            break
    assert 2 <= passes <= 6
    n1 = o.st.npart
    assert n1 > n0
    pr, pi = o.st.pr[:, :n1], o.st.pi[:, :n1]
    assert abs(pr[16].sum() - m0) <= 1e-13 * m0
    for a, r in enumerate((1, 3, 5)):
        assert abs((pr[16] * pr[r]).sum() - p0[a]) <= 1e-13 * np.abs(pr[16] * pr[r]).sum()
    tags = pi[1].astype(np.int64) & 0xffffffff
    assert len(np.unique(tags)) == n1
    code = pi[3]
    assert ((code & 15) <= lt.nlev).all() and (code & ~(15 | 48 | 192 | 1536) == 0).all()
    # every piece sits in the block that holds its centre
    for p in range(0, n1, 97):
        b = pi[0, p]
        for a in range(3):
            x = pr[2 * a, p]
            assert ms.mb_size[b, a] <= x < ms.mb_size[b, 3 + a]
    # the deposit still carries the whole coupled mass
    assert o.cloud_deposit_qp(0.05) == 0
    want = (pr[16] * 0.05 / (pr[15] + 0.05)).sum()
    assert abs(_deposited_mass(o, ms) - want) <= 1e-12 * want


def test_split_budget_takes_the_first_events():
    """cloud_split_budget: the split events are taken in particle order while the pieces
    appended before them stay below the budget; the pieces appended are the first ones of the
    unbudgeted split (the same tags and rows), at least the budget and at most 26 beyond it,
    and mass and momentum are kept."""
    ms = _mesh()
    st = refined_state(ms, [0.1], [0.5], 1, seed=14, vel_noise=0.2)
    lt = _oracle_tables(ms)
    st.pi[3, :st.npart] = 0
    n0 = st.npart
    full = oracle.Oracle(st, dict(scheme=2))
    full.set_leaf_tables(lt)
    nf = full.cloud_split_p1(capi.split_params(max_level=1), n0)
    budget = 5000
    assert nf > 2 * budget
    o = oracle.Oracle(st, dict(scheme=2))
    o.set_leaf_tables(lt)
    nb = o.cloud_split_p1(capi.split_params(max_level=1, budget=budget), n0)
    assert budget <= nb <= budget + 26
    np.testing.assert_array_equal(o.st.pr[:, n0:n0 + nb], full.st.pr[:, n0:n0 + nb])
    np.testing.assert_array_equal(o.st.pi[:, n0:n0 + nb], full.st.pi[:, n0:n0 + nb])
    m0 = st.pr[16, :n0].sum()
    assert abs(o.st.pr[16, :n0 + nb].sum() - m0) <= 1e-13 * m0
    # the waiting clouds are untouched
    changed = (o.st.pi[3, :n0] != st.pi[3, :n0]) | (o.st.pr[16, :n0] != st.pr[16, :n0])
    last = int(np.nonzero(changed)[0].max())
    np.testing.assert_array_equal(o.st.pr[:, last + 1:n0], st.pr[:, last + 1:n0])
