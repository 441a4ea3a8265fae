"""Uniform single-level MeshBlock geometry in the layout of the C ABI (include/dustb.h).

Mirrors what AthenaK's Mesh hands the dust module on one rank: ``mb_size`` (RegionSize of
every MeshBlock, src/mesh/mesh.hpp:25-29), the index ranges of ``mb_indcs``
(src/mesh/mesh.cpp:320-360: js = ks = 0 in a collapsed direction) and, per block, the gid
of the same-level neighbour in each of the 26 directions (the first sub-slot
NeighborIndex(ox1, ox2, ox3, 0, 0) of ``pmb->nghbr``, src/mesh/nghbr_index.hpp:29).
Blocks are numbered lexicographically, x1 fastest.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# RegionSize field order
X1MIN, X2MIN, X3MIN, X1MAX, X2MAX, X3MAX, DX1, DX2, DX3 = range(9)


def dir_index(o1: int, o2: int, o3: int) -> int:
    """Slot of direction (o1, o2, o3) in the 27-entry neighbour table."""
    return (o3 + 1) * 9 + (o2 + 1) * 3 + (o1 + 1)


@dataclass
class MeshSpec:
    nx: tuple            # active cells per MeshBlock (nx1, nx2, nx3)
    nblocks: tuple       # MeshBlocks per direction
    ng: int
    lo: tuple
    hi: tuple
    three_d: bool
    multi_d: bool
    x3bc: int            # 0 periodic, 1 reflect, 2 outflow
    mb_size: np.ndarray = field(repr=False)   # (nmb, 9) float64
    nghbr: np.ndarray = field(repr=False)     # (nmb, 27) int32
    gids: int = 0
    shear_x1: bool = False                    # shear-periodic x1 faces (3-D shearing box)

    @property
    def sb_gid(self) -> np.ndarray:
        """(2, nb3, nb2) int32: gid of the inner (0) and outer (1) x1-face block at (b3, b2)
        (blocks are numbered (b3*nb2 + b2)*nb1 + b1)."""
        nb1, nb2, nb3 = self.nblocks
        t = np.zeros((2, nb3, nb2), np.int32)
        for b3 in range(nb3):
            for b2 in range(nb2):
                t[0, b3, b2] = (b3 * nb2 + b2) * nb1 + self.gids
                t[1, b3, b2] = (b3 * nb2 + b2) * nb1 + nb1 - 1 + self.gids
        return t

    @property
    def nmb(self) -> int:
        return int(self.mb_size.shape[0])

    @property
    def n(self):
        """Padded extents (n1, n2, n3) of one block's mesh arrays."""
        n1 = self.nx[0] + 2 * self.ng
        n2 = self.nx[1] + 2 * self.ng if self.multi_d else 1
        n3 = self.nx[2] + 2 * self.ng if self.three_d else 1
        return n1, n2, n3

    @property
    def starts(self):
        """(is, js, ks) of the active cells."""
        return (self.ng, self.ng if self.multi_d else 0, self.ng if self.three_d else 0)

    @property
    def ncell_active(self) -> int:
        return self.nmb * self.nx[0] * self.nx[1] * self.nx[2]

    def field_shape(self, nvar: int):
        n1, n2, n3 = self.n
        return (self.nmb, nvar, n3, n2, n1)

    def active(self, a):
        """View of the active cells of a (nmb, nvar, n3, n2, n1) array."""
        is_, js, ks = self.starts
        return a[:, :, ks:ks + self.nx[2], js:js + self.nx[1], is_:is_ + self.nx[0]]

    def cell_volume(self) -> float:
        v = self.mb_size[0, DX1] * self.mb_size[0, DX2]
        if self.three_d:
            v *= self.mb_size[0, DX3]
        return float(v)


def uniform_mesh(ncells=(32, 32, 32), nblock=(16, 16, 16), ng=2,
                 lo=(-0.5, -0.5, -0.5), hi=(0.5, 0.5, 0.5), x3bc=0,
                 shear_x1=False) -> MeshSpec:
    """A uniform mesh of ncells cells split into blocks of nblock cells; periodic in x1, x2
    and, unless x3bc != 0, in x3; shear_x1: the x1 faces are shear-periodic (3-D)."""
    three_d = ncells[2] > 1
    multi_d = ncells[1] > 1
    if not multi_d:
        raise ValueError("the dust step needs a 2-D or 3-D mesh")
    for a in range(3):
        if ncells[a] % nblock[a]:
            raise ValueError("mesh cells must be a multiple of the block cells")
    if ng < 2:
        raise ValueError("the dust module requires nghost >= 2")
    nb = tuple(ncells[a] // nblock[a] for a in range(3))
    nmb = nb[0] * nb[1] * nb[2]
    L = [hi[a] - lo[a] for a in range(3)]
    mb = np.zeros((nmb, 9), np.float64)
    ng_tab = np.full((nmb, 27), -1, np.int32)
    for bk in range(nb[2]):
        for bj in range(nb[1]):
            for bi in range(nb[0]):
                m = (bk * nb[1] + bj) * nb[0] + bi
                b = (bi, bj, bk)
                for a in range(3):
                    # block edges as AthenaK forms them: a linear interpolation of the mesh
                    # extent at the block's logical location
                    f0 = b[a] / nb[a]
                    f1 = (b[a] + 1) / nb[a]
                    x0 = lo[a] * (1.0 - f0) + hi[a] * f0 if b[a] > 0 else lo[a]
                    x1 = lo[a] * (1.0 - f1) + hi[a] * f1 if b[a] < nb[a] - 1 else hi[a]
                    mb[m, a] = x0
                    mb[m, 3 + a] = x1
                    mb[m, 6 + a] = (x1 - x0) / nblock[a]
                for o3 in (-1, 0, 1):
                    for o2 in (-1, 0, 1):
                        for o1 in (-1, 0, 1):
                            if (o1, o2, o3) == (0, 0, 0):
                                continue
                            if not three_d and o3 != 0:
                                continue
                            t = [bi + o1, bj + o2, bk + o3]
                            ok = True
                            for a in range(3):
                                if t[a] < 0 or t[a] >= nb[a]:
                                    if a == 2 and x3bc != 0:
                                        ok = False
                                    t[a] %= nb[a]
                            if ok:
                                ng_tab[m, dir_index(o1, o2, o3)] = (t[2] * nb[1] + t[1]) * nb[0] + t[0]
    if not three_d:
        mb[:, X3MIN] = lo[2]
        mb[:, X3MAX] = hi[2]
        mb[:, DX3] = hi[2] - lo[2]
    if shear_x1 and not three_d:
        raise ValueError("shear-periodic x1 faces need a 3-D mesh")
    return MeshSpec(nx=tuple(nblock), nblocks=nb, ng=ng, lo=tuple(lo), hi=tuple(hi),
                    three_d=three_d, multi_d=multi_d, x3bc=x3bc, mb_size=mb, nghbr=ng_tab,
                    shear_x1=bool(shear_x1))


def box_ensemble_mesh(side: int, nbox: int, ng: int = 2, L: float = 1.0) -> MeshSpec:
    """nbox independent periodic boxes of side^3 cells as one MeshBlock pack: every block
    covers the same domain [0, L]^3 and is its own neighbour in all 26 directions (a
    periodic box of one MeshBlock), so one call of the drag step advances every box."""
    if ng < 2:
        raise ValueError("the dust module requires nghost >= 2")
    mb = np.zeros((nbox, 9), np.float64)
    mb[:, X1MAX] = mb[:, X2MAX] = mb[:, X3MAX] = L
    mb[:, DX1] = mb[:, DX2] = mb[:, DX3] = L / side
    nb = np.full((nbox, 27), -1, np.int32)
    for d in range(27):
        if d != dir_index(0, 0, 0):
            nb[:, d] = np.arange(nbox, dtype=np.int32)
    return MeshSpec(nx=(side, side, side), nblocks=(nbox, 1, 1), ng=ng, lo=(0.0,) * 3,
                    hi=(L,) * 3, three_d=True, multi_d=True, x3bc=0, mb_size=mb, nghbr=nb)
