"""ctypes front end of the CPU oracle (oracle/liboracle_dust.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker.  The product path never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from athenak_b200 import capi
from athenak_b200.inputs import DustState

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_dust.so")


def build(force: bool = False) -> str:
    """Compile the oracle with the system gcc (OpenMP if available)."""
    src = os.path.join(HERE, "dust_oracle.c")
    hdr = os.path.join(HERE, "..", "include", "dustb.h")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB
    base = ["gcc", "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-shared", "-o", LIB, src, "-lm"]
    try:
        subprocess.run(base[:4] + ["-fopenmp"] + base[4:], check=True, capture_output=True)
    except subprocess.CalledProcessError:
        subprocess.run(base, check=True, capture_output=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        P = C.POINTER(capi.DustbCtx)
        D, VP, I = C.c_double, C.c_void_p, C.c_int
        sig = {
            "oracle_set_threads": ([I], None),
            "oracle_register_copy": ([P], None),
            "oracle_gas_rk_noflux": ([P, D, D], None),
            "oracle_history_gas": ([P, D], None),
            "oracle_push_imex": ([P, D, D, D, D], None),
            "oracle_route": ([P, VP], C.c_uint),
            "oracle_deposit_qp": ([P, D, D], C.c_uint),
            "oracle_ghost_add": ([P, VP, I], None),
            "oracle_ghost_copy": ([P, VP, I, I], None),
            "oracle_solve_ustar": ([P], None),
            "oracle_dc1_sweep": ([P, D, D], C.c_uint),
            "oracle_gather_kick_pmbr": ([P, D, D], C.c_uint),
            "oracle_apply_pmbr": ([P, D], None),
            "oracle_newdt": ([P], D),
            "oracle_tstop_extrema": ([P, I, VP], None),
            "oracle_sort_order": ([P, VP, VP], None),
            "oracle_sort_particles": ([P, VP, VP], None),
            "oracle_cloud_order": ([P, VP, VP], None),
            "oracle_cloud_order_check": ([P, VP, VP, I], I),
            "oracle_pc2_predictor": ([P, D, I], C.c_uint),
            "oracle_pc2_apply_predictor": ([P, D], D),
            "oracle_pc2_midpoint": ([P], None),
            "oracle_pc2_advance": ([P, D], C.c_uint),
            "oracle_pc2_commit": ([P, D], None),
            "oracle_imex_cycle": ([P, D, D, VP, VP], C.c_uint),
            "oracle_pc2_cycle": ([P, D, VP, VP], C.c_uint),
            "oracle_phst": ([P, VP, VP, VP], C.c_uint),
            "oracle_point_gravity_density": ([P, VP], C.c_uint),
            "oracle_point_gravity_gather": ([P, VP, VP, C.c_longlong], C.c_uint),
            "oracle_point_science_fields": ([P, VP, I, I], C.c_uint),
            "oracle_point_force_field": ([P, VP, VP], None),
            "oracle_cloud_deposit_qp": ([P, D, D], C.c_uint),
            "oracle_gather_pack": ([P, VP, VP], None),
            "oracle_cloud_gather_kick": ([P, D, D, VP], C.c_uint),
            "oracle_cloud_dc1_sweep": ([P, D, D], C.c_uint),
            "oracle_cloud_apply_pmbr": ([P, D, D], None),
            "oracle_cloud_imex_cycle": ([P, D, D, VP, VP], C.c_uint),
            "oracle_cloud_pc2_cycle": ([P, D, VP, VP], C.c_uint),
            "oracle_dep_plan": ([VP, I, VP, VP, VP, VP, VP, VP, C.c_longlong, C.c_longlong], I),
            "oracle_dep_apply": ([I, VP, VP, VP, VP, VP, I, I], None),
            "oracle_ghost_copy_ml": ([P, VP, I, VP], None),
            "oracle_operator_particles": ([P, D], C.c_uint),
            "oracle_dc_correct": ([P], None),
            "oracle_leaf_tables": ([VP, I, VP, VP, VP] + [VP] * 9, I),
            "oracle_cloud_instant_switch": ([P, I], I),
            "oracle_cloud_split_p1": ([P, C.POINTER(capi.DustbCloudSplit), C.c_ulonglong], I),
        }
        for name, (args, res) in sig.items():
            f = getattr(_lib, name)
            f.argtypes = args
            f.restype = res
    return _lib


def imex2p_coeffs(gamma):
    """imex2+ tableau (src/driver/driver.cpp:278-300)."""
    g0 = [1.0, (2.0 * gamma - 1.0) / (2.0 * gamma * gamma), 1.0]
    g1 = [0.0, 1.0 - (2.0 * gamma - 1.0) / (2.0 * gamma * gamma), 0.0]
    b = [gamma, 1.0 / (2.0 * gamma), 0.0]
    atw22 = (1.0 - 2.0 * gamma * gamma) / 2.0 / gamma
    return g0, g1, b, atw22


GAMMA_DEFAULT = 1.707106781186547   # 1 + 1/sqrt(2), driver.cpp:201


class Oracle:
    """The oracle's copy of a DustState (host arrays) and its context."""

    def __init__(self, st: DustState, phys: dict, threads: int = 1):
        self.st = st.copy()
        ms = st.mesh
        self.mesh = ms
        self.arr = {
            "pr": self.st.pr, "pi": self.st.pi, "u0": self.st.u0,
            "u1": np.zeros(ms.field_shape(4)), "qdep": np.zeros(ms.field_shape(5)),
            "ustar": np.zeros(ms.field_shape(3)), "dmom": np.zeros(ms.field_shape(3)),
            "resid": np.zeros(ms.field_shape(4)), "work": np.zeros(ms.field_shape(3)),
            "mb_size": np.ascontiguousarray(ms.mb_size),
            "nghbr": np.ascontiguousarray(ms.nghbr),
            "sb_gid": np.ascontiguousarray(ms.sb_gid),
        }
        if getattr(ms, "nghbr56", None) is not None:
            self.arr["mb_lev"] = np.ascontiguousarray(ms.lloc[:, 0])
            self.arr["nghbr_ml"] = np.ascontiguousarray(ms.nghbr56)
        self.phys = dict(phys)
        self.ctx = capi.make_ctx(ms, self.arr, self.st.npart, self.st.stride, self.phys)
        self.threads = threads
        self.x3_removed = np.zeros(2)

    def set_time(self, t):
        """The mesh time the next calls use (the shear offset of shear-periodic x1 faces)."""
        self.ctx.mesh.time = float(t)

    def __getattr__(self, name):
        arr = self.__dict__.get("arr")
        if arr is not None and name in arr:
            return arr[name]
        raise AttributeError(name)

    def call(self, name, *args):
        L = lib()
        L.oracle_set_threads(self.threads)
        return getattr(L, "oracle_" + name)(C.byref(self.ctx), *args)

    # --- single tasks ---
    def register_copy(self):
        self.call("register_copy")

    def push_imex(self, gam0, gam1, beta_dt, atw_dt):
        self.call("push_imex", gam0, gam1, beta_dt, atw_dt)

    def route(self):
        return self.call("route", self.x3_removed.ctypes.data)

    def deposit_qp(self, a_dt, sh=0.0):
        return self.call("deposit_qp", a_dt, sh)

    def ghost_add(self, name, nvar):
        self.call("ghost_add", self.arr[name].ctypes.data, nvar)

    def ghost_copy(self, name, nvar, x3_bcs=1):
        self.call("ghost_copy", self.arr[name].ctypes.data, nvar, x3_bcs)

    def ghost_copy_ml(self, name, nvar):
        """The copy exchange of a refined mesh (restriction, same / coarser / finer neighbours,
        prolongation)."""
        ms = self.mesh
        cn = [ms.nx[a] // 2 + 2 * ms.ng for a in range(3)]
        ca = np.zeros(ms.nmb * nvar * cn[0] * cn[1] * cn[2])
        self.call("ghost_copy_ml", self.arr[name].ctypes.data, nvar, ca.ctypes.data)

    def solve_ustar(self):
        self.call("solve_ustar")

    def dc1_sweep(self, a_dt, sh=0.0):
        return self.call("dc1_sweep", a_dt, sh)

    def gather_kick_pmbr(self, a_dt, sh=0.0):
        return self.call("gather_kick_pmbr", a_dt, sh)

    def apply_pmbr(self, a_dt):
        self.call("apply_pmbr", a_dt)

    def history_gas(self, atw_dt):
        self.call("history_gas", atw_dt)

    def gas_rk_noflux(self, g0, g1):
        self.call("gas_rk_noflux", g0, g1)

    def newdt(self):
        return self.call("newdt")

    def tstop_extrema(self, nspecies):
        out = np.zeros(2)
        self.call("tstop_extrema", nspecies, out.ctypes.data)
        return out

    def sort_order(self):
        n = self.st.npart
        order = np.zeros(max(n, 1), np.int32)
        keys = np.zeros(max(n, 1), np.int64)
        self.call("sort_order", order.ctypes.data, keys.ctypes.data)
        return order[:n], keys[:n]

    def cloud_order(self):
        """UpdateCloudOrder's rebuild: (ord, tag)."""
        n = self.st.npart
        ord_ = np.zeros(max(n, 1), np.int32)
        tag = np.zeros(max(n, 1), np.uint64)
        self.call("cloud_order", ord_.ctypes.data, tag.ctypes.data)
        return ord_[:n], tag[:n]

    def cloud_order_check(self, ord_, tag):
        ord_ = np.ascontiguousarray(ord_, np.int32)
        tag = np.ascontiguousarray(tag, np.uint64)
        return self.call("cloud_order_check", ord_.ctypes.data, tag.ctypes.data, len(ord_))

    def sort_particles(self):
        spr = np.zeros_like(self.st.pr)
        spi = np.zeros_like(self.st.pi)
        self.call("sort_particles", spr.ctypes.data, spi.ctypes.data)
        self.st.pr[...] = spr
        self.st.pi[...] = spi

    # --- pc2 ---
    def pc2_predictor(self, dt, rate_dep=1):
        return self.call("pc2_predictor", dt, rate_dep)

    def pc2_apply_predictor(self, dt):
        return self.call("pc2_apply_predictor", dt)

    def pc2_midpoint(self):
        self.call("pc2_midpoint")

    def pc2_advance(self, dt):
        return self.call("pc2_advance", dt)

    def pc2_commit(self, wpred):
        self.call("pc2_commit", wpred)

    # --- cycles ---
    def imex_cycle(self, dt, gamma=GAMMA_DEFAULT, sh=(0.0, 0.0)):
        shv = (C.c_double * 2)(*sh)
        return self.call("imex_cycle", gamma, dt, C.cast(shv, C.c_void_p),
                         self.x3_removed.ctypes.data)

    def pc2_cycle(self, dt):
        chi = C.c_double(0.0)
        err = self.call("pc2_cycle", dt, C.cast(C.byref(chi), C.c_void_p),
                        self.x3_removed.ctypes.data)
        return err, chi.value

    # --- diagnostics ---
    def phst(self, chi=None):
        """ParticleHistory's row (16 doubles) and the error word."""
        row = np.zeros(16)
        field = np.zeros(self.mesh.field_shape(1))
        ch = None if chi is None else np.array([chi], np.float64)
        err = self.call("phst", capi.ptr(ch), field.ctypes.data, row.ctypes.data)
        return row, err

    # --- point-particle fields (self-gravity, outputs) ---
    def point_gravity_density(self):
        """DepositPointGravityDensity: (owned density field, error word)."""
        owned = np.zeros(self.mesh.field_shape(1))
        err = self.call("point_gravity_density", owned.ctypes.data)
        return owned, err

    def point_gravity_gather(self, owned):
        """GatherPointGravityAcceleration over the owned (nmb, 3, ...) field: (3 x npart, err)."""
        owned = np.ascontiguousarray(owned, np.float64)
        n = self.st.npart
        acc = np.zeros((3, max(n, 1)))
        err = self.call("point_gravity_gather", owned.ctypes.data, acc.ctypes.data, max(n, 1))
        return acc[:, :n], err

    def point_force_field(self, owned):
        """The gather's force field: owned on the active cells, the transposed remap in the
        ghost cells."""
        owned = np.ascontiguousarray(owned, np.float64)
        f = np.zeros(self.mesh.field_shape(3))
        self.call("point_force_field", owned.ctypes.data, f.ctypes.data)
        return f

    # --- refinable clouds on a uniform 3-D mesh (plain P1 hat clouds, PLEV = level) ---
    def cloud_deposit_qp(self, a_dt, sh=0.0):
        return self.call("cloud_deposit_qp", a_dt, sh)

    def gather_pack(self, v=None):
        """PackGatherField3D of v (default u*): (nmb, n3, n2, n1, 12)."""
        v = self.arr["ustar"] if v is None else np.ascontiguousarray(v, np.float64)
        ms = self.mesh
        n1, n2, n3 = ms.n
        gp = np.zeros((ms.nmb, n3, n2, n1, 12))
        self.call("gather_pack", v.ctypes.data, gp.ctypes.data)
        return gp

    def cloud_gather_kick(self, a_dt, sh=0.0, gp=None):
        gp = self.gather_pack() if gp is None else np.ascontiguousarray(gp, np.float64)
        return self.call("cloud_gather_kick", a_dt, sh, gp.ctypes.data)

    def cloud_dc1_sweep(self, a_dt, sh=0.0):
        return self.call("cloud_dc1_sweep", a_dt, sh)

    def cloud_apply_pmbr(self, a_dt, sh=0.0):
        self.call("cloud_apply_pmbr", a_dt, sh)

    def cloud_imex_cycle(self, dt, gamma=GAMMA_DEFAULT, sh=(0.0, 0.0)):
        shv = (C.c_double * 2)(*sh)
        return self.call("cloud_imex_cycle", gamma, dt, C.cast(shv, C.c_void_p),
                         self.x3_removed.ctypes.data)

    def cloud_pc2_cycle(self, dt):
        chi = C.c_double(0.0)
        err = self.call("cloud_pc2_cycle", dt, C.cast(C.byref(chi), C.c_void_p),
                        self.x3_removed.ctypes.data)
        return err, chi.value

    # --- refinable clouds on a refined 3-D mesh ---
    def set_leaf_tables(self, lt):
        """The leaf tables (athenak_b200.amr.LeafTables, host arrays): the cloud calls then
        take the leaf traversal."""
        self.leaf_arrays = {k: np.ascontiguousarray(v) for k, v in lt.arrays.items()}
        self.leaf = capi.leaf_tables_struct(self.leaf_arrays, lt.nlev, lt.nfine, lt.root_dx)
        self.ctx.mesh.leaf = C.addressof(self.leaf)

    def ensure_capacity(self, n):
        """Grows the particle rows to hold n particles (a quarter more)."""
        st = self.st
        if n <= st.stride:
            return
        cap = int(n + n // 4)
        pr = np.zeros((17, cap))
        pi = np.zeros((5, cap), np.int32)
        pr[:, :st.npart] = st.pr[:, :st.npart]
        pi[:, :st.npart] = st.pi[:, :st.npart]
        st.pr, st.pi = pr, pi
        self.arr["pr"], self.arr["pi"] = pr, pi
        self.ctx.part.pr, self.ctx.part.pi = pr.ctypes.data, pi.ctypes.data
        self.ctx.part.stride = cap

    def cloud_instant_switch(self, level_cap):
        return self.call("cloud_instant_switch", int(level_cap))

    def cloud_split_p1(self, split, tag0):
        """The moving P1 split; returns the pieces appended (npart grows by them)."""
        n = self.call("cloud_split_p1", C.byref(split), C.c_ulonglong(tag0))
        if n < 0:
            # the count alone: make room for every cloud's at most 26 pieces, then split
            self.ensure_capacity(self.st.npart * 27)
            n = self.call("cloud_split_p1", C.byref(split), C.c_ulonglong(tag0))
        self.st.npart += n
        self.ctx.part.npart = self.st.npart
        return n

    def point_science_fields(self, mass_only=False, species=-1):
        """DepositPointScienceFields: (out field with 1 or 4 vars, err)."""
        out = np.zeros(self.mesh.field_shape(1 if mass_only else 4))
        err = self.call("point_science_fields", out.ctypes.data, int(mass_only), int(species))
        return out, err

    def momentum(self):
        """Total (gas, dust) momentum vectors over active cells / live particles."""
        ms = self.mesh
        g = ms.active(self.arr["u0"])[:, 1:4].sum(axis=(0, 2, 3, 4)) * ms.cell_volume()
        n = self.st.npart
        pr = self.st.pr
        m = pr[16, :n]
        d = np.array([(m * pr[1, :n]).sum(), (m * pr[3, :n]).sum(), (m * pr[5, :n]).sum()])
        return g, d


def dep_plan(ms, x3mode=0):
    """The general deposit remap of a refined 3-D mesh by the oracle's brute-force build
    (finest-level unit cubes): an athenak_b200.amr.DepPlan."""
    from athenak_b200.amr import DepPlan, plan_geometry
    L = lib()
    geo = plan_geometry(ms, x3mode)
    lloc = np.ascontiguousarray(ms.lloc, np.int32)
    counts = np.zeros(3, np.int32)
    rc = L.oracle_dep_plan(geo.ctypes.data, ms.nmb, lloc.ctypes.data, counts.ctypes.data,
                           None, None, None, None, 0, 0)
    if rc != 0:
        raise RuntimeError(f"oracle_dep_plan failed ({rc})")
    nseg, nent = int(counts[0]), int(counts[1])
    seg_tgt = np.zeros(max(nseg, 1), np.int32)
    seg_ptr = np.zeros(nseg + 1, np.int32)
    ent_src = np.zeros(max(nent, 1), np.int32)
    ent_w = np.zeros(max(nent, 1), np.float64)
    rc = L.oracle_dep_plan(geo.ctypes.data, ms.nmb, lloc.ctypes.data, counts.ctypes.data,
                           seg_tgt.ctypes.data, seg_ptr.ctypes.data, ent_src.ctypes.data,
                           ent_w.ctypes.data, nseg, nent)
    if rc != 0:
        raise RuntimeError(f"oracle_dep_plan failed ({rc})")
    return DepPlan(seg_tgt[:nseg], seg_ptr, ent_src[:nent], ent_w[:nent])


def dep_apply(plan, a):
    """GeneralApply of plan to the (nmb, nvar, n3, n2, n1) array a, in place."""
    a = np.ascontiguousarray(a) if not a.flags.c_contiguous else a
    nvar = int(a.shape[1])
    ncell = int(a.shape[2] * a.shape[3] * a.shape[4])
    lib().oracle_dep_apply(plan.nseg, plan.seg_tgt.ctypes.data, plan.seg_ptr.ctypes.data,
                           plan.ent_src.ctypes.data, plan.ent_w.ctypes.data, a.ctypes.data,
                           nvar, ncell)
    return a
