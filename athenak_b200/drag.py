"""Host front end of the drag step: device arrays in the reference layout plus the task
calls of DustGasDrag, each forwarding to one C-ABI entry point (include/dustb.h).

torch is used only to own device memory and streams; every computation is a kernel of
libdustb.so.  The task names follow the reference's DustGasDrag members
(src/dust/dust_pm.cpp, dust_push.cpp, dust_solver.cpp, dust_newdt.cpp).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .inputs import DustState

GAMMA_DEFAULT = 1.707106781186547   # 1 + 1/sqrt(2), src/driver/driver.cpp:201


class _null:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


def _stream_ptr(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


class DeviceDust:
    """One MeshBlockPack's dust state on the GPU, in the reference layout."""

    def __init__(self, st: DustState, phys: dict, device="cuda", stride=None):
        if not torch.cuda.is_available():
            raise RuntimeError("the dust drag step runs on a CUDA device only")
        self.lib = capi.load()
        self.mesh = st.mesh
        self.device = torch.device(device)
        self.npart = st.npart
        self.nspecies = st.nspecies
        ms = st.mesh
        f64 = dict(dtype=torch.float64, device=self.device)
        self.stride = int(stride or st.stride)
        pr = torch.zeros((17, self.stride), **f64)
        pi = torch.zeros((5, self.stride), dtype=torch.int32, device=self.device)
        pr[:, :st.stride].copy_(torch.from_numpy(st.pr[:, :min(st.stride, self.stride)]))
        pi[:, :st.stride].copy_(torch.from_numpy(st.pi[:, :min(st.stride, self.stride)]))
        self.t = {
            "pr": pr, "pi": pi,
            "u0": torch.from_numpy(st.u0).to(self.device),
            "u1": torch.zeros(ms.field_shape(4), **f64),
            "qdep": torch.zeros(ms.field_shape(5), **f64),
            "ustar": torch.zeros(ms.field_shape(3), **f64),
            "dmom": torch.zeros(ms.field_shape(3), **f64),
            "resid": torch.zeros(ms.field_shape(4), **f64),
            "work": torch.zeros(ms.field_shape(3), **f64),
            "mb_size": torch.from_numpy(np.ascontiguousarray(ms.mb_size)).to(self.device),
            "nghbr": torch.from_numpy(np.ascontiguousarray(ms.nghbr)).to(self.device),
            "sb_gid": torch.from_numpy(np.ascontiguousarray(ms.sb_gid)).to(self.device),
            "err": torch.zeros(1, dtype=torch.int32, device=self.device),
            "x3_removed": torch.zeros(2, **f64),
            "scalar": torch.zeros(2, **f64),
        }
        if getattr(ms, "nghbr56", None) is not None:
            # a refined mesh: block levels and the 56 neighbour slots
            self.t["mb_lev"] = torch.from_numpy(np.ascontiguousarray(ms.lloc[:, 0])).to(self.device)
            self.t["nghbr_ml"] = torch.from_numpy(np.ascontiguousarray(ms.nghbr56)).to(self.device)
        self.phys = dict(phys)
        self._rebuild_ctx()

    @classmethod
    def empty(cls, mesh, npart, phys, device="cuda", nspecies=1):
        """Zeroed device arrays for npart particles (filled by seed_uniform)."""
        from .inputs import DustState
        st = DustState(mesh, np.zeros((17, 1)), np.zeros((5, 1), np.int32), 0,
                       np.zeros((mesh.nmb, 4, 1, 1, 1)), nspecies, [], [])
        self = cls.__new__(cls)
        self.lib = capi.load()
        self.mesh = mesh
        self.device = torch.device(device)
        self.npart = int(npart)
        self.nspecies = nspecies
        self.stride = int(npart)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.t = {
            "pr": torch.zeros((17, self.stride), **f64),
            "pi": torch.zeros((5, self.stride), dtype=torch.int32, device=self.device),
            "u0": torch.zeros(mesh.field_shape(4), **f64),
            "u1": torch.zeros(mesh.field_shape(4), **f64),
            "qdep": torch.zeros(mesh.field_shape(5), **f64),
            "ustar": torch.zeros(mesh.field_shape(3), **f64),
            "dmom": torch.zeros(mesh.field_shape(3), **f64),
            "resid": torch.zeros(mesh.field_shape(4), **f64),
            "work": torch.zeros(mesh.field_shape(3), **f64),
            "mb_size": torch.from_numpy(np.ascontiguousarray(mesh.mb_size)).to(self.device),
            "nghbr": torch.from_numpy(np.ascontiguousarray(mesh.nghbr)).to(self.device),
            "sb_gid": torch.from_numpy(np.ascontiguousarray(mesh.sb_gid)).to(self.device),
            "err": torch.zeros(1, dtype=torch.int32, device=self.device),
            "x3_removed": torch.zeros(2, **f64),
            "scalar": torch.zeros(2, **f64),
        }
        if getattr(mesh, "nghbr56", None) is not None:
            # a refined mesh: block levels and the 56 neighbour slots
            self.t["mb_lev"] = torch.from_numpy(np.ascontiguousarray(mesh.lloc[:, 0])).to(self.device)
            self.t["nghbr_ml"] = torch.from_numpy(np.ascontiguousarray(mesh.nghbr56)).to(self.device)
        self.phys = dict(phys)
        self._rebuild_ctx()
        return self

    def seed_uniform(self, desc, stream=None):
        rc = self.lib.dustb_seed_uniform(self.pctx, C.byref(desc), _stream_ptr(stream))
        capi.check(rc, "seed_uniform")

    def init_gas_ghosts(self, stream=None):
        """Gives u0's ghost cells the values a step expects (the hydro's exchange and boundary
        values agree with the cells they stand for): the copy exchange, then the planes
        beyond physical x3 faces copied from the block's edge plane, ghost columns included.
        For generated states, whose every cell (ghosts included) is drawn independently."""
        self.ghost_copy("u0", int(self.t["u0"].shape[1]), x3_bcs=0, stream=stream)
        ms = self.mesh
        if not (ms.three_d and ms.x3bc):
            return
        u = self.t["u0"]
        ng, nx3 = ms.ng, ms.nx[2]
        nb = np.asarray(ms.nghbr)
        lo = torch.from_numpy(np.nonzero(nb[:, 4] < 0)[0]).to(self.device)    # no block below
        hi = torch.from_numpy(np.nonzero(nb[:, 22] < 0)[0]).to(self.device)   # none above
        with torch.cuda.stream(stream) if stream is not None else _null():
            if lo.numel():
                u[lo, :, :ng] = u[lo, :, ng:ng + 1].expand(-1, -1, ng, -1, -1)
            if hi.numel():
                u[hi, :, ng + nx3:] = u[hi, :, ng + nx3 - 1:ng + nx3].expand(-1, -1, ng, -1, -1)

    def _rebuild_ctx(self):
        self.ctx = capi.make_ctx(self.mesh, self.t, self.npart, self.stride, self.phys)
        self.ctx.mesh.time = self.__dict__.get("time", 0.0)
        if self.__dict__.get("leaf") is not None:
            self.ctx.mesh.leaf = C.addressof(self.leaf)
        self.pctx = C.byref(self.ctx)

    def ensure_capacity(self, n):
        """Grows the particle rows to hold n particles (a quarter more), live rows kept."""
        if n <= self.stride:
            return
        cap = int(n + n // 4)
        pr = torch.zeros((17, cap), dtype=torch.float64, device=self.device)
        pi = torch.zeros((5, cap), dtype=torch.int32, device=self.device)
        pr[:, :self.npart].copy_(self.t["pr"][:, :self.npart])
        pi[:, :self.npart].copy_(self.t["pi"][:, :self.npart])
        self.t["pr"], self.t["pi"] = pr, pi
        self.stride = cap
        self._rebuild_ctx()

    def detach_rows(self):
        """Frees the reference rows (pr, pi) and passes them as detached (NULL, npart kept):
        between a mixed import and export only the shadow and the mesh fields are used."""
        self.t["pr"] = None
        self.t["pi"] = None
        self._rebuild_ctx()

    def attach_rows(self, pr, pi):
        """Attaches reference rows (17 x stride float64, 5 x stride int32 device tensors)."""
        self.t["pr"], self.t["pi"] = pr, pi
        self.stride = int(pr.shape[1])
        self._rebuild_ctx()

    def set_time(self, t):
        """The mesh time the next calls use (the shear offset of shear-periodic x1 faces)."""
        self.time = float(t)
        self.ctx.mesh.time = self.time

    def __getattr__(self, name):
        t = self.__dict__.get("t")
        if t is not None and name in t:
            return t[name]
        raise AttributeError(name)

    def _call(self, name, *args, stream=None):
        rc = getattr(self.lib, "dustb_" + name)(self.pctx, *args, _stream_ptr(stream))
        capi.check(rc, name)

    # ---- tasks (one C-ABI call each) ----
    def register_copy(self, stream=None):
        self._call("register_copy", stream=stream)

    def gas_rk_noflux(self, g0, g1, stream=None):
        self._call("gas_rk_noflux", g0, g1, stream=stream)

    def history_gas(self, atw_dt, stream=None):
        self._call("history_gas", atw_dt, stream=stream)

    def push_imex(self, gam0, gam1, beta_dt, atw_dt, stream=None):
        self._call("push_imex", gam0, gam1, beta_dt, atw_dt, stream=stream)

    def route(self, stream=None):
        self._call("route", self.t["x3_removed"].data_ptr(), stream=stream)

    def deposit_qp(self, a_dt, sh=0.0, stream=None):
        self._call("deposit_qp", a_dt, sh, stream=stream)

    def ghost_add(self, name, nvar, stream=None):
        self._call("ghost_add", self.t[name].data_ptr(), nvar, stream=stream)

    def ghost_copy(self, name, nvar, x3_bcs=1, stream=None):
        self._call("ghost_copy", self.t[name].data_ptr(), nvar, x3_bcs, stream=stream)

    def set_dep_plan(self, plan):
        """The general deposit remap of a refined mesh (athenak_b200.amr.DepPlan), copied to
        the device; ghost_add_plan applies it."""
        dev = dict(device=self.device)
        self.t["plan_tgt"] = torch.from_numpy(plan.seg_tgt).to(**dev)
        self.t["plan_ptr"] = torch.from_numpy(plan.seg_ptr).to(**dev)
        self.t["plan_src"] = torch.from_numpy(plan.ent_src).to(**dev)
        self.t["plan_w"] = torch.from_numpy(plan.ent_w).to(**dev)
        self.plan = capi.DustbDepPlan(plan.nseg, self.t["plan_tgt"].data_ptr(),
                                      self.t["plan_ptr"].data_ptr(),
                                      self.t["plan_src"].data_ptr(),
                                      self.t["plan_w"].data_ptr())

    def ghost_copy_ml(self, name, nvar, stream=None):
        """The copy exchange of a refined mesh (dustb_ghost_copy_ml) with its coarse-array
        scratch."""
        nb = int(self.lib.dustb_ghost_copy_ml_bytes(C.byref(self.ctx.mesh), nvar))
        if nb <= 0:
            raise RuntimeError("dustb_ghost_copy_ml_bytes rejected the mesh")
        ca = self.t.get("coarse")
        if ca is None or ca.numel() * 8 < nb:
            ca = self.t["coarse"] = torch.empty(nb // 8, dtype=torch.float64, device=self.device)
        self._call("ghost_copy_ml", self.t[name].data_ptr(), nvar, ca.data_ptr(), nb,
                   stream=stream)

    def ghost_add_plan(self, name, nvar, stream=None):
        """MeshBoundaryValuesDep's general path on a refined mesh: the ghost deposits of name
        remapped by the plan of set_dep_plan (dustb_ghost_add_plan)."""
        self._call("ghost_add_plan", C.byref(self.plan), self.t[name].data_ptr(), nvar,
                   stream=stream)

    def solve_ustar(self, stream=None):
        self._call("solve_ustar", stream=stream)

    def dc1_sweep(self, a_dt, sh=0.0, stream=None):
        self._call("dc1_sweep", a_dt, sh, stream=stream)

    def gather_kick_pmbr(self, a_dt, sh=0.0, stream=None):
        self._call("gather_kick_pmbr", a_dt, sh, stream=stream)

    def apply_pmbr(self, a_dt, stream=None):
        self._call("apply_pmbr", a_dt, stream=stream)

    def newdt(self, dt_cfl=1.0, stream=None):
        out = self.t["scalar"]
        self._call("newdt", dt_cfl, out.data_ptr(), stream=stream)
        return out[0]

    def tstop_extrema(self, stream=None):
        out = self.t["scalar"]
        self._call("tstop_extrema", out.data_ptr(), stream=stream)
        return out

    def pc2_predictor(self, dt, rate_dep=1, stream=None):
        self._call("pc2_predictor", dt, rate_dep, stream=stream)

    def pc2_apply_predictor(self, dt, stream=None):
        out = self.t["scalar"]
        self._call("pc2_apply_predictor", dt, out.data_ptr(), stream=stream)
        return out[0]

    def pc2_midpoint(self, stream=None):
        self._call("pc2_midpoint", stream=stream)

    def pc2_advance(self, dt, stream=None):
        self._call("pc2_advance", dt, stream=stream)

    def pc2_commit(self, wpred, stream=None):
        self._call("pc2_commit", wpred, stream=stream)

    # ---- cycles ----
    def imex_cycle(self, dt, gamma=GAMMA_DEFAULT, sh=(0.0, 0.0), stream=None):
        co = capi.DustbImexCoeffs()
        co.gamma, co.dt = gamma, dt
        co.sh[0], co.sh[1] = sh
        rc = self.lib.dustb_imex_cycle(self.pctx, C.byref(co), self.t["x3_removed"].data_ptr(),
                                       _stream_ptr(stream))
        capi.check(rc, "imex_cycle")

    def refined_imex_cycle(self, dt, gamma=GAMMA_DEFAULT, stream=None):
        """One imex2+ cycle on a refined mesh (dustb_refined_imex_cycle) with the plan of
        set_dep_plan."""
        co = capi.DustbImexCoeffs()
        co.gamma, co.dt = gamma, dt
        nb = int(self.lib.dustb_ghost_copy_ml_bytes(C.byref(self.ctx.mesh),
                                                    int(self.t["u0"].shape[1])))
        ca = self.t.get("coarse")
        if ca is None or ca.numel() * 8 < nb:
            ca = self.t["coarse"] = torch.empty(nb // 8, dtype=torch.float64, device=self.device)
        rc = self.lib.dustb_refined_imex_cycle(self.pctx, C.byref(self.plan), C.byref(co),
                                               ca.data_ptr(), nb, self.t["x3_removed"].data_ptr(),
                                               _stream_ptr(stream))
        capi.check(rc, "refined_imex_cycle")

    def pc2_cycle(self, dt, stream=None):
        out = self.t["scalar"]
        rc = self.lib.dustb_pc2_cycle(self.pctx, dt, out.data_ptr(),
                                      self.t["x3_removed"].data_ptr(), _stream_ptr(stream))
        capi.check(rc, "pc2_cycle")
        return out[0]

    def phst(self, chi_max=None, stream=None):
        """ParticleHistory's row (16 doubles, on the device): particle sums, the densest
        cell of the mass deposit, chi_max (a device scalar, or None)."""
        n = int(self.lib.dustb_phst_scratch_bytes(C.byref(self.ctx.mesh), self.npart))
        s = self.t.get("phst_scratch")
        if s is None or s.numel() < n:
            s = torch.empty(n, dtype=torch.uint8, device=self.device)
            self.t["phst_scratch"] = s
        row = torch.zeros(16, dtype=torch.float64, device=self.device)
        chi = 0 if chi_max is None else chi_max.data_ptr()
        self._call("phst", chi, row.data_ptr(), s.data_ptr(), s.numel(), stream=stream)
        return row

    # ---- refinable clouds on a uniform 3-D mesh ----
    def cloud_deposit_qp(self, a_dt, sh=0.0, stream=None):
        self._call("cloud_deposit_qp", a_dt, sh, stream=stream)

    def _gpack(self):
        n = int(self.lib.dustb_cloud_gpack_bytes(C.byref(self.ctx.mesh))) // 8
        gp = self.t.get("gpack")
        if gp is None or gp.numel() < n:
            gp = torch.empty(n, dtype=torch.float64, device=self.device)
            self.t["gpack"] = gp
        return gp

    def cloud_gather_kick(self, a_dt, sh=0.0, stream=None):
        gp = self._gpack()
        self._call("cloud_gather_kick", a_dt, sh, gp.data_ptr(), stream=stream)
        return gp

    def cloud_dc1_sweep(self, a_dt, sh=0.0, stream=None):
        self._call("cloud_dc1_sweep", a_dt, sh, self._gpack().data_ptr(), stream=stream)

    def cloud_apply_pmbr(self, a_dt, sh=0.0, stream=None):
        self._call("cloud_apply_pmbr", a_dt, sh, stream=stream)

    def cloud_imex_cycle(self, dt, gamma=GAMMA_DEFAULT, sh=(0.0, 0.0), stream=None):
        co = capi.DustbImexCoeffs()
        co.gamma, co.dt = gamma, dt
        co.sh[0], co.sh[1] = sh
        self._call("cloud_imex_cycle", C.byref(co), self._gpack().data_ptr(),
                   self.t["x3_removed"].data_ptr(), stream=stream)

    # ---- refinable clouds on a refined 3-D mesh ----
    def set_leaf_tables(self, lt):
        """The leaf traversal's block geometry (athenak_b200.amr.LeafTables) copied to the
        device and set in the mesh: the cloud calls then integrate over the actual leaves."""
        tabs = {k: torch.from_numpy(np.ascontiguousarray(v)).to(self.device)
                for k, v in lt.arrays.items()}
        if self.t.get("nghbr_ml") is not None:
            nb = int(self.lib.dustb_ghost_copy_ml_bytes(C.byref(self.ctx.mesh), 3))
            tabs["coarse"] = torch.empty(nb // 8, dtype=torch.float64, device=self.device)
        for k, v in tabs.items():
            self.t["leaf_" + k] = v
        self.leaf = capi.leaf_tables_struct(tabs, lt.nlev, lt.nfine, lt.root_dx)
        self._rebuild_ctx()

    def cloud_refined_imex_cycle(self, dt, gamma=GAMMA_DEFAULT, stream=None):
        """One imex2+ cycle of the clouds on a refined mesh (dustb_cloud_refined_imex_cycle)."""
        co = capi.DustbImexCoeffs()
        co.gamma, co.dt = gamma, dt
        nb = int(self.lib.dustb_ghost_copy_ml_bytes(C.byref(self.ctx.mesh),
                                                    int(self.t["u0"].shape[1])))
        ca = self.t.get("coarse")
        if ca is None or ca.numel() * 8 < nb:
            ca = self.t["coarse"] = torch.empty(nb // 8, dtype=torch.float64, device=self.device)
        self._call("cloud_refined_imex_cycle", C.byref(co), self._gpack().data_ptr(),
                   ca.data_ptr(), nb, self.t["x3_removed"].data_ptr(), stream=stream)

    def cloud_instant_switch(self, level_cap, stream=None) -> int:
        """CloudInstantSwitch (dustb_cloud_instant_switch); returns the clouds changed."""
        n = C.c_int(0)
        s = self.t.get("switch_scratch")
        if s is None:
            s = self.t["switch_scratch"] = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._call("cloud_instant_switch", int(level_cap), C.byref(n), s.data_ptr(),
                   stream=stream)
        return int(n.value)

    def cloud_split_p1(self, split, tag0, stream=None) -> int:
        """The moving P1 split (dustb_cloud_split_p1) with new tags from tag0; the rows grow when
        the pieces need room.  Returns the pieces appended (npart grows by them)."""
        nb = int(self.lib.dustb_cloud_split_scratch_bytes(self.npart))
        s = self.t.get("split_scratch")
        if s is None or s.numel() < nb:
            s = self.t["split_scratch"] = torch.empty(nb, dtype=torch.uint8, device=self.device)
        n = C.c_int(0)
        rc = self.lib.dustb_cloud_split_p1(self.pctx, C.byref(split), C.c_ulonglong(tag0),
                                           C.byref(n), s.data_ptr(), s.numel(), _stream_ptr(stream))
        if rc == capi.DUSTB_ESCRATCH and self.npart + n.value > self.stride:
            self.ensure_capacity(self.npart + n.value)
            rc = self.lib.dustb_cloud_split_p1(self.pctx, C.byref(split), C.c_ulonglong(tag0),
                                               C.byref(n), s.data_ptr(), s.numel(),
                                               _stream_ptr(stream))
        capi.check(rc, "cloud_split_p1")
        self.npart += int(n.value)
        self._rebuild_ctx()
        return int(n.value)

    def cloud_pc2_cycle(self, dt, stream=None):
        chi = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._call("cloud_pc2_cycle", dt, chi.data_ptr(), self._gpack().data_ptr(),
                   self.t["x3_removed"].data_ptr(), stream=stream)
        return chi

    # ---- point-particle fields (self-gravity, outputs) ----
    def _field(self, nvar):
        return torch.zeros(self.mesh.field_shape(nvar), dtype=torch.float64, device=self.device)

    def point_gravity_density(self, stream=None):
        """DepositPointGravityDensity: the owned TSC density field (ghost cells zero)."""
        owned, halo = self._field(1), self._field(1)
        self._call("point_gravity_density", owned.data_ptr(), halo.data_ptr(), stream=stream)
        return owned

    def point_gravity_gather(self, owned, stream=None, return_field=False):
        """GatherPointGravityAcceleration: the (3, npart) acceleration over owned (nmb, 3, ...)
        (and, with return_field, the force field with its transposed ghost cells)."""
        n = self.npart
        halo = self._field(3)
        acc = torch.empty((3, max(n, 1)), dtype=torch.float64, device=self.device)
        self._call("point_gravity_gather", owned.data_ptr(), halo.data_ptr(), acc.data_ptr(),
                   max(n, 1), stream=stream)
        return (acc[:, :n], halo) if return_field else acc[:, :n]

    def point_science_fields(self, mass_only=False, species=-1, stream=None):
        """DepositPointScienceFields: m/V and m v/V (or m/V alone) on the active cells."""
        nv = 1 if mass_only else 4
        out, halo = self._field(nv), self._field(nv)
        self._call("point_science_fields", out.data_ptr(), halo.data_ptr(), int(mass_only),
                   int(species), stream=stream)
        return out

    # ---- sort ----
    def _scratch(self):
        n = int(self.lib.dustb_sort_scratch_bytes(C.byref(self.ctx.mesh), self.npart))
        s = self.t.get("sort_scratch")
        if s is None or s.numel() < n:
            s = torch.empty(n, dtype=torch.uint8, device=self.device)
            self.t["sort_scratch"] = s
        return s

    def cell_index(self, stream=None):
        ms = self.mesh
        ncell = ms.ncell_active
        order = torch.empty(max(self.npart, 1), dtype=torch.int32, device=self.device)
        cstart = torch.empty(ncell + 1, dtype=torch.int32, device=self.device)
        s = self._scratch()
        rc = self.lib.dustb_cell_index(self.pctx, order.data_ptr(), cstart.data_ptr(),
                                       s.data_ptr(), s.numel(), _stream_ptr(stream))
        capi.check(rc, "cell_index")
        return order[:self.npart], cstart

    def cloud_order(self, stream=None):
        """UpdateCloudOrder's rebuild: the particles in (block, cell, index) order without
        moving them, and the 64-bit tag of each indexed particle (int32, int64 tensors)."""
        n = self.npart
        ord_ = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        tag = torch.empty(max(n, 1), dtype=torch.int64, device=self.device)
        s = self._scratch()
        self._call("cloud_order", ord_.data_ptr(), tag.data_ptr(), s.data_ptr(), s.numel(),
                   stream=stream)
        return ord_[:n], tag[:n]

    def cloud_order_identity(self, stream=None):
        """The index after a sort in cell order: slot k holds particle k."""
        n = self.npart
        ord_ = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        tag = torch.empty(max(n, 1), dtype=torch.int64, device=self.device)
        self._call("cloud_order_identity", ord_.data_ptr(), tag.data_ptr(), stream=stream)
        return ord_[:n], tag[:n]

    def cloud_order_check(self, ord_, tag, stream=None) -> int:
        """The number of index entries whose slot no longer holds the indexed particle."""
        bad = torch.empty(1, dtype=torch.int32, device=self.device)
        self._call("cloud_order_check", ord_.data_ptr(), tag.data_ptr(), int(ord_.numel()),
                   bad.data_ptr(), stream=stream)
        return int(bad.item())

    def sort_by_cell(self, stream=None):
        """SortParticles: sort into spare arrays, then swap them in (as the reference)."""
        s = self._scratch()
        spr = torch.empty_like(self.t["pr"])
        spi = torch.empty_like(self.t["pi"])
        rc = self.lib.dustb_sort_by_cell(self.pctx, spr.data_ptr(), spi.data_ptr(), s.data_ptr(),
                                         s.numel(), _stream_ptr(stream))
        capi.check(rc, "sort_by_cell")
        self.t["pr"], self.t["pi"] = spr, spi
        self._rebuild_ctx()

    # ---- host views ----
    def error_word(self) -> int:
        return int(self.t["err"].item())

    def host(self, name):
        a = self.t[name]
        if name in ("pr", "pi"):
            a = a[:, :self.npart]
        return a.detach().cpu().numpy()

    def momentum(self):
        ms = self.mesh
        u0 = self.t["u0"]
        is_, js, ks = ms.starts
        act = u0[:, 1:4, ks:ks + ms.nx[2], js:js + ms.nx[1], is_:is_ + ms.nx[0]]
        g = act.sum(dim=(0, 2, 3, 4)) * ms.cell_volume()
        pr = self.t["pr"][:, :self.npart]
        m = pr[16]
        d = torch.stack([(m * pr[1]).sum(), (m * pr[3]).sum(), (m * pr[5]).sum()])
        return g.cpu().numpy(), d.cpu().numpy()
