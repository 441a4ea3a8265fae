"""ctypes mirror of include/dustb.h: the structs, the constants and the loader of the CUDA
library (athenak_b200/libdustb.so).  The library is required: there is no CPU path."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdustb.so")

DUSTB_NGP, DUSTB_CIC, DUSTB_TSC = 0, 1, 2
DUSTB_ESCRATCH = -3
SOLVER_LOCAL, SOLVER_APPLYA, SOLVER_DC1, SOLVER_DC2 = 0, 1, 2, 3
X3_PERIODIC, X3_REFLECT, X3_OUTFLOW = 0, 1, 2
ERR_HALO, ERR_ROUTE, ERR_NGHBR, ERR_PGID, ERR_TSTOP, ERR_WINDOW = 1, 2, 4, 8, 16, 32
ERR_TIMEOUT, ERR_POINT, ERR_CLOUD = 64, 128, 256


class DustbMesh(C.Structure):
    _fields_ = [("nmb", C.c_int), ("gids", C.c_int), ("nx1", C.c_int), ("nx2", C.c_int),
                ("nx3", C.c_int), ("ng", C.c_int), ("multi_d", C.c_int), ("three_d", C.c_int),
                ("x3bc", C.c_int),
                ("x1min", C.c_double), ("x1max", C.c_double), ("x2min", C.c_double),
                ("x2max", C.c_double), ("x3min", C.c_double), ("x3max", C.c_double),
                ("mb_size", C.c_void_p), ("nghbr", C.c_void_p),
                ("shear_x1", C.c_int), ("sb_nb2", C.c_int), ("sb_nb3", C.c_int),
                ("sb_gid", C.c_void_p), ("time", C.c_double),
                ("mb_lev", C.c_void_p), ("nghbr_ml", C.c_void_p), ("leaf", C.c_void_p)]


LEAF_MAXNB = 64


class DustbLeafTables(C.Structure):
    _fields_ = [("nlev", C.c_int), ("nfine", C.c_int * 3), ("root_dx", C.c_double * 3),
                ("fbox", C.c_void_p), ("blev", C.c_void_p), ("nnb", C.c_void_p),
                ("nb", C.c_void_p), ("nbs", C.c_void_p), ("nbmax", C.c_void_p),
                ("safe", C.c_void_p), ("lockey", C.c_void_p), ("locblk", C.c_void_p),
                ("coarse", C.c_void_p), ("coarse_bytes", C.c_longlong)]


class DustbCloudSplit(C.Structure):
    _fields_ = [("max_level", C.c_int), ("split_everywhere", C.c_int),
                ("split_overlap", C.c_int), ("split_buffer", C.c_int), ("slack", C.c_double),
                ("budget", C.c_longlong)]


def split_params(max_level, everywhere=False, overlap=True, buffer=0, slack=0.02,
                 budget=0) -> DustbCloudSplit:
    """The split's controls (<dust>/cloud_split_*; slack: cloud_split_slack, 0.02; budget:
    cloud_split_budget, 0 for none)."""
    sp = DustbCloudSplit()
    sp.max_level, sp.split_everywhere = int(max_level), int(everywhere)
    sp.split_overlap, sp.split_buffer, sp.slack = int(overlap), int(buffer), float(slack)
    sp.budget = int(budget)
    return sp


def leaf_tables_struct(tabs: dict, nlev: int, nfine, root_dx) -> DustbLeafTables:
    """A DustbLeafTables over the arrays of tabs (numpy for the oracle, torch CUDA tensors for
    the library; the keys of athenak_b200.amr.leaf_tables)."""
    t = DustbLeafTables()
    t.nlev = int(nlev)
    for a in range(3):
        t.nfine[a] = int(nfine[a])
        t.root_dx[a] = float(root_dx[a])
    for k in ("fbox", "blev", "nnb", "nb", "nbs", "nbmax", "safe", "lockey", "locblk"):
        setattr(t, k, ptr(tabs[k]))
    if tabs.get("coarse") is not None:
        t.coarse = ptr(tabs["coarse"])
        t.coarse_bytes = int(tabs["coarse"].numel() * 8) if hasattr(tabs["coarse"], "numel") \
            else int(tabs["coarse"].nbytes)
    return t


class DustbParticles(C.Structure):
    _fields_ = [("pr", C.c_void_p), ("pi", C.c_void_p), ("stride", C.c_longlong),
                ("npart", C.c_int)]


class DustbFields(C.Structure):
    _fields_ = [("u0", C.c_void_p), ("u1", C.c_void_p), ("nvar_gas", C.c_int),
                ("qdep", C.c_void_p), ("ustar", C.c_void_p), ("dmom", C.c_void_p),
                ("resid", C.c_void_p), ("work", C.c_void_p)]


class DustbPhysics(C.Structure):
    _fields_ = [("scheme", C.c_int), ("back_reaction", C.c_int), ("consistent_gas", C.c_int),
                ("drag_solver", C.c_int), ("shearing_box", C.c_int), ("stratified", C.c_int),
                ("pc2_feedback_damping", C.c_int),
                ("qshear", C.c_double), ("omega0", C.c_double), ("const_accel_phi", C.c_double),
                ("x3_deposit_drop", C.c_int)]


class DustbDepPlan(C.Structure):
    _fields_ = [("nseg", C.c_int), ("seg_tgt", C.c_void_p), ("seg_ptr", C.c_void_p),
                ("ent_src", C.c_void_p), ("ent_w", C.c_void_p)]


class DustbCtx(C.Structure):
    _fields_ = [("mesh", DustbMesh), ("part", DustbParticles), ("f", DustbFields),
                ("phys", DustbPhysics), ("err", C.c_void_p)]


class DustbSeedDesc(C.Structure):
    _fields_ = [("seed", C.c_ulonglong), ("nspecies", C.c_int), ("ppc", C.c_int * 8),
                ("taus", C.c_double * 8), ("mass", C.c_double * 8), ("vx", C.c_double * 8),
                ("vy", C.c_double * 8), ("vz", C.c_double * 8), ("vel_noise", C.c_double),
                ("rho0", C.c_double), ("ug", C.c_double * 3), ("gas_noise", C.c_double),
                ("nb1", C.c_int), ("nb2", C.c_int), ("nb3", C.c_int),
                ("ts_lo", C.c_double), ("ts_hi", C.c_double), ("mass_slope", C.c_double),
                ("hp", C.c_double), ("nsh", C.c_int), ("omega0", C.c_double),
                ("qshear", C.c_double)]


class DustbImexCoeffs(C.Structure):
    _fields_ = [("gamma", C.c_double), ("dt", C.c_double), ("sh", C.c_double * 2)]


def ptr(a) -> int:
    """Raw address of a numpy array or a torch tensor (None -> NULL)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def make_ctx(mesh, arrays, npart, stride, phys) -> DustbCtx:
    """arrays: dict with pr, pi, u0, u1, qdep, ustar, dmom, resid, work, mb_size, nghbr,
    err (numpy for the oracle, torch CUDA tensors for the library).  phys: dict of the
    DustbPhysics fields."""
    c = DustbCtx()
    m = c.mesh
    m.nmb, m.gids = mesh.nmb, mesh.gids
    m.nx1, m.nx2, m.nx3 = mesh.nx
    m.ng = mesh.ng
    m.multi_d, m.three_d = int(mesh.multi_d), int(mesh.three_d)
    m.x3bc = mesh.x3bc
    m.x1min, m.x2min, m.x3min = mesh.lo
    m.x1max, m.x2max, m.x3max = mesh.hi
    m.mb_size = ptr(arrays["mb_size"])
    m.nghbr = ptr(arrays["nghbr"])
    m.shear_x1 = int(mesh.shear_x1)
    m.sb_nb2, m.sb_nb3 = mesh.nblocks[1], mesh.nblocks[2]
    m.sb_gid = ptr(arrays["sb_gid"]) if mesh.shear_x1 else None
    m.time = 0.0
    # refined meshes: the block levels and the 56 neighbour slots
    if arrays.get("nghbr_ml") is not None:
        m.mb_lev = ptr(arrays["mb_lev"])
        m.nghbr_ml = ptr(arrays["nghbr_ml"])
    c.part.pr, c.part.pi = ptr(arrays["pr"]), ptr(arrays["pi"])
    c.part.stride, c.part.npart = int(stride), int(npart)
    f = c.f
    f.u0, f.u1 = ptr(arrays["u0"]), ptr(arrays["u1"])
    f.nvar_gas = 4
    f.qdep, f.ustar, f.dmom = ptr(arrays["qdep"]), ptr(arrays["ustar"]), ptr(arrays["dmom"])
    f.resid, f.work = ptr(arrays["resid"]), ptr(arrays["work"])
    p = c.phys
    p.scheme = phys.get("scheme", DUSTB_TSC)
    p.back_reaction = int(phys.get("back_reaction", True))
    p.consistent_gas = int(phys.get("consistent_gas", True))
    p.drag_solver = phys.get("drag_solver", SOLVER_DC1)
    p.shearing_box = int(phys.get("shearing_box", False))
    p.stratified = int(phys.get("stratified", False))
    p.pc2_feedback_damping = int(phys.get("pc2_feedback_damping", True))
    p.qshear = phys.get("qshear", 1.5)
    p.omega0 = phys.get("omega0", 1.0)
    p.const_accel_phi = phys.get("const_accel_phi", 0.0)
    p.x3_deposit_drop = int(phys.get("x3_deposit_drop", False))
    c.err = ptr(arrays.get("err"))
    return c


_lib = None


def load() -> C.CDLL:
    """The CUDA library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run athenak_b200.build.build()")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


VP, D, I, LL = C.c_void_p, C.c_double, C.c_int, C.c_longlong
CTXP = C.POINTER(DustbCtx)
MESHP = C.POINTER(DustbMesh)

# name -> argtypes (restype int unless noted); the exported symbols of include/dustb.h
SIGNATURES = {
    "dustb_version": [],
    "dustb_register_copy": [CTXP, VP],
    "dustb_gas_rk_noflux": [CTXP, D, D, VP],
    "dustb_history_gas": [CTXP, D, VP],
    "dustb_push_imex": [CTXP, D, D, D, D, VP],
    "dustb_route": [CTXP, VP, VP],
    "dustb_deposit_qp": [CTXP, D, D, VP],
    "dustb_ghost_add": [CTXP, VP, I, VP],
    "dustb_ghost_copy": [CTXP, VP, I, I, VP],
    "dustb_ghost_add_plan": [CTXP, C.POINTER(DustbDepPlan), VP, I, VP],
    "dustb_ghost_copy_ml_bytes": [MESHP, I],
    "dustb_ghost_copy_ml": [CTXP, VP, I, VP, LL, VP],
    "dustb_solve_ustar": [CTXP, VP],
    "dustb_dc1_sweep": [CTXP, D, D, VP],
    "dustb_gather_kick_pmbr": [CTXP, D, D, VP],
    "dustb_apply_pmbr": [CTXP, D, VP],
    "dustb_newdt": [CTXP, D, VP, VP],
    "dustb_tstop_extrema": [CTXP, VP, VP],
    "dustb_sort_scratch_bytes": [MESHP, I],
    "dustb_cell_index": [CTXP, VP, VP, VP, LL, VP],
    "dustb_sort_by_cell": [CTXP, VP, VP, VP, LL, VP],
    "dustb_pc2_predictor": [CTXP, D, I, VP],
    "dustb_pc2_apply_predictor": [CTXP, D, VP, VP],
    "dustb_pc2_midpoint": [CTXP, VP],
    "dustb_pc2_advance": [CTXP, D, VP],
    "dustb_pc2_commit": [CTXP, D, VP],
    "dustb_imex_cycle": [CTXP, C.POINTER(DustbImexCoeffs), VP, VP],
    "dustb_dc1_sweep_plan": [CTXP, C.POINTER(DustbDepPlan), D, VP, LL, VP],
    "dustb_refined_imex_cycle": [CTXP, C.POINTER(DustbDepPlan), C.POINTER(DustbImexCoeffs), VP,
                                 LL, VP, VP],
    "dustb_pc2_cycle": [CTXP, D, VP, VP, VP],
    "dustb_seed_uniform": [CTXP, C.POINTER(DustbSeedDesc), VP],
    "dustb_cell_index_static": [CTXP, VP, VP, VP],
    "dustb_cell_index_static_reset": [],
    "dustb_phst_scratch_bytes": [MESHP, I],
    "dustb_phst": [CTXP, VP, VP, VP, LL, VP],
    "dustb_cloud_order": [CTXP, VP, VP, VP, LL, VP],
    "dustb_cloud_order_identity": [CTXP, VP, VP, VP],
    "dustb_cloud_order_check": [CTXP, VP, VP, I, VP, VP],
    "dustb_point_gravity_density": [CTXP, VP, VP, VP],
    "dustb_point_gravity_gather": [CTXP, VP, VP, VP, LL, VP],
    "dustb_point_science_fields": [CTXP, VP, VP, I, I, VP],
    "dustb_cloud_deposit_qp": [CTXP, D, D, VP],
    "dustb_cloud_gpack_bytes": [MESHP],
    "dustb_cloud_gather_kick": [CTXP, D, D, VP, VP],
    "dustb_cloud_dc1_sweep": [CTXP, D, D, VP, VP],
    "dustb_cloud_apply_pmbr": [CTXP, D, D, VP],
    "dustb_cloud_imex_cycle": [CTXP, C.POINTER(DustbImexCoeffs), VP, VP, VP],
    "dustb_cloud_refined_imex_cycle": [CTXP, C.POINTER(DustbImexCoeffs), VP, VP, LL, VP, VP],
    "dustb_cloud_instant_switch": [CTXP, I, C.POINTER(C.c_int), VP, VP],
    "dustb_cloud_split_scratch_bytes": [I],
    "dustb_cloud_split_p1": [CTXP, C.POINTER(DustbCloudSplit), C.c_ulonglong,
                             C.POINTER(C.c_int), VP, LL, VP],
    "dustb_cloud_pc2_predictor": [CTXP, D, I, VP, VP],
    "dustb_cloud_pc2_advance": [CTXP, D, VP, VP],
    "dustb_cloud_pc2_cycle": [CTXP, D, VP, VP, VP, VP],
    "dustb_pbin_scratch_bytes": [I],
    "dustb_pbin_rows": [CTXP, VP, VP, D, VP, LL, VP],
    "dustb_pbin_pack": [CTXP, VP, I, I, I, VP, VP],
    "dustb_pbin_shuffle": [VP, LL, I, LL, VP, VP],
}
RESTYPES = {"dustb_sort_scratch_bytes": LL, "dustb_ghost_copy_ml_bytes": LL, "dustb_phst_scratch_bytes": LL,
            "dustb_pbin_scratch_bytes": LL, "dustb_cloud_gpack_bytes": LL,
            "dustb_cloud_split_scratch_bytes": LL,
            "dustb_last_error": C.c_char_p}
# declared by athenak_b200.mixed (they take its DustbMixedParams struct)
EXTRA_SIGNATURES = {"dustb_mixed_workspace_bytes", "dustb_mixed_import", "dustb_mixed_export",
                    "dustb_mixed_imex_cycle", "dustb_mixed_sort", "dustb_mixed_timing",
                    "dustb_mixed_kernel_times", "dustb_mixed_pc2_cycle", "dustb_mixed_tune"}


def _declare(lib):
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, C.c_int)
    lib.dustb_last_error.argtypes = []
    lib.dustb_last_error.restype = C.c_char_p


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = load().dustb_last_error()
        raise RuntimeError(f"{what} failed with status {rc}: {msg.decode() if msg else ''}")
