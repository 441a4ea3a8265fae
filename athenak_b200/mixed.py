"""Host front end of the mixed-precision form (include/dustb.h, dustb_mixed_*).

A MixedDust owns a DeviceDust (the reference-layout FP64 particle rows and mesh fields) and
the caller-side workspace of the compact particle shadow.  import_() builds the shadow from
the FP64 rows, imex_cycle() advances it (mesh fields in FP64), export() writes it back.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .drag import DeviceDust, GAMMA_DEFAULT, _stream_ptr

KERNELS = ["count", "fill", "deposit_qp", "operator", "kick", "consistent", "cells", "move",
           "window"]


class DustbMixedParams(C.Structure):
    _fields_ = [("dx", C.c_double * 3), ("rows_per_tile", C.c_int), ("chunk", C.c_int),
                ("variant", C.c_int), ("x3_removed", C.c_void_p), ("root_level", C.c_int),
                ("plan", C.c_void_p), ("coarse", C.c_void_p), ("coarse_bytes", C.c_longlong)]


_declared = False


def _declare(lib):
    global _declared
    if _declared:
        return
    P = C.POINTER(capi.DustbCtx)
    MP = C.POINTER(DustbMixedParams)
    VP, LL = C.c_void_p, C.c_longlong
    for name, args in {
        "dustb_mixed_import": [P, MP, VP, LL, VP],
        "dustb_mixed_export": [P, MP, VP, LL, VP],
        "dustb_mixed_sort": [P, MP, VP, LL, VP],
        "dustb_mixed_imex_cycle": [P, MP, VP, LL, C.POINTER(capi.DustbImexCoeffs), VP],
        "dustb_mixed_pc2_cycle": [P, MP, VP, LL, C.c_double, VP, VP],
        "dustb_mixed_tune": [P, MP, VP, LL, C.c_double, VP, VP],
    }.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.dustb_mixed_workspace_bytes.argtypes = [C.POINTER(capi.DustbMesh), C.c_int]
    lib.dustb_mixed_workspace_bytes.restype = LL
    lib.dustb_mixed_timing.argtypes = [C.c_int]
    lib.dustb_mixed_timing.restype = C.c_int
    lib.dustb_mixed_kernel_times.argtypes = [VP, VP, C.c_int]
    lib.dustb_mixed_kernel_times.restype = C.c_int
    _declared = True


class MixedDust:
    """Mixed-precision drag step over a DeviceDust's reference arrays."""

    def __init__(self, st=None, phys=None, dev: DeviceDust | None = None, rows_per_tile=0,
                 chunk=0, do_import=True, variant=0):
        self.dev = dev if dev is not None else DeviceDust(st, phys)
        self.lib = self.dev.lib
        _declare(self.lib)
        ms = self.dev.mesh
        self.mp = DustbMixedParams()
        d = ms.mb_size[0]
        self.mp.dx[0], self.mp.dx[1], self.mp.dx[2] = float(d[6]), float(d[7]), float(d[8])
        self.mp.rows_per_tile = rows_per_tile
        self.mp.chunk = chunk
        self.mp.variant = variant
        self.mp.x3_removed = self.dev.t["x3_removed"].data_ptr()
        if getattr(ms, "nghbr56", None) is not None:
            # a refined mesh: the root level's cell size, the deposit remap set on the device
            # arrays (DeviceDust.set_dep_plan) and the copy exchange's scratch for the gas state
            root = int(ms.root_level)
            lev0 = int(ms.lloc[0, 0])
            for a in range(3):
                self.mp.dx[a] = float(ms.mb_size[0, 6 + a]) * float(2 ** (lev0 - root))
            self.mp.root_level = root
            if getattr(self.dev, "plan", None) is None:
                raise RuntimeError("a refined mesh needs DeviceDust.set_dep_plan first")
            self.mp.plan = C.addressof(self.dev.plan)
            nvg = int(self.dev.t["u0"].shape[1])
            nb = int(self.lib.dustb_ghost_copy_ml_bytes(C.byref(self.dev.ctx.mesh), nvg))
            ca = self.dev.t.get("coarse")
            if ca is None or ca.numel() * 8 < nb:
                ca = self.dev.t["coarse"] = torch.empty(nb // 8, dtype=torch.float64,
                                                        device=self.dev.device)
            self.mp.coarse = ca.data_ptr()
            self.mp.coarse_bytes = nb
        nbytes = int(self.lib.dustb_mixed_workspace_bytes(C.byref(self.dev.ctx.mesh), self.dev.npart))
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=self.dev.device)
        if do_import:
            self.import_()

    def _ws(self):
        return self.ws.data_ptr(), self.ws.numel()

    def import_(self, stream=None):
        p, n = self._ws()
        capi.check(self.lib.dustb_mixed_import(self.dev.pctx, C.byref(self.mp), p, n,
                                               _stream_ptr(stream)), "mixed_import")

    def export(self, stream=None):
        p, n = self._ws()
        capi.check(self.lib.dustb_mixed_export(self.dev.pctx, C.byref(self.mp), p, n,
                                               _stream_ptr(stream)), "mixed_export")

    def sort(self, stream=None):
        p, n = self._ws()
        capi.check(self.lib.dustb_mixed_sort(self.dev.pctx, C.byref(self.mp), p, n,
                                             _stream_ptr(stream)), "mixed_sort")

    def imex_cycle(self, dt, gamma=GAMMA_DEFAULT, sh=(0.0, 0.0), stream=None):
        """One imex2+ cycle; sh: the implicit shear shift of stages 1 and 2 (3-D shearing
        box: the deposit and gather weights sit at y + sh x)."""
        co = capi.DustbImexCoeffs()
        co.gamma, co.dt = gamma, dt
        co.sh[0], co.sh[1] = sh
        p, n = self._ws()
        capi.check(self.lib.dustb_mixed_imex_cycle(self.dev.pctx, C.byref(self.mp), p, n,
                                                   C.byref(co), _stream_ptr(stream)),
                   "mixed_imex_cycle")

    def pc2_cycle(self, dt, stream=None):
        """One pc2 cycle; returns the device scalar chi_max (dt times the largest
        predicted rate over rho)."""
        out = self.dev.t["scalar"]
        p, n = self._ws()
        capi.check(self.lib.dustb_mixed_pc2_cycle(self.dev.pctx, C.byref(self.mp), p, n, dt,
                                                  out.data_ptr(), _stream_ptr(stream)),
                   "mixed_pc2_cycle")
        return out[0]

    def capture(self, cycle):
        """Captures one call of `cycle` (a zero-argument function launching one cycle on
        the current stream, e.g. lambda: mx.imex_cycle(dt)) into a CUDA graph; replay()
        advances the state by one cycle.  Every kernel argument is fixed at capture (the
        shadow, the workspace, the reference arrays and dt), so the graph stays valid while
        none of them is reallocated.  Run one eager cycle of the same shape first (it sets
        the kernels' shared-memory limits, which a capture does not)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            cycle()
        return g

    def tune(self, a_dt, stream=None):
        """The library's autotuner (dustb_mixed_tune): picks rows per tile, particles per pass
        and the launch form on this workspace; returns (rows_per_tile, chunk, grid, ms)."""
        p, n = self._ws()
        ms = C.c_double(0.0)
        capi.check(self.lib.dustb_mixed_tune(self.dev.pctx, C.byref(self.mp), p, n, a_dt,
                                             C.byref(ms), _stream_ptr(stream)), "mixed_tune")
        return (self.mp.rows_per_tile, self.mp.chunk, int(bool(self.mp.variant & 8)), ms.value)

    def set_tiles(self, rows_per_tile=0, chunk=0, variant=None):
        self.mp.rows_per_tile = rows_per_tile
        self.mp.chunk = chunk
        if variant is not None:
            self.mp.variant = variant

    # ---- timing ----
    def timing(self, on: bool):
        self.lib.dustb_mixed_timing(1 if on else 0)

    def kernel_times(self):
        nk = len(KERNELS)
        ms = (C.c_double * nk)()
        n = (C.c_int * nk)()
        self.lib.dustb_mixed_kernel_times(C.cast(ms, C.c_void_p), C.cast(n, C.c_void_p), nk)
        return {KERNELS[k]: (ms[k], n[k]) for k in range(nk)}

    # ---- host views ----
    def export_velocities(self):
        self.export()
        torch.cuda.synchronize()
        pr = self.dev.host("pr")
        return pr[1], pr[3], pr[5]

    def error_word(self):
        return self.dev.error_word()
