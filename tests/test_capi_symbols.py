"""The C-ABI library loads without a GPU and exports every function include/dustb.h
declares; the host-side argument checks reject bad contexts before any CUDA call."""
import ctypes as C
import os
import re

import pytest

from athenak_b200 import capi
from athenak_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^(?:int|long long|const char \*)\s*(dustb_[a-z0-9_]+)\s*\(",
                                    src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    build()
    lib = C.CDLL(capi.LIB_PATH)
    names = declared()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    names = declared()
    covered = set(capi.SIGNATURES) | {"dustb_last_error"} | set(getattr(capi, "EXTRA_SIGNATURES", {}))
    assert names <= covered, sorted(names - covered)


def test_invalid_context_is_rejected_on_the_host():
    lib = capi.load()
    ctx = capi.DustbCtx()          # all zero: no mesh
    assert lib.dustb_push_imex(C.byref(ctx), 1.0, 0.0, 0.1, 0.0, None) == -1
    assert lib.dustb_deposit_qp(C.byref(ctx), 0.1, 0.0, None) == -1
    assert lib.dustb_version() >= 1


def test_detached_rows_are_rejected_where_rows_are_read():
    """A context with its particle rows detached (pr = pi = NULL, npart kept) passes only where
    no row is read: the mixed import and export refuse it on the host, before any CUDA call."""
    from athenak_b200.mesh import uniform_mesh
    from athenak_b200.mixed import DustbMixedParams, _declare
    lib = capi.load()
    _declare(lib)
    import numpy as np
    ms = uniform_mesh((8, 8, 8), (8, 8, 8), 2, (0.0,) * 3, (1.0,) * 3)
    arrays = {k: np.zeros(ms.field_shape(5)) for k in ("u0", "u1", "qdep", "ustar", "dmom",
                                                       "resid", "work")}
    arrays.update(mb_size=np.ascontiguousarray(ms.mb_size), nghbr=np.ascontiguousarray(ms.nghbr),
                  sb_gid=None, pr=None, pi=None, err=np.zeros(1, np.int32))
    ctx = capi.make_ctx(ms, arrays, 100, 100, {})
    mp = DustbMixedParams()
    mp.dx[0] = mp.dx[1] = mp.dx[2] = 1.0 / 8
    ws = np.zeros(16, np.uint8)
    for fn in (lib.dustb_mixed_import, lib.dustb_mixed_export):
        assert fn(C.byref(ctx), C.byref(mp), ws.ctypes.data, ws.size, None) == -1
    # the FP64 particle tasks refuse it as well
    assert lib.dustb_push_imex(C.byref(ctx), 1.0, 0.0, 0.1, 0.0, None) == -1
