"""Build recipe of the CUDA library athenak_b200/libdustb.so (sm_100a, in-tree).

The .cu files under csrc/ (UNITS) are compiled by nvcc for sm_100a and linked into one shared library
with C linkage entry points (include/dustb.h).  The FP64 translation units are compiled with
--fmad=false so their per-particle arithmetic rounds as the CPU oracle's does.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdustb.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# translation units and their extra flags
UNITS = {
    "dustb_fp64.cu": ["--fmad=false"],
    "dustb_sort.cu": [],
    "dustb_mixed.cu": [],
    "dustb_seed.cu": [],
    "dustb_output.cu": [],
    "dustb_amr.cu": ["--fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "dustb.h"))
    newest = max(os.path.getmtime(p) for p in deps)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xptxas", "-v" if verbose else "-O3", "-rdc=false", "-c", src, "-o", obj, *extra]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {unit}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return OUT


HOST_SRCS = [os.path.join(HERE, "host", f) for f in ("dust_gas_drag.cpp", "pbin.cpp",
                                                      "restart.cpp", "dep_plan.cpp",
                                                      "leaf_tables.cpp")]
HOST_HDRS = [os.path.join(HERE, "host", f) for f in ("dust_gas_drag.hpp", "pbin.hpp",
                                                      "restart.hpp", "dep_plan.hpp",
                                                      "leaf_tables.hpp")]
HOST_LIB = os.path.join(HERE, "libdustb_host.so")


def have_zlib() -> bool:
    """zlib (header and library) for the compressed pbin format (version 3)."""
    return os.path.exists("/usr/include/zlib.h") and any(
        os.path.exists(os.path.join(d, "libz.so"))
        for d in ("/usr/lib/x86_64-linux-gnu", "/usr/lib64", "/usr/lib", "/lib/x86_64-linux-gnu"))


def cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def build_host(force: bool = False) -> str:
    """The C++ host layer (athenak_b200/host: DustGasDrag's task functions over the C ABI)
    as libdustb_host.so, linked against libdustb.so."""
    lib = build(force)
    newest = max(os.path.getmtime(p) for p in (*HOST_SRCS, *HOST_HDRS, lib))
    if not force and os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= newest:
        return HOST_LIB
    cu = cuda_home()
    z = have_zlib()
    zlink = ["-lz"] if z else []
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", HOST_LIB, *HOST_SRCS,
           f"-DATHENAK_B200_HAVE_ZLIB={1 if z else 0}", "-pthread",
           f"-I{cu}/include", f"-L{HERE}", "-ldustb", f"-L{cu}/lib64", "-lcudart", *zlink,
           "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{cu}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("host layer build failed")
    return HOST_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
