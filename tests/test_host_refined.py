"""The C++ host layer on a refined 3-D mesh (tests/host/refined_drag.cpp): DustGasDrag with
SetRefinedMesh (the general deposit remap and the multilevel copy exchange behind RecvDepQP,
RecvUstar, RecvPMBR, RecvU and the dc1 sweeps) and, for refinable clouds, SetLeafTables,
SetCloudSplit and RefineClouds (the P1 split, then the instant switch) at the start of every
cycle.  Its cycles must equal the library's fused forms on the same inputs (which the oracle
pins in tests/test_gpu_amr.py and tests/test_gpu_clouds_refined.py): the point-particle
imex2+/dc1 cycles of dustb_refined_imex_cycle, and the clouds' split, switch and
dustb_cloud_refined_imex_cycle, to 1e-12 of each row's scale, blocks and codes exactly."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from athenak_b200 import capi
from athenak_b200.amr import (build_dep_plan, leaf_tables, refined_mesh, refined_state,
                              sphere_refine)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "host", "_build", "refined_drag")


def build_program() -> str:
    from athenak_b200 import build
    host = build.build_host()
    cu = build.cuda_home()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    pkg = os.path.dirname(host)
    cmd = ["g++", "-std=c++17", "-O2", "-o", EXE, os.path.join(ROOT, "tests", "host", "refined_drag.cpp"),
           f"-I{cu}/include", f"-L{pkg}", "-ldustb_host", "-ldustb", f"-L{cu}/lib64", "-lcudart",
           f"-Wl,-rpath,{pkg}", f"-Wl,-rpath,{cu}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def test_refined_host_program_builds():
    assert os.path.exists(build_program())


def _mesh():
    return refined_mesh((4, 4, 4), (8, 8, 8), 2, refine=sphere_refine((0.1, 0.05, -0.02), (0.3, 0.15)))


def write_case(path, ms, st, plan, lt, phys, dt, gamma, clouds, ncycles, stride, split_max_level=-1,
               next_tag=0):
    """The case file of refined_drag.cpp (its header comment gives the layout)."""
    pr = np.zeros((17, stride))
    pi = np.zeros((5, stride), np.int32)
    pr[:, :st.npart] = st.pr[:, :st.npart]
    pi[:, :st.npart] = st.pi[:, :st.npart]
    h = np.array([ms.nmb, *ms.nx, ms.ng, ms.x3bc, st.npart, stride, st.u0.shape[1], plan.nseg,
                  plan.ent_src.size, lt.nlev, *lt.nfine, phys["scheme"], 1,
                  int(phys.get("consistent_gas", True)), phys["drag_solver"], int(clouds),
                  int(clouds), split_max_level, next_tag, ncycles], np.int64)
    r = np.array([ms.lo[0], ms.hi[0], ms.lo[1], ms.hi[1], ms.lo[2], ms.hi[2], dt, gamma,
                  *lt.root_dx, 0.02], np.float64)
    a = lt.arrays
    with open(path, "wb") as f:
        for x in (h, r, ms.mb_size.astype(np.float64), ms.nghbr.astype(np.int32),
                  ms.lloc[:, 0].astype(np.int32), ms.nghbr56.astype(np.int32), plan.seg_tgt,
                  plan.seg_ptr, plan.ent_src, plan.ent_w, a["fbox"], a["blev"], a["nnb"], a["nb"],
                  a["nbs"], a["nbmax"], a["safe"], a["lockey"], a["locblk"], pr, pi,
                  st.u0.astype(np.float64)):
            np.ascontiguousarray(x).tofile(f)


def read_result(path, u0_shape):
    with open(path, "rb") as f:
        n = int(np.fromfile(f, np.int64, 1)[0])
        pr = np.fromfile(f, np.float64, 17 * n).reshape(17, n)
        pi = np.fromfile(f, np.int32, 5 * n).reshape(5, n)
        u0 = np.fromfile(f, np.float64, int(np.prod(u0_shape))).reshape(u0_shape)
    return pr, pi, u0


def _compare(pr, pi, u0, g):
    import torch
    torch.cuda.synchronize()
    n = g.npart
    assert pr.shape[1] == n
    np.testing.assert_array_equal(pi, g.host("pi")[:, :n])
    b = g.host("pr")
    for r in range(17):
        sc = max(np.abs(b[r, :n]).max(), 1e-300)
        assert np.abs(pr[r] - b[r, :n]).max() <= 1e-12 * sc, r
    ub = g.t["u0"].cpu().numpy()
    for v in range(u0.shape[1]):
        sc = np.abs(ub[:, v]).max()
        assert np.abs(u0[:, v] - ub[:, v]).max() <= 1e-12 * sc, v


@pytest.mark.gpu
@pytest.mark.parametrize("clouds", [False, True])
def test_host_layer_on_a_refined_mesh(clouds):
    from athenak_b200.drag import DeviceDust
    from oracle.oracle import GAMMA_DEFAULT
    exe = build_program()
    ms = _mesh()
    plan = build_dep_plan(ms, 0)
    lt = leaf_tables(ms)
    st = refined_state(ms, [0.02, 0.5], [1.0, 0.5], 1, seed=31, vel_noise=0.3, gas_noise=0.05,
                       vd=[0.5, -0.3])
    st.pi[3, :st.npart] = lt.arrays["blev"][st.pi[0, :st.npart]]   # clouds at their leaf's level
    phys = dict(scheme=2, drag_solver=2, consistent_gas=True)
    dt = 0.2 * ms.mb_size[:, 6].min() / np.abs(st.pr[[1, 3, 5], :st.npart]).max()
    ncyc = 2
    stride = st.npart * 6
    with tempfile.TemporaryDirectory() as tmp:
        case, res = os.path.join(tmp, "case.bin"), os.path.join(tmp, "result.bin")
        write_case(case, ms, st, plan, lt, phys, dt, GAMMA_DEFAULT, clouds, ncyc, stride,
                   split_max_level=1 if clouds else -1, next_tag=st.npart)
        r = subprocess.run([exe, case, res], capture_output=True, text=True, timeout=600)
        print(r.stdout)
        assert r.returncode == 0, r.stdout + r.stderr
        pr, pi, u0 = read_result(res, st.u0.shape)
    g = DeviceDust(st, phys, stride=stride)
    g.set_dep_plan(plan)
    if clouds:
        g.set_leaf_tables(lt)
        sp = capi.split_params(max_level=1)       # cloud_split_max_level = 1
        tag = st.npart
    for _ in range(ncyc):
        if clouds:
            tag += g.cloud_split_p1(sp, tag)
            g.cloud_instant_switch(1)
            g.cloud_refined_imex_cycle(dt)
        else:
            g.refined_imex_cycle(dt)
    if clouds:
        assert g.npart > st.npart
    _compare(pr, pi, u0, g)
