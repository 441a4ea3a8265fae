"""The C++ host layer (athenak_b200/host: DustGasDrag's task functions over the C ABI): it
builds, and its parity program (tests/host/drag_parity.cpp, which drives the task list of
imex2+ and pc2 cycles on the GPU and the CPU oracle on the same seeded inputs) agrees."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "host", "_build", "drag_parity")


def build_parity_program() -> str:
    from athenak_b200 import build
    from oracle import oracle
    host = build.build_host()
    oracle.build()
    cu = build.cuda_home()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    pkg, orc = os.path.dirname(host), os.path.join(ROOT, "oracle")
    cmd = ["g++", "-std=c++17", "-O2", "-o", EXE, os.path.join(ROOT, "tests", "host", "drag_parity.cpp"),
           f"-I{cu}/include", f"-L{pkg}", "-ldustb_host", "-ldustb", f"-L{orc}", "-loracle_dust",
           f"-L{cu}/lib64", "-lcudart", f"-Wl,-rpath,{pkg}", f"-Wl,-rpath,{orc}",
           f"-Wl,-rpath,{cu}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def test_host_layer_and_parity_program_build():
    assert os.path.exists(build_parity_program())


@pytest.mark.gpu
def test_host_task_list_matches_oracle():
    exe = build_parity_program()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 7
