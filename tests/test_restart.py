"""The particle section of the restart file ("AKPRST01", src/dust/dust_restart.cpp) from the
C++ host layer (athenak_b200/host/restart.hpp).  The tool's own checks: a section written and
parsed back (rows and records bit for bit), a version-1 section parsed (high tag words 0, the
int32 counter), damaged sections rejected; and a reader of the layout written from its
description here: the head (version 2, 8-byte reals, 4-byte ints, 1 rank, 17 + 5 columns,
the total size), the records in the reference's order and sizes, the rows of the live
particles only (the capacity tail left out), the end marker.  The device round trip (rows
copied off the GPU, restored into arrays of another capacity) is a GPU test."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "host", "_build", "restart_tool")

ORDER = ["tag_state", "rank_blocks", "merge_pass", "species_table", "resample", "resample_clk",
         "merge_clk", "split", "coarsen_n", "amr_regrids", "regrid_evt", "regrid_evt_t",
         "x3_ledger", "cloud_ord_n", "cloud_ord", "cloud_ord_tag"]
SIZES = {"tag_state": 24, "rank_blocks": 12, "merge_pass": 4, "resample": 16,
         "resample_clk": 48, "merge_clk": 40, "split": 32, "coarsen_n": 32, "amr_regrids": 4,
         "regrid_evt": 48, "regrid_evt_t": 16, "cloud_ord_n": 12}


def build_tool() -> str:
    from athenak_b200 import build
    host = build.build_host()
    cu = build.cuda_home()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    pkg = os.path.dirname(host)
    cmd = ["g++", "-std=c++17", "-O2", "-o", EXE, os.path.join(ROOT, "tests", "host", "restart_tool.cpp"),
           f"-I{cu}/include", f"-L{pkg}", "-ldustb_host", "-ldustb", f"-L{cu}/lib64", "-lcudart",
           f"-Wl,-rpath,{pkg}", f"-Wl,-rpath,{cu}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def read_section(raw):
    assert raw[:8] == b"AKPRST01" and raw[-8:] == b"AKPRST01"
    head = np.frombuffer(raw[8:32], "<i4")
    total = int(np.frombuffer(raw[32:40], "<u8")[0])
    np_ = int(np.frombuffer(raw[40:48], "<i8")[0])
    dtnew = float(np.frombuffer(raw[48:56], "<f8")[0])
    nstate = int(np.frombuffer(raw[56:60], "<i4")[0])
    assert total == len(raw)
    recs, at, end = [], 60, 60 + nstate
    while at < end:
        name = raw[at:at + 16].rstrip(b"\0").decode()
        n = int(np.frombuffer(raw[at + 16:at + 20], "<i4")[0])
        recs.append((name, raw[at + 20:at + 20 + n]))
        at += 20 + n
    assert at == end
    nr, ni = int(head[4]), int(head[5])
    pr = np.frombuffer(raw[end:end + 8 * nr * np_], "<f8").reshape(nr, np_)
    pi = np.frombuffer(raw[end + 8 * nr * np_:len(raw) - 8], "<i4").reshape(ni, np_)
    return head, np_, dtnew, recs, pr, pi


def test_host_sections(tmp_path):
    exe = build_tool()
    r = subprocess.run([exe, "host", str(tmp_path)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 10
    head, n, dtnew, recs, pr, pi = read_section((tmp_path / "host.rst").read_bytes())
    assert list(head) == [2, 8, 4, 1, 17, 5] and dtnew == 0.125
    assert [name for name, _ in recs] == ORDER
    for name, data in recs:
        if name in SIZES:
            assert len(data) == SIZES[name], name
    rec = dict(recs)
    assert list(np.frombuffer(rec["tag_state"], "<u8")) == [1, 123456789012, 123456789999]
    led = np.frombuffer(rec["x3_ledger"], "<f8")
    assert led[4] == 4 and len(led) == 9 and list(led[:4]) == [0.25, 12, 0.01, 2]
    assert list(np.frombuffer(rec["cloud_ord_n"], "<i4")) == [1, 3, 40]
    assert rec["species_table"].decode().startswith("nspecies = 3")
    raw = (tmp_path / "host.rows").read_bytes()
    cnt, stride = np.frombuffer(raw[:16], "<i8")
    rpr = np.frombuffer(raw[16:16 + 8 * 17 * stride], "<f8").reshape(17, stride)
    rpi = np.frombuffer(raw[16 + 8 * 17 * stride:], "<i4").reshape(5, stride)
    assert n == cnt
    np.testing.assert_array_equal(pr, rpr[:, :n])
    np.testing.assert_array_equal(pi, rpi[:, :n])


def test_rank_sections(tmp_path):
    """A run on several ranks appends one section per rank in rank order (src/dust/
    dust_restart.cpp): the tool's checks (split, exact own sections, other block layouts
    gathered from every section, damaged files rejected), and the file read here: two
    sections, each with ranks written = 2 in its head and its own rank_blocks record."""
    exe = build_tool()
    r = subprocess.run([exe, "ranks", str(tmp_path)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 10
    raw = (tmp_path / "ranks.rst").read_bytes()
    total0 = int(np.frombuffer(raw[32:40], "<u8")[0])
    blocks = []
    for sec, n in ((raw[:total0], 10), (raw[total0:], 7)):
        head, np_, dtnew, recs, pr, pi = read_section(sec)
        assert list(head) == [2, 8, 4, 2, 17, 5] and np_ == n
        blocks.append(list(np.frombuffer(dict(recs)["rank_blocks"], "<i4")))
        lo, nb = blocks[-1][1], blocks[-1][2]
        assert np.all((pi[0] >= lo) & (pi[0] < lo + nb))
    assert blocks == [[0, 0, 4], [1, 4, 4]]


@pytest.mark.gpu
def test_device_round_trip(tmp_path):
    exe = build_tool()
    r = subprocess.run([exe, "device", str(tmp_path)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(": ok") == 4
