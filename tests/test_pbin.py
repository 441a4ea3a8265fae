"""The particle science file (pbin, src/outputs/pbin.cpp) written by the C++ host layer
(athenak_b200/host/pbin.hpp): a reader of the format written from its description here checks
the preamble, the footer and the file size, the column directory, the 64-byte alignment, the
constants and every column against the rows the file was written from (active rows only, in
array order; tags from both words; float32 columns rounded from the float64 rows), for format
version 2 and the compressed version 3 (byte shuffle per chunk, one zlib stream per chunk).
The files written from host rows must be byte-identical to the golden files' digests
(tests/golden/pbin_golden.json, recorded after the reference's own reader parsed them).  The
device path (the active rows found and the columns packed and shuffled on the GPU) is a GPU
test."""
import hashlib
import json
import os
import subprocess
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "host", "_build", "pbin_tool")
GOLDEN = os.path.join(ROOT, "tests", "golden", "pbin_golden.json")


def build_tool() -> str:
    from athenak_b200 import build
    host = build.build_host()
    cu = build.cuda_home()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    pkg = os.path.dirname(host)
    cmd = ["g++", "-std=c++17", "-O2", "-o", EXE, os.path.join(ROOT, "tests", "host", "pbin_tool.cpp"),
           f"-I{cu}/include", f"-L{pkg}", "-ldustb_host", "-ldustb", f"-L{cu}/lib64", "-lcudart",
           f"-Wl,-rpath,{pkg}", f"-Wl,-rpath,{cu}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def read_pbin(path):
    """(preamble, sections, columns {name: array}, blocks {name: array}, constants)."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"AKPBIN01"
    assert int.from_bytes(raw[8:12], "little") == 0x01020304
    version = int.from_bytes(raw[12:16], "little")
    text_bytes, data_start, data_bytes, n_part, n_blocks, zero = np.frombuffer(raw[16:64], "<u8")
    assert zero == 0 and data_start % 64 == 0 and data_start >= 64 + text_bytes
    assert raw[data_start + data_bytes:data_start + data_bytes + 8] == b"AKPBEND1"
    assert int(np.frombuffer(raw[data_start + data_bytes + 8:], "<u8")[0]) == len(raw)
    assert raw[64 + text_bytes:data_start] == b"\0" * (data_start - 64 - text_bytes)
    text = raw[64:64 + text_bytes].decode()
    head, sep, dump = text.partition("\n[input]\n")
    assert sep
    sections, cols, consts, chunks, cur = {}, [], {}, [], None
    for line in head.split("\n")[1:]:
        if not line.strip() or line.startswith("#"):
            continue
        if line.startswith("["):
            cur = line.strip()[1:-1]
            sections.setdefault(cur, {})
            continue
        key, value = (x.strip() for x in line.split("=", 1))
        if cur == "columns" and key == "column":
            cols.append(value.split())
        elif cur == "constants" and key == "constant":
            t = value.split()
            consts[t[1]] = np.array([t[3]]).astype(np.float64 if "f" in t[2] else np.uint64)[0]
        elif cur == "chunks" and key == "chunk":
            chunks.append(value.split())
        else:
            sections[cur][key] = value.split("  #")[0].strip()
    out, blocks = {}, {}
    for t in cols:
        table, name, dtype, count, offset, nbytes = t[:6]
        count, offset, nbytes = int(count), int(offset), int(nbytes)
        assert offset % 64 == 0 and offset + nbytes <= data_bytes
        region = raw[data_start + offset:data_start + offset + nbytes]
        enc = t[6] if len(t) > 6 else "raw"
        size = np.dtype(dtype).itemsize
        if enc == "raw":
            assert nbytes == count * size
            arr = np.frombuffer(region, dtype)
        else:
            assert version == 3
            mine = [c for c in chunks if c[0] == name]
            parts, row, at = [], 0, offset
            for c in mine:
                first, rows, off, sb = int(c[2]), int(c[3]), int(c[4]), int(c[5])
                assert first == row and off == at
                if rows:
                    data = zlib.decompress(raw[data_start + off:data_start + off + sb])
                    sh = np.frombuffer(data, np.uint8).reshape(size, rows)
                    parts.append(sh.T.copy().reshape(-1))
                else:
                    assert sb == 0
                row += rows
                at += sb
            assert row == count and at == offset + nbytes
            arr = (np.concatenate(parts) if parts else np.zeros(0, np.uint8)).view(dtype)
        (out if table == "particles" else blocks)[name] = arr
    pre = dict(version=version, n_particles=int(n_part), n_blocks=int(n_blocks))
    return pre, sections, out, blocks, consts, dump


def read_rows(path):
    raw = open(path, "rb").read()
    n, stride = np.frombuffer(raw[:16], "<i8")
    pr = np.frombuffer(raw[16:16 + 8 * 17 * stride], "<f8").reshape(17, stride)[:, :n]
    pi = np.frombuffer(raw[16 + 8 * 17 * stride:], "<i4").reshape(5, stride)[:, :n]
    return pr, pi


def check_file(pbin, rows, n_species=None):
    pre, sec, cols, blocks, consts, dump = read_pbin(pbin)
    pr, pi = read_rows(rows)
    act = pr[16] != 0.0
    n = int(act.sum())
    assert pre["n_particles"] == n and len(cols["id"]) == n
    assert int(sec["particles"]["zero_mass_rows_excluded"]) == int((~act).sum())
    tag = (pi[4].astype(np.int64).astype(np.uint64) << np.uint64(32)) | \
        (pi[1].astype(np.int64) & 0xFFFFFFFF).astype(np.uint64)
    np.testing.assert_array_equal(cols["id"], tag[act])
    single = sec["particles"]["particle_real_precision"] == "single"
    for name, r in (("x1", 0), ("x2", 2), ("x3", 4), ("v1", 1), ("v2", 3), ("v3", 5),
                    ("mass", 16), ("stopping_time", 15)):
        if name in cols:
            np.testing.assert_array_equal(cols[name], pr[r, act].astype(np.float32 if single else np.float64))
        else:   # the header constants stay float64
            assert name in consts and np.all(pr[r, act] == consts[name])
    if "species" in cols:
        np.testing.assert_array_equal(cols["species"], pi[2, act].astype(np.uint32))
    else:
        assert consts["species"] == 0 and np.all(pi[2, act] == 0)
    assert pre["n_blocks"] == len(blocks["gid"])
    np.testing.assert_array_equal(blocks["gid"], np.arange(pre["n_blocks"]))
    # the block topology hash (FNV-1a 64 from the format's start value)
    h = 1469598103934665603
    arr = np.stack([blocks["level"].astype(np.int64), blocks["lx1"], blocks["lx2"],
                    blocks["lx3"]], axis=1).astype("<i8").tobytes()
    for b in arr:
        h = ((h ^ b) * 1099511628211) & ((1 << 64) - 1)
    assert sec["snapshot"]["block_topology_hash"] == f"0x{h:016x}"
    assert dump.rstrip().endswith("<par_end>")
    return pre, sec


def test_host_written_files(tmp_path):
    exe = build_tool()
    r = subprocess.run([exe, "host", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    golden = json.load(open(GOLDEN))
    for name in golden["files"]:
        pbin = tmp_path / f"{name}.pbin"
        pre, sec = check_file(str(pbin), str(tmp_path / f"{name}.rows"))
        assert pre["version"] == golden["files"][name]["version"]
        digest = hashlib.sha256(pbin.read_bytes()).hexdigest()
        assert digest == golden["files"][name]["sha256"], name
    # the constants: one species with species_fixed t_s and equal masses
    _, sec, cols, _, consts, _ = read_pbin(str(tmp_path / "one_species_constants.pbin"))
    assert sec["particles"]["constant_columns"] == "species stopping_time mass"
    assert "species" not in cols and "mass" not in cols
    _, sec, cols, _, _, _ = read_pbin(str(tmp_path / "two_species.pbin"))
    assert sec["particles"]["constant_columns"] == "none"
    assert sec["frame"]["velocity_frame"] == "shear_relative"


@pytest.mark.gpu
def test_device_written_files(tmp_path):
    exe = build_tool()
    r = subprocess.run([exe, "device", str(tmp_path)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    for name in ("device_v2", "device_v2_single", "device_v3"):
        pre, sec = check_file(str(tmp_path / f"{name}.pbin"), str(tmp_path / f"{name}.rows"))
        assert pre["version"] == (3 if name == "device_v3" else 2)
        assert int(sec["particles"]["zero_mass_rows_excluded"]) > 0


@pytest.mark.gpu
def test_device_rows_pack_and_shuffle_through_the_c_abi():
    """dustb_pbin_rows / _pack / _shuffle against numpy on the same rows: the active rows in
    array order across many tiles, the counts and the mass range, every column, the shuffle."""
    import ctypes as C
    import torch
    from athenak_b200 import capi
    from athenak_b200.drag import DeviceDust
    from athenak_b200.inputs import make_state
    from athenak_b200.mesh import uniform_mesh
    ms = uniform_mesh((32, 32, 32), (16, 16, 16), 2, (-0.5,) * 3, (0.5,) * 3)
    st = make_state(ms, [0.1, 0.3], [1.0, 0.5], 2, seed=12, vel_noise=0.05)
    n = st.npart
    rng = np.random.default_rng(4)
    st.pr[16, :n][rng.random(n) < 0.2] = 0.0          # massless rows, left out
    st.pr[16, 5] = -1.0                               # an invalid mass (written, counted)
    st.pi[4, :n:9] = -3                               # tags >= 2^63
    g = DeviceDust(st, {})
    lib = capi.load()
    s = torch.empty(int(lib.dustb_pbin_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    stats = torch.zeros(7, dtype=torch.float64, device="cuda")
    capi.check(lib.dustb_pbin_rows(g.pctx, idx.data_ptr(), stats.data_ptr(), 0.1, s.data_ptr(),
                                   s.numel(), None), "pbin_rows")
    raw = stats.cpu().numpy()
    counts = raw[:5].view(np.int64)
    pr, pi = st.pr[:, :n], st.pi[:, :n]
    act = pr[16] != 0.0
    want_idx = np.nonzero(act)[0]
    k = len(want_idx)
    np.testing.assert_array_equal(idx[:k].cpu().numpy(), want_idx)
    assert list(counts) == [k, int((~act).sum()), int((~(pr[16, act] > 0)).sum()),
                            int((pi[4, act] < 0).sum()),
                            int(((pi[2, act] != 0) | (pr[15, act] != 0.1)).sum())]
    assert raw[5] == pr[16, act].min() and raw[6] == pr[16, act].max()
    out = torch.empty(k * 8, dtype=torch.uint8, device="cuda")
    for col, row in ((2, 0), (3, 2), (4, 4), (5, 1), (6, 3), (7, 5), (8, 16), (9, 15)):
        for single in (0, 1):
            capi.check(lib.dustb_pbin_pack(g.pctx, idx.data_ptr(), k, col, single, out.data_ptr(),
                                           None), "pbin_pack")
            dt = np.float32 if single else np.float64
            got = out[:k * np.dtype(dt).itemsize].cpu().numpy().view(dt)
            np.testing.assert_array_equal(got, pr[row, act].astype(dt))
    capi.check(lib.dustb_pbin_pack(g.pctx, idx.data_ptr(), k, 0, 0, out.data_ptr(), None), "pack")
    tag = (pi[4].astype(np.int64).astype(np.uint64) << np.uint64(32)) | \
        (pi[1].astype(np.int64) & 0xFFFFFFFF).astype(np.uint64)
    ids = out.cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(ids, tag[act])
    capi.check(lib.dustb_pbin_pack(g.pctx, idx.data_ptr(), k, 1, 0, out.data_ptr(), None), "pack")
    np.testing.assert_array_equal(out[:4 * k].cpu().numpy().view(np.uint32), pi[2, act])
    # the byte shuffle of the id column, chunk by chunk (a ragged last chunk)
    capi.check(lib.dustb_pbin_pack(g.pctx, idx.data_ptr(), k, 0, 0, out.data_ptr(), None), "pack")
    chunk = 1000
    sh = torch.empty_like(out)
    capi.check(lib.dustb_pbin_shuffle(out.data_ptr(), k, 8, chunk, sh.data_ptr(), None), "shuffle")
    b = ids.view(np.uint8).reshape(k, 8)
    want = np.concatenate([b[r0:r0 + chunk].T.reshape(-1) for r0 in range(0, k, chunk)])
    np.testing.assert_array_equal(sh.cpu().numpy(), want)
