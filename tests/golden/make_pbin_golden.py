"""Generates tests/golden/pbin_golden.json: the particle science files that
tests/host/pbin_tool.cpp writes from host rows (athenak_b200/host/pbin.cpp), each read by
the reference's own reader (vis/python/pbin.py of the reference tree, given as the first
argument) whose columns must equal the rows the file was written from and whose check()
must report no problem.  Records each file's format version, particle count and SHA-256, so
that tests/test_pbin.py can require byte-identical files without the reference tree.

    python tests/golden/make_pbin_golden.py <reference tree>
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.test_pbin import build_tool, read_rows  # noqa: E402

ROWS = (("x1", 0), ("x2", 2), ("x3", 4), ("v1", 1), ("v2", 3), ("v3", 5), ("mass", 16),
        ("stopping_time", 15))


def main(ref_tree):
    sys.path.insert(0, os.path.join(ref_tree, "vis", "python"))
    import pbin as ref_pbin                     # the reference's reader
    exe = build_tool()
    out = {"files": {}}
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([exe, "host", d], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        for f in sorted(os.listdir(d)):
            if not f.endswith(".pbin"):
                continue
            name = f[:-5]
            path = os.path.join(d, f)
            snap = ref_pbin.read(path)
            problems = ref_pbin.check(snap)
            assert problems == [], (name, problems)
            pr, pi = read_rows(os.path.join(d, name + ".rows"))
            act = pr[16] != 0.0
            single = snap.header["particles"]["particle_real_precision"] == "single"
            for col, row in ROWS:
                # the columns in the file's precision; the header constants stay float64
                const = col in snap.constant_columns
                want = pr[row, act].astype(np.float32 if single and not const else np.float64)
                np.testing.assert_array_equal(np.asarray(snap.columns[col]), want)
            np.testing.assert_array_equal(np.asarray(snap.columns["species"]), pi[2, act])
            tag = (pi[4].astype(np.int64).astype(np.uint64) << np.uint64(32)) | \
                (pi[1].astype(np.int64) & 0xFFFFFFFF).astype(np.uint64)
            np.testing.assert_array_equal(np.asarray(snap.columns["id"]), tag[act])
            out["files"][name] = {
                "version": int(snap.preamble["version"]),
                "n_particles": int(len(snap)),
                "constant_columns": sorted(snap.constant_columns),
                "sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
            }
    with open(os.path.join(HERE, "pbin_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main(sys.argv[1])
