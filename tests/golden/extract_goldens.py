"""Generates tests/golden/reference_goldens.json from the msbg-rs test sources.

The reference's differential tests hard-code golden values produced by the
original C++ MSBG binaries.  This script reads them as text from a checkout of
msbg-rs (the first argument, else the MSBG_RS_DIR environment variable) and
writes them, with their file:line provenance, into reference_goldens.json,
which the tests load.  Run it only where the reference checkout exists:

    python tests/golden/extract_goldens.py path/to/msbg-rs
"""
from __future__ import annotations

import json
import os
import re
import sys


def _floats(text: str):
    return [float(t) for t in re.findall(r"-?\d+(?:\.\d+)?(?:e-?\d+)?", text)]


def _block(src: str, start_pat: str, end_pat: str = r"\];"):
    m = re.search(start_pat, src)
    if not m:
        raise SystemExit(f"pattern not found: {start_pat}")
    rest = src[m.end():]
    e = re.search(end_pat, rest)
    line = src[: m.start()].count("\n") + 1
    return rest[: e.start()], line


def main(root: str) -> None:
    out = {}
    # tests/difftest_stencil.rs
    p = os.path.join(root, "tests", "difftest_stencil.rs")
    s = open(p).read()
    idx_text, idx_line = _block(s, r"const SAMPLE_IDX: \[usize; 10\] = \[", r"\];")
    gold_text, gold_line = _block(s, r"const GOLDEN: \[\[f32; 10\]; 3\] = \[")
    g = [_floats(row) for row in re.findall(r"\[([^\[\]]+)\]", gold_text)]
    out["stencil"] = {
        "source": f"tests/difftest_stencil.rs:{idx_line},{gold_line}",
        "sample_idx": [int(v) for v in _floats(idx_text)],
        "golden": {"laplacian": g[0], "mean_curvature": g[1], "bilaplacian": g[2]},
        "dt": 0.01, "tol": 1e-4, "block_id": 21,
    }
    # tests/difftest_smoother.rs
    p = os.path.join(root, "tests", "difftest_smoother.rs")
    s = open(p).read()
    idx_text, idx_line = _block(s, r"const SAMPLE_IDX: \[usize; 12\] = \[")
    gold_text, gold_line = _block(s, r"const GOLDEN: \[\[f32; 12\]; 2\] = \[")
    g = [_floats(row) for row in re.findall(r"\[([^\[\]]+)\]", gold_text)]
    out["smoother"] = {
        "source": f"tests/difftest_smoother.rs:{idx_line},{gold_line}",
        "sample_idx": [int(v.replace("_", "")) for v in re.findall(r"[\d_]+", idx_text)],
        "golden": {"laplacian": g[0], "mean_curvature": g[1]},
        "dt": 0.01, "iterations": 4, "tol": {"laplacian": 1e-4, "mean_curvature": 1e-3},
    }
    # tests/difftest_interp.rs
    p = os.path.join(root, "tests", "difftest_interp.rs")
    s = open(p).read()
    pos_text, pos_line = _block(s, r"const POSITIONS: \[\[f32; 3\]; 8\] = \[")
    gold_text, gold_line = _block(s, r"const GOLDEN: \[\[f32; 14\]; 8\] = \[")
    out["interp"] = {
        "source": f"tests/difftest_interp.rs:{pos_line},{gold_line}",
        "positions": [_floats(r) for r in re.findall(r"\[([^\[\]]+)\]", pos_text)],
        "golden": [_floats(r) for r in re.findall(r"\[([^\[\]]+)\]", gold_text)],
        "tol": 1e-4,
        "columns": "linear value, gx, gy, gz, cubic value, gx, gy, gz, fxx, fyy, fzz, fxy, fxz, fyz",
    }
    # tests/difftest_cpp.rs
    p = os.path.join(root, "tests", "difftest_cpp.rs")
    s = open(p).read()
    m = re.search(r"const CPP_HASH: u64 = (0x[0-9a-f]+);", s)
    out["sparse_grid_hash"] = {
        "source": f"tests/difftest_cpp.rs:{s[: m.start()].count(chr(10)) + 1}",
        "hash": m.group(1),
    }
    # src/multires/sort.rs known answers
    p = os.path.join(root, "src", "multires", "sort.rs")
    s = open(p).read()
    answers = re.findall(r"assert_eq!\(morton3\((\d+), (\d+), (\d+)\), (0b[01]+|\d+)\);", s)
    out["morton3"] = {
        "source": "src/multires/sort.rs:63-100",
        "cases": [[int(a), int(b), int(c), int(v, 0)] for a, b, c, v in answers],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MSBG_RS_DIR")
    if not src:
        sys.exit("usage: extract_goldens.py path/to/msbg-rs (or set MSBG_RS_DIR)")
    main(src)
