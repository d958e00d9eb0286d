"""Extracts the reference's known-answer assertions for the MPM kernels into known_answers.json.

Reads the Rust unit tests of the reference project as text (nothing is compiled or run):
  ae_particle/src/mpm_solver.rs    b_spline / b_spline_deriv        (tests at :1595-1609)
  ae_compute/src/mpm_compute.rs    quadratic_weight(_grad)           (tests at :1103-1132)
and records every `assert!((f(x) - e).abs() < tol)` / `assert!(f(x).abs() < tol)` with its
file:line.  Run once where the reference checkout is available:

    python tests/golden/extract_known_answers.py /path/to/reference
"""
from __future__ import annotations

import json
import os
import re
import sys

FILES = ["ae_particle/src/mpm_solver.rs", "ae_compute/src/mpm_compute.rs"]
FUNCS = ("b_spline", "b_spline_deriv", "quadratic_weight", "quadratic_weight_grad")
NUM = r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"
PAT_DIFF = re.compile(r"assert!\(\s*\(\s*(\w+)\((%s)\)\s*([-+])\s*\(?\s*(%s)\s*\)?\s*\)\.abs\(\)\s*<\s*(%s)" % (NUM, NUM, NUM))
PAT_ZERO = re.compile(r"assert!\(\s*\(?\s*(\w+)\((%s)\)\s*\)?\.abs\(\)\s*<\s*(%s)" % (NUM, NUM))


def extract(ref_root: str) -> list[dict]:
    out = []
    for rel in FILES:
        with open(os.path.join(ref_root, rel), encoding="utf-8") as f:
            lines = f.read().splitlines()
        for i, line in enumerate(lines, 1):
            m = PAT_DIFF.search(line)
            if m and m.group(1) in FUNCS:
                e = float(m.group(4))
                out.append({"function": m.group(1), "arg": float(m.group(2)),
                            "expected": e if m.group(3) == "-" else -e, "tol": float(m.group(5)),
                            "source": "%s:%d" % (rel, i)})
                continue
            m = PAT_ZERO.search(line)
            if m and m.group(1) in FUNCS:
                out.append({"function": m.group(1), "arg": float(m.group(2)), "expected": 0.0,
                            "tol": float(m.group(3)), "source": "%s:%d" % (rel, i)})
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % sys.argv[0])
    root = sys.argv[1]
    rows = extract(root)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "known_answers.json"), "w") as f:
        json.dump(rows, f, indent=1)
    print("%d assertions" % len(rows))
