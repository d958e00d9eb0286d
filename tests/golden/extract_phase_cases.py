"""Extracts the phase-transition known answers of the reference's scenario test into phase_cases.json.

Reads game/src/bin/scenario_test.rs (test_phase_transition_scenario, :217-265) as text (nothing is
compiled or run): every `PhaseTest { name, material, temps: [..], expected: [MpssPhase::..] }`.
Each particle starts Solid (MpssBuffer::spawn) and goes through one apply_phase_transitions call.

    python tests/golden/extract_phase_cases.py /path/to/reference
"""
from __future__ import annotations

import json
import os
import re
import sys

SRC = "game/src/bin/scenario_test.rs"
PHASES = {"Solid": 0, "Liquid": 1, "Gas": 2, "Plasma": 3, "Granular": 4, "Crystal": 5, "Amorphous": 6}
PAT = re.compile(r"PhaseTest\s*\{\s*name:\s*\"(\w+)\",\s*material:\s*(\d+),\s*temps:\s*\[([^\]]*)\],\s*"
                 r"expected:\s*\[([^\]]*)\]", re.S)


def extract(ref_root: str) -> list[dict]:
    with open(os.path.join(ref_root, SRC), encoding="utf-8") as f:
        text = f.read()
    out = []
    for m in PAT.finditer(text):
        line = text.count("\n", 0, m.start()) + 1
        temps = [float(t) for t in m.group(3).split(",") if t.strip()]
        phases = [PHASES[p] for p in re.findall(r"MpssPhase::(\w+)", m.group(4))]
        out.append({"name": m.group(1), "material": int(m.group(2)), "temps": temps, "expected": phases,
                    "start": PHASES["Solid"], "source": "%s:%d" % (SRC, line)})
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <reference checkout root>" % sys.argv[0])
    root = sys.argv[1]
    rows = extract(root)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "phase_cases.json"), "w") as f:
        json.dump(rows, f, indent=1)
    print("%d cases" % len(rows))
