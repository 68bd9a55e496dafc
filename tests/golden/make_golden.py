"""Extracts the reference's own known answers for the contact path into
reference_known_answers.json.

Run where the reference sources are mounted, with REFERENCE_ROOT naming the reference project's root; the
committed JSON is what the tests read, so they run without the reference.  Sources read:
  Solver/CollisionDetector/lbvh.cpp         LBVH::unit_test answers (Morton codes) and the
                                            expected ranges / splits / children / parents
                                            written beside fn_build_inner_nodes
  Solver/CollisionDetector/narrow_phase.cpp NarrowPhasesDetector::unit_test VF / EE CCD cases
"""
from __future__ import annotations

import json
import os
import re
import sys

REF = os.environ.get("REFERENCE_ROOT", "")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_known_answers.json")


def _read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def _ints(s):
    return [int(v) for v in re.findall(r"-?\d+", s)]


def _vec3(src, name):
    m = re.search(name + r"\s*=\s*luisa::make_float3\(([^)]*)\)", src)
    return [float(v) for v in m.group(1).split(",")]


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("set REFERENCE_ROOT to the reference project's root")
    lbvh = _read("Solver/CollisionDetector/lbvh.cpp")
    m32 = re.search(r"answer_morton32\s*=\s*\{([^}]*)\}", lbvh)
    m64 = re.search(r"answer_morton64\s*=\s*\{([^}]*)\}", lbvh)
    ranges = re.search(r"Should be \[(0 -> 7[^\]]*)\]", lbvh)
    splits = re.search(r"Should be \[(4, 0, 1[^\]]*)\]", lbvh)
    children = re.search(r"Should be (\[\[4, 5\].*?)\n", lbvh)
    parents = re.search(r"Should be \[(0, 2, 4[^\]]*)\]", lbvh)
    rng = [tuple(int(x) for x in p.split("->")) for p in ranges.group(1).split(",")]
    ch = [[int(a), int(b)] for a, b in re.findall(r"\[(\d+), (\d+)\]", children.group(1))]

    npc = _read("Solver/CollisionDetector/narrow_phase.cpp")
    vf = {
        "desire_toi": float(re.search(r"const float desire_toi = ([0-9.]+)", npc).group(1)),
        "offset": 1e-3,
        **{k: _vec3(npc, "case_" + k) for k in ("t0_p", "t1_p", "t0_f0", "t0_f1", "t0_f2", "t1_f0", "t1_f1", "t1_f2")},
    }
    ee_src = npc[npc.index("// EE CCD Test"):]
    ee = {
        "thickness": float(re.search(r"const float thickenss = ([0-9.]+)", ee_src).group(1)),
        **{k: _vec3(ee_src, "case_" + k) for k in ("ea_t0_p0", "ea_t0_p1", "eb_t0_p0", "eb_t0_p1", "ea_t1_p0",
                                                    "ea_t1_p1", "eb_t1_p0", "eb_t1_p1")},
    }
    data = {
        "source": "LuisaComputeSimulator unit tests (lbvh.cpp LBVH::unit_test, narrow_phase.cpp unit_test)",
        "lbvh_unit": {
            "leaves": 8,
            "morton32": _ints(m32.group(1)),
            "morton64": _ints(m64.group(1)),
            "ranges": [list(r) for r in rng],
            "splits": _ints(splits.group(1)),
            "children": ch[:7],
            "parents_nonroot": _ints(parents.group(1))[1:],
        },
        "refit_complete_tree": {"depths": list(range(1, 11)), "root": "[0, 2^depth]^3"},
        "vf_ccd": vf,
        "ee_ccd": ee,
    }
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(OUT)


if __name__ == "__main__":
    sys.exit(main())
