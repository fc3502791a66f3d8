"""Extract the reference's hex-exact golden vectors into JSON fixtures.

The reference (GazzolaLab/elasticapp, "Elastica++") pins its Cosserat-rod step
against PyElastica-generated FP64 state written as C++ brace literals
(``std::strtod("0x1.8p-3", nullptr)`` or plain decimals) inside its Catch2
tests:

* ``tests/Unit/Systems/CosseratRods/FullRodTest/Test_PerturbedRodStep.cpp``
  (explicitly damped rod; 1 rod after 0/1/2/3/5 PositionVerlet steps and
  2 rods after 3 steps),
* ``tests/Unit/Systems/CosseratRods/FullRodTest/Test_PerturbedRodStepWithoutDamping.cpp``
  (undamped rod; 1 rod after 0/1/3/5 steps),
* ``tests/Unit/Systems/CosseratRods/FullRodTest/Test_PerturbedRod.cpp``
  (state injection round trips for 2 rods).

This script reads those files as text (nothing is compiled or run) and writes
``tests/golden/<name>.json``.  Every number is stored as ``float.hex`` so the
fixtures are bit-exact.  Run it from a checkout that has the reference at
``/root/reference`` (or pass ``--reference``); the JSON it produced is
committed, so the tests never need the reference at run time.

Layout conventions kept from the reference (``CosseratRodTraits.hpp``):
vectors are 3 x N row-major (row = x, y, z), tensors are 3 x 3 x N
(page = director d_k, row = lab component, column = element).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REL_DIR = "tests/Unit/Systems/CosseratRods/FullRodTest"
FILES = {
    "perturbed_rod_step": "Test_PerturbedRodStep.cpp",
    "perturbed_rod_step_without_damping": "Test_PerturbedRodStepWithoutDamping.cpp",
    "perturbed_rod": "Test_PerturbedRod.cpp",
}

DECL = re.compile(
    r"blaze::Dynamic(Vector|Matrix|Tensor)<elastica::real_t>\s+"
    r"ROD(\d+)_(\w+?)_(REPLACED|PYEL)\(\s*([0-9UL,\s]+)\);\s*"
    r"ROD\d+_\w+?_(?:REPLACED|PYEL)\s*=\s*(\{.*\});"
)
NUM = re.compile(r'std::strtod\("([^"]+)",\s*nullptr\)|(-?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)')


def parse_values(literal: str) -> list[float]:
    out = []
    for m in NUM.finditer(literal):
        if m.group(1) is not None:
            out.append(float.fromhex(m.group(1)))
        else:
            out.append(float(m.group(2)))
    return out


def parse_file(path: str) -> list[dict]:
    """Return one dict per ELASTICA_TEST_CASE with its blocks of literals."""
    cases: list[dict] = []
    case = None
    section = None
    with open(path, "r", encoding="utf-8") as f:
        lines = f.readlines()
    for lineno, line in enumerate(lines, start=1):
        m = re.search(r'ELASTICA_TEST_CASE\(\s*"([^"]+)"', line)
        if m is None and "ELASTICA_TEST_CASE(" in line:
            # name on the next line
            m = re.search(r'"([^"]+)"', lines[lineno])
        if m is not None:
            case = {"name": m.group(1), "line": lineno, "inject": {},
                    "sections": [], "epsilon": None, "n_rods": 0}
            cases.append(case)
            section = None
            continue
        if case is None:
            continue
        m = re.search(r'SECTION\("([^"]+)"\)', line)
        if m:
            section = {"name": m.group(1), "line": lineno, "steps": 0,
                       "epsilon": None, "expected": {}}
            case["sections"].append(section)
            continue
        m = re.search(r"approx\.epsilon\(([-+0-9.eE]+)\)", line)
        if m:
            eps = float(m.group(1))
            if section is not None:
                section["epsilon"] = eps
            continue
        m = re.search(r"Approx::custom\(\)\.epsilon\(([-+0-9.eE]+)\)", line)
        if m:
            case["epsilon"] = float(m.group(1))
            continue
        m = re.search(r"std::size_t step = (\d+);", line)
        if m and section is not None:
            section["steps"] = int(m.group(1))
            continue
        m = DECL.search(line)
        if m:
            kind, rod, field, tag, dims, literal = m.groups()
            dims = [int(d.strip().rstrip("UL")) for d in dims.split(",")]
            values = parse_values(literal)
            n = 1
            for d in dims:
                n *= d
            if len(values) != n:
                raise ValueError(f"{path}:{lineno}: {field} has {len(values)} values, dims {dims}")
            rod = int(rod)
            case["n_rods"] = max(case["n_rods"], rod + 1)
            entry = {"dims": dims, "hex": [v.hex() for v in values], "line": lineno}
            if tag == "REPLACED":
                case["inject"].setdefault(str(rod), {})[field] = entry
            else:
                # expected values: inside a SECTION, or at test-case level
                target = section["expected"] if section is not None else case.setdefault("expected", {})
                target.setdefault(str(rod), {})[field] = entry
    return cases


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args(argv)
    for name, fname in FILES.items():
        path = os.path.join(args.reference, REL_DIR, fname)
        cases = parse_file(path)
        doc = {
            "source": f"{REL_DIR}/{fname}",
            "generator": "tests/golden/make_golden.py (text extraction, no reference code executed)",
            "note": "Values are PyElastica FP64 outputs embedded in the reference's Catch2 tests; "
                    "float.hex strings; vectors 3xN row-major, tensors 3x3xN page-major.",
            "cases": cases,
        }
        out = os.path.join(args.out, f"{name}.json")
        with open(out, "w", encoding="utf-8") as f:
            json.dump(doc, f, indent=1, sort_keys=True)
        n_sec = sum(len(c["sections"]) for c in cases)
        print(f"{out}: {len(cases)} cases, {n_sec} sections")
    return 0


if __name__ == "__main__":
    sys.exit(main())
