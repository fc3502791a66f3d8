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
* ``tests/Unit/Systems/States/Expressions/SO3/Test_SO3PrimitiveAddAssign.cpp``
  (the director update from the identity by a fixed rotation vector, applied
  repeatedly; written to ``so3_add_assign.json``).

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


SO3_FILE = "tests/Unit/Systems/States/Expressions/SO3/Test_SO3PrimitiveAddAssign.cpp"
SO3_EXPECTED = re.compile(r"H_mat (expected_result_(\d))\{(.*?)\};", re.S)
SO3_DIRECTION = re.compile(r"DH_mat _derivative_data\{(.*?)\};", re.S)
SO3_ANGLE = re.compile(r"_derivative_data \*= ([0-9.]+) \* M_PI / 180\.0;")
SO3_TIMES = re.compile(r"Time first\(([0-9.]+)\), second\(([0-9.]+)\)")


def parse_so3(path: str) -> dict:
    """Rotation-vector inputs and the expected directors after 1, 2, 3
    applications of the SO(3) update.  Each expected tensor is 3 x 3 x 1 in
    page-major order, i.e. 9 values q[3 k + j] = component j of director d_k."""
    text = open(path, encoding="utf-8").read()

    def line_of(pos: int) -> int:
        return text.count("\n", 0, pos) + 1

    expected = []
    for m in SO3_EXPECTED.finditer(text):
        values = parse_values(m.group(3))
        if len(values) != 9:
            raise ValueError(f"{path}:{line_of(m.start())}: {m.group(1)} has {len(values)} values")
        expected.append({"name": m.group(1), "applications": int(m.group(2)), "line": line_of(m.start()),
                         "hex": [v.hex() for v in values]})
    d = SO3_DIRECTION.search(text)
    a = SO3_ANGLE.search(text)
    t = SO3_TIMES.search(text)
    if not (expected and d and a and t):
        raise ValueError(f"{path}: SO(3) test layout not recognised")
    direction = parse_values(d.group(1))
    return {
        "direction": [v.hex() for v in direction], "direction_line": line_of(d.start()),
        "angle_deg": float(a.group(1)).hex(), "angle_line": line_of(a.start()),
        "time_delta": (float(t.group(2)) - float(t.group(1))).hex(), "time_line": line_of(t.start()),
        "expected": expected,
    }

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
    so3 = parse_so3(os.path.join(args.reference, SO3_FILE))
    doc = {
        "source": SO3_FILE,
        "generator": "tests/golden/make_golden.py (text extraction, no reference code executed)",
        "note": "Rotation vector = time_delta * angle_deg * pi / 180 * direction / |direction|, applied "
                "to the identity director; expected directors q[3k+j] = component j of d_k; float.hex.",
        **so3,
    }
    out = os.path.join(args.out, "so3_add_assign.json")
    with open(out, "w", encoding="utf-8") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    print(f"{out}: {len(so3['expected'])} expected directors")
    return 0


if __name__ == "__main__":
    sys.exit(main())
