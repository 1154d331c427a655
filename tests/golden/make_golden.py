"""Regenerate the golden fixtures of tests/golden/ from the reference sources.

The reference (Rust) cannot be built in this environment, so its known-answer
tables are read from its test sources as text:
  toro_star.json  <- fluid/crates/compressible/src/exact.rs, test
                     `toro_star_values` (Toro Tables 4.2/4.3, Tests 1-5, γ = 1.4,
                     with the test's tolerances).
Usage: python tests/golden/make_golden.py REFERENCE_ROOT
(REFERENCE_ROOT: the root of a checkout of the reference repository.)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def toro_star(ref_root):
    path = os.path.join(ref_root, "fluid/crates/compressible/src/exact.rs")
    src = open(path).read()
    body = src[src.index("fn toro_star_values"):]
    body = body[body.index("let cases = ["):body.index("];")]
    num = r"(-?[0-9.]+)"
    tup = rf"\(\({num}, {num}, {num}\), \({num}, {num}, {num}\), {num}, {num}\)"
    cases = []
    for m in re.finditer(tup, body):
        v = [float(x) for x in m.groups()]
        cases.append({"left": v[0:3], "right": v[3:6], "p_star": v[6], "u_star": v[7]})
    start = src[:src.index("fn toro_star_values")].count("\n") + 1
    return {
        "source": "fluid/crates/compressible/src/exact.rs:%d (toro_star_values)" % start,
        "gamma": 1.4,
        "tolerance": "|p - p*| <= 1e-4 max(|p*|, 1) + 1e-5; |u - u*| <= 1e-4 max(|u*|, 1)",
        "cases": cases,
    }


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py REFERENCE_ROOT")
    ref = sys.argv[1]
    data = toro_star(ref)
    assert len(data["cases"]) == 5, data
    with open(os.path.join(HERE, "toro_star.json"), "w") as f:
        json.dump(data, f, indent=1)
    print("wrote toro_star.json with", len(data["cases"]), "cases")


if __name__ == "__main__":
    main()
