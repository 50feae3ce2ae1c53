"""Copy the reference's yielding-suite known answers into a JSON fixture.

The reference's VonMisesYieldingSuite and ByerleeYieldingSuite (Underworld/Rheology/tests/
{VonMises,Byerlee}YieldingSuite.cxx) run the model of testYieldCriterion.xml and write,
for every material point that yields during a non-linear iteration after the first,
"Material yielded at time T (step S) within:" and the x and y extents of those points,
each formatted "%12.4g".  Their expected outputs are
Underworld/Rheology/tests/expected/test{VonMises,Byerlee}YieldCriterion.expected.  This
script stores those lines and the numbers in them in tests/golden/yield_suites.json.  Run
here, where the reference is mounted:

    python tests/golden/make_yield_golden.py /root/reference
"""
import json
import os
import re
import sys


def parse(path):
    lines = [ln.rstrip("\n") for ln in open(path) if ln.strip()]
    m = re.match(r"Material yielded at time\s+(\S+) \(step (\d+)\) within:", lines[0])
    ext = {}
    for ln in lines[1:]:
        a, lo, hi = re.match(r"\s*(\w): +(\S+) - +(\S+)", ln).groups()
        ext[a] = [float(lo), float(hi)]
    return {"lines": lines, "time": float(m.group(1)), "step": int(m.group(2)), "extents": ext}


def main(ref):
    base = os.path.join(ref, "Underworld", "Rheology", "tests", "expected")
    out = {kind: parse(os.path.join(base, f"test{kind}YieldCriterion.expected")) for kind in ("VonMises", "Byerlee")}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "yield_suites.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["GALE_REFERENCE_DIR"])
