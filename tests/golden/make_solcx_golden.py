"""The reference's recorded solCx convergence study as a fixture.

Underworld/SysTest/PerformanceTests/expected/Underworld_Velic_solCx-analysis.cvg-convergence-rates.dat
holds, for testVelicSolCx.xml at 16², 32² and 64² elements, the relative L2 errors of
VelocityField (2 components), PressureField and StrainRateField (3 components) against the
Velic solCx analytic solution, and their convergence rates (slope of log error against
log h) with the correlation of each fit.  This script copies those numbers into
tests/golden/solcx_rates.json:

    GALE_REFERENCE_DIR=<reference tree> python tests/golden/make_solcx_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REL = "Underworld/SysTest/PerformanceTests/expected/Underworld_Velic_solCx-analysis.cvg-convergence-rates.dat"


def parse(text):
    rows, rates, corr, labels = [], None, None, None
    for line in text.splitlines():
        t = line.split()
        if not t or line.startswith("---"):
            continue
        if t[0] == "#Res":
            labels = t[1:]
        elif t[0] == "cvg." and t[1] == "rate":
            rates = [float(v) for v in t[2:]]
        elif t[0] == "corr.":
            corr = [float(v) for v in t[1:]]
        elif rates is None and len(t) == 7 and "e" in t[0]:
            rows.append([float(v) for v in t])
    return {"columns": labels, "h": [r[0] for r in rows], "errors": [r[1:] for r in rows], "rates": rates,
            "correlation": corr, "source": REL}


def main(ref):
    with open(os.path.join(ref, REL)) as f:
        d = parse(f.read())
    with open(os.path.join(HERE, "solcx_rates.json"), "w") as f:
        json.dump(d, f, indent=1)
    print(d)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["GALE_REFERENCE_DIR"])
