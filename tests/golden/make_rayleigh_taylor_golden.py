"""Convert the reference's RayleighTaylorBenchmark regression checkpoint (step 10) into the
fixture tests/golden/rayleigh_taylor_benchmark.npz.

Source: Underworld/SysTest/RegressionTests/expected/RayleighTaylorBenchmark.xml/*.00010.h5
of the reference (checkpoint format version 1), read with gale_b200.checkpoint.load (no
libhdf5).  The 81,300 material points are kept as every 20th point (positions and material
indices) to keep the fixture small; fields, times and counts are kept whole.  Run from the
repository root:

    python tests/golden/make_rayleigh_taylor_golden.py /root/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from gale_b200 import checkpoint  # noqa: E402

REL = "Underworld/SysTest/RegressionTests/expected/RayleighTaylorBenchmark.xml"
STRIDE = 20


def load(ref_root: str) -> dict:
    c = checkpoint.load(os.path.join(ref_root, REL), 10)
    return {
        "velocity": c["velocity"],
        "pressure": c["pressure"],
        "positions_every_20th": c["positions"][::STRIDE],
        "material_every_20th": c["material_index"][::STRIDE],
        "points": np.array([len(c["positions"])]),
        "light_points": np.array([int((c["material_index"] == 1).sum())]),
        "current_time": np.array([c["current_time"]]),
        "dt": np.array([c["dt"]]),
        "vertices": c["vertices"],
    }


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = os.path.join(HERE, "rayleigh_taylor_benchmark.npz")
    np.savez_compressed(out, **load(ref))
    print("wrote", out)
