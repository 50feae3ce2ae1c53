"""The FP64 oracle's solution of the 2D viscoplastic extension configuration at full size
(extension_2d: 256×64 elements, 40 points per element, three layers, Drucker–Prager upper
crust with strain weakening, walls pulled at ±1, 20 Picard steps) as a fixture.

The oracle (oracle/gale_oracle.c) runs SystemLinearEquations_NonLinearExecute's loop, 20
Picard steps, twice: with Uzawa tolerance 1e-8 (inner 1e-10) — the reference solution —
and with the benchmark's Uzawa tolerance 1e-5 and the reference's inner tolerance 1e-6, to
record the oracle's own distance from the tight run.  Stored: velocity and pressure of the
tight run (float32), the per-point yield flags of both runs (bit-packed), the Picard
residuals and the 1e-5 run's velocity error:  tests/golden/extension_solution.npz.  Takes
about 13 minutes on 6 host threads:

    python tests/golden/make_extension_solution.py [threads]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gale_b200 import workloads  # noqa: E402
from gale_b200.stokes import UzawaSolver  # noqa: E402
from oracle import oracle  # noqa: E402


def main(threads):
    oracle.build()
    oracle.set_threads(threads)
    w = workloads.extension_2d()
    t0 = time.time()
    O = w.apply(oracle.OracleProblem(w.mesh))
    ut, pt, st_t = O.picard(w.picard, UzawaSolver(tolerance=1e-8, innerRtolFactor=0.01, maxIterations=20000,
                                                  innerMaxIterations=400000))
    yt = O.point_yield()[1]
    O = w.apply(oracle.OracleProblem(w.mesh))
    u5, p5, st5 = O.picard(w.picard, UzawaSolver(tolerance=1e-5))
    y5 = O.point_yield()[1]
    err5 = float(np.linalg.norm(u5 - ut) / np.linalg.norm(ut))
    np.savez(os.path.join(HERE, "extension_solution.npz"), u=ut.astype(np.float32),
             p=(pt - pt.mean()).astype(np.float32), yielded=np.packbits(yt), yielded_rtol5=np.packbits(y5),
             picard_residual=np.array([st_t["residual"], st5["residual"]]),
             picard_iterations=np.array([st_t["iterations"], st5["iterations"]]),
             oracle_rtol5_u_err=np.array([err5]), n_points=np.array([yt.shape[0]]), seconds=np.array([time.time() - t0]))
    print(st_t, st5, err5, time.time() - t0)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1))
