"""The FP64 oracle's converged solution of the 3D creep configuration at 32³ (creep_3d with
n = 32: 27 points per element, FK viscosity exp(9.21(0.5 − T)), Ra = 1e6, free slip) as a
fixture, with the oracle's own error at the benchmark tolerance.

The oracle (oracle/gale_oracle.c, the C restatement of the reference's path) solves the
Uzawa iteration to tolerance 1e-10 with inner Jacobi-CG tolerance 1e-12 (the discrete
solution to ~1e-9), and once more to the benchmark's Uzawa tolerance 1e-6 with the
reference's inner tolerance 1e-7.  The per-point viscosity of every 16th point (input
order) is kept too.  Stored as float32 (relative rounding 6e-8):
tests/golden/creep32_solution.npz.  Takes about ten minutes on 8 host threads:

    python tests/golden/make_creep_solution.py [threads]
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


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main(threads, n=32):
    oracle.build()
    oracle.set_threads(threads)
    w = workloads.creep_3d(n=n)
    O = w.apply(oracle.OracleProblem(w.mesh))
    O.assemble()
    t0 = time.time()
    tight = UzawaSolver(tolerance=1e-10, innerRtolFactor=0.01, maxIterations=5000, innerMaxIterations=400000)
    u, p, st = O.uzawa(tight)
    t1 = time.time()
    u6, p6, st6 = O.uzawa(UzawaSolver(tolerance=1e-6))
    pc, p6c = p - p.mean(), p6 - p6.mean()
    np.savez(os.path.join(HERE, f"creep{n}_solution.npz"), u=u.astype(np.float32), p=pc.astype(np.float32),
             eta_every16=O.point_viscosity()[::16].astype(np.float32),
             outer_iterations=np.array([st["outer_iterations"]]), inner_iterations=np.array([st["inner_iterations"]]),
             rel_residual=np.array([st["rel_residual"]]),
             oracle_rtol6_err=np.array([rel(u6, u), rel(p6c, pc)]),
             oracle_rtol6_iterations=np.array([st6["outer_iterations"], st6["inner_iterations"]]),
             seconds=np.array([t1 - t0]))
    print(st, st6, t1 - t0, time.time() - t1)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1))
