"""The batched CTA solver (gale_b200/csrc/gg_cta.cu): one launch solves every problem of a
batch, one CTA per problem (needs a B200).

- every problem reaches the Uzawa tolerance, and its velocity and pressure are as close to
  the oracle's converged solution as the FP64 oracle's own solve at the same tolerance
  (within 1.5× plus 1e-6), on uneven sizes;
- the element applies sum over parity classes and the reductions run in a fixed order, so
  solving the same batch twice gives the same bits;
- the batch reports one kernel launch per problem (the shared launch).
"""
import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import StokesProblem, UzawaSolver

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_cta_batch_against_oracle_and_reproducible(oracle_mod):
    ws = workloads.batch_sinkers(count=8, sizes=(16, 24, 32, 48))
    prm = UzawaSolver(tolerance=1e-6, precision="mixed", inner="mg")
    probs = [w.apply(StokesProblem(w.mesh)) for w in ws]
    first = StokesProblem.solve_batch(probs, prm, workers=4)
    second = StokesProblem.solve_batch(probs, prm, workers=4)
    for (u1, p1, s1), (u2, p2, s2) in zip(first, second):
        assert np.array_equal(u1, u2) and np.array_equal(p1, p2)
        assert s1["kernel_launches"] == 1
    for w, (u, p, st) in zip(ws, first):
        assert st["rel_residual"] <= 1e-6
        O = w.apply(oracle_mod.OracleProblem(w.mesh))
        O.assemble()
        ut, pt, _ = O.uzawa(UzawaSolver(tolerance=1e-11, innerRtolFactor=0.01, maxIterations=5000,
                                        innerMaxIterations=200000))
        uo, po, _ = O.uzawa(UzawaSolver(tolerance=1e-6))
        pc, ptc, poc = p - p.mean(), pt - pt.mean(), po - po.mean()
        assert rel(u, ut) <= 1.5 * rel(uo, ut) + 1e-6, (w.mesh.elements[0], rel(u, ut), rel(uo, ut))
        assert rel(pc, ptc) <= 1.5 * rel(poc, ptc) + 1e-6, (w.mesh.elements[0], rel(pc, ptc), rel(poc, ptc))
