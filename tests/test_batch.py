"""Batched uneven sweep: many independent problems through gg_solve_batch (needs a B200)."""
import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import StokesProblem, UzawaSolver

pytestmark = pytest.mark.gpu


def test_batch_matches_one_at_a_time(oracle_mod):
    ws = workloads.batch_sinkers(count=10, sizes=(8, 12, 16, 24))
    prm = UzawaSolver(tolerance=1e-7, precision="fp64")
    probs = [w.apply(StokesProblem(w.mesh)) for w in ws]
    res = StokesProblem.solve_batch(probs, prm, workers=4)
    for w, (u, p, st) in zip(ws, res):
        assert st["rel_residual"] <= 1e-7
        O = w.apply(oracle_mod.OracleProblem(w.mesh))
        O.assemble()
        uo, po, so = O.uzawa(prm)
        assert abs(st["outer_iterations"] - so["outer_iterations"]) <= 1
        # both stop at rel. pressure residual 1e-7; the GPU's moment-form sums round
        # differently from the oracle's assembled blocks, so the two iterates agree to the
        # solve tolerance times the problem's conditioning, not bitwise
        assert np.linalg.norm(u - uo) <= 1e-4 * np.linalg.norm(uo)


def test_batch_mixed_multigrid_and_status():
    ws = workloads.batch_sinkers(count=6, sizes=(16, 32))
    probs = [w.apply(StokesProblem(w.mesh)) for w in ws]
    res = StokesProblem.solve_batch(probs, UzawaSolver(tolerance=1e-6, precision="mixed", inner="mg"), workers=3)
    assert all(st["rel_residual"] <= 1e-6 for _, _, st in res)
    # a failing member is reported with its index
    bad = ws[0].apply(StokesProblem(ws[0].mesh))
    bad.set_points(np.ascontiguousarray(ws[0].coords[:10]))  # empty elements
    from gale_b200.stokes import GaleError
    with pytest.raises(GaleError):
        StokesProblem.solve_batch([probs[1], bad], UzawaSolver(tolerance=1e-6), workers=2)
