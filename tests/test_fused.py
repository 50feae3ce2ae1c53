"""Persistent multigrid FCG (one cooperative launch per inner solve) against the
graph-captured kernel sequence it replaces (needs a B200)."""
import os

import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import StokesProblem, UzawaSolver

pytestmark = pytest.mark.gpu


def _solve(G, fused, **kw):
    old = os.environ.get("GALE_B200_FUSED_FCG")
    os.environ["GALE_B200_FUSED_FCG"] = "1" if fused else "0"
    try:
        return G.solve(UzawaSolver(precision="mixed", inner="mg", **kw))
    finally:
        if old is None:
            del os.environ["GALE_B200_FUSED_FCG"]
        else:
            os.environ["GALE_B200_FUSED_FCG"] = old


@pytest.mark.parametrize("case", ["sinker_2d", "creep_3d"])
def test_fused_matches_graph_path(case):
    w = workloads.sinker_2d() if case == "sinker_2d" else workloads.creep_3d(n=32)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("mixed")
    tight = dict(tolerance=1e-9, innerRtolFactor=0.01)
    ug, pg, sg = _solve(G, False, **tight)
    uf, pf, sf = _solve(G, True, **tight)
    assert sf["rel_residual"] <= 1e-9 and sg["rel_residual"] <= 1e-9
    # same algorithm, different FP32 atomic order: same discrete solution, near-equal counts
    assert np.linalg.norm(uf - ug) <= 1e-6 * np.linalg.norm(ug)
    pc = lambda q: q - q.mean()
    assert np.linalg.norm(pc(pf) - pc(pg)) <= 1e-6 * np.linalg.norm(pc(pg))
    assert abs(sf["outer_iterations"] - sg["outer_iterations"]) <= 2
    assert sf["inner_iterations"] <= 1.1 * sg["inner_iterations"] + 5
    # one launch per inner sweep instead of a graph of ~100 kernels per iteration
    assert sf["kernel_launches"] < 0.5 * sg["kernel_launches"]


def test_fused_default_rtol_and_repeat():
    w = workloads.creep_3d(n=16)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("mixed")
    u1, p1, s1 = _solve(G, True, tolerance=1e-6)
    u2, p2, s2 = _solve(G, True, tolerance=1e-6)
    assert s1["rel_residual"] <= 1e-6 and s2["rel_residual"] <= 1e-6
    assert s1["outer_iterations"] == s2["outer_iterations"]
    assert np.linalg.norm(u1 - u2) <= 1e-5 * np.linalg.norm(u1)
