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


def _solve_uzawa(G, fused_uzawa, **kw):
    old = os.environ.get("GALE_B200_FUSED_UZAWA")
    os.environ["GALE_B200_FUSED_UZAWA"] = "1" if fused_uzawa else "0"
    try:
        return G.solve(UzawaSolver(precision="mixed", inner="mg", **kw))
    finally:
        if old is None:
            del os.environ["GALE_B200_FUSED_UZAWA"]
        else:
            os.environ["GALE_B200_FUSED_UZAWA"] = old


@pytest.mark.parametrize("case", ["sinker_2d", "creep_3d"])
@pytest.mark.parametrize("recycle", [True, False])
def test_uzawa_one_launch_matches_host_loop(case, recycle):
    """The whole mixed Uzawa solve as one persistent launch against the host-driven loop
    (one kernel at a time, a device-to-host read after every reduction): the same outer
    and inner algorithm, so the same discrete solution and near-equal iteration counts."""
    w = workloads.sinker_2d() if case == "sinker_2d" else workloads.creep_3d(n=32)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("mixed")
    tight = dict(tolerance=1e-9, innerRtolFactor=0.01, recycle=recycle)
    uh, ph, sh = _solve_uzawa(G, False, **tight)
    uf, pf, sf = _solve_uzawa(G, True, **tight)
    assert sh["uzawa_fused"] == 0 and sf["uzawa_fused"] == 1
    assert sf["rel_residual"] <= 1e-9 and sh["rel_residual"] <= 1e-9
    assert np.linalg.norm(uf - uh) <= 1e-6 * np.linalg.norm(uh)
    pc = lambda q: q - q.mean()
    assert np.linalg.norm(pc(pf) - pc(ph)) <= 1e-6 * np.linalg.norm(pc(ph))
    assert abs(sf["outer_iterations"] - sh["outer_iterations"]) <= 2
    assert abs(sf["inner_iterations"] - sh["inner_iterations"]) <= 0.1 * sh["inner_iterations"] + 5
    assert sf["inner_solves"] == sf["outer_iterations"] + 2
    # one launch for the solve (the host loop: hundreds)
    assert sf["fused_launches"] == 1 and sf["kernel_launches"] <= 2
    assert sh["kernel_launches"] > 50 * sf["kernel_launches"]


def test_uzawa_one_launch_iteration_limit():
    """maxIterations reached inside the launch: GG_ERR_NOT_CONVERGED with the residual
    reached, as from the host loop."""
    from gale_b200 import abi
    from gale_b200.stokes import GaleError
    w = workloads.creep_3d(n=16)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("mixed")
    errs = []
    for fused in (False, True):
        with pytest.raises(GaleError) as ei:
            _solve_uzawa(G, fused, tolerance=1e-12, maxIterations=3)
        assert ei.value.code == abi.GG_ERR_NOT_CONVERGED
        errs.append(ei.value.stats)
    assert errs[0]["outer_iterations"] == errs[1]["outer_iterations"] == 4
    assert errs[1]["uzawa_fused"] == 1
    assert abs(errs[0]["rel_residual"] - errs[1]["rel_residual"]) <= 1e-3 * errs[0]["rel_residual"]
