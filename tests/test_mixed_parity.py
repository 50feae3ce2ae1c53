"""The mixed FP32/FP64 path against the CPU FP64 oracle on the benchmark's own
configuration family (needs a B200).

creep_3d at 32³ (27 points per element, FK viscosity with a 1e4 contrast, Ra = 1e6, free
slip): tests/golden/creep32_solution.npz holds the oracle's solution converged to Uzawa
tolerance 1e-10 (inner 1e-12) and the oracle's own error at the benchmark tolerance 1e-6
(made by tests/golden/make_creep_solution.py).

Stated tolerance of the mixed path: at any Uzawa tolerance it is as accurate as the FP64
solver at that tolerance — its velocity and pressure errors against the converged oracle
solution are at most 1.5× the FP64 solver's own errors plus 1e-6.  The velocity and
pressure errors are relative L2 (pressure after removing its mean: the free-slip box leaves
it defined up to a constant, and the reference removes no null space,
Stokes_SLE_UzawaSolver.cxx:648-650).
"""
import os

import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import StokesProblem, UzawaSolver

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def creep32():
    ref = np.load(os.path.join(HERE, "golden", "creep32_solution.npz"))
    w = workloads.creep_3d(n=32)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    return w, G, ref


def test_point_viscosity_is_the_oracles(creep32):
    w, G, ref = creep32
    G.build_operator("mixed")
    eta = G.point_viscosity()[::16]
    assert rel(eta, ref["eta_every16"].astype(np.float64)) < 1e-6  # fixture stored in FP32


def test_mixed_at_benchmark_tolerance(creep32):
    w, G, ref = creep32
    ut, pt = ref["u"].astype(np.float64), ref["p"].astype(np.float64)
    eu_oracle, ep_oracle = ref["oracle_rtol6_err"]
    G.build_operator("mixed")
    u, p, st = G.solve(UzawaSolver(tolerance=1e-6, precision="mixed", inner="mg", smoothingDegree=3))
    assert st["rel_residual"] <= 1e-6
    assert rel(u, ut) <= 1.5 * eu_oracle + 1e-6, (rel(u, ut), eu_oracle)
    assert rel(p - p.mean(), pt) <= 1.5 * ep_oracle + 1e-6, (rel(p - p.mean(), pt), ep_oracle)


def test_mixed_at_tight_tolerance_matches_fp64(creep32):
    # at Uzawa tolerance 1e-9 both paths sit ~1e-6 (velocity) from the discrete solution;
    # the mixed one stays within the stated tolerance of the FP64 path's own error
    w, G, ref = creep32
    ut, pt = ref["u"].astype(np.float64), ref["p"].astype(np.float64)
    tight = dict(tolerance=1e-9, innerRtolFactor=0.01, maxIterations=5000)
    G.build_operator("fp64")
    u64, p64, _ = G.solve(UzawaSolver(precision="fp64", innerMaxIterations=400000, **tight))
    G.build_operator("mixed")
    um, pm, st = G.solve(UzawaSolver(precision="mixed", inner="mg", smoothingDegree=3, **tight))
    e64u, e64p = rel(u64, ut), rel(p64 - p64.mean(), pt)
    emu, emp = rel(um, ut), rel(pm - pm.mean(), pt)
    assert e64u < 1e-5 and e64p < 1e-4, (e64u, e64p)
    assert emu <= 1.5 * e64u + 1e-6, (emu, e64u)
    assert emp <= 1.5 * e64p + 1e-6, (emp, e64p)


@pytest.fixture(scope="module")
def extension():
    ref = np.load(os.path.join(HERE, "golden", "extension_solution.npz"))
    return workloads.extension_2d(), ref


def test_extension_picard_full_size(extension):
    # extension_2d at full size (256×64, 40 points per element, 20 Picard steps): the mixed
    # path at the benchmark's Uzawa tolerance 1e-5 stays within the stated tolerance of the
    # oracle's tight run (the oracle's own 1e-5 run is 4e-5 from it), with the same yielded
    # points
    w, ref = extension
    ut, pt = ref["u"].astype(np.float64), ref["p"].astype(np.float64)
    n = int(ref["n_points"][0])
    yt = np.unpackbits(ref["yielded"])[:n]
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    u, p, st = G.picard(w.picard, UzawaSolver(tolerance=1e-5, precision="mixed", inner="mg"))
    assert st["iterations"] == int(ref["picard_iterations"][1])
    e5 = float(ref["oracle_rtol5_u_err"][0])
    assert rel(u, ut) <= 1.5 * e5 + 1e-6, (rel(u, ut), e5)
    _, y = G.point_yield()
    assert np.mean(y != yt) <= 1e-4, int((y != yt).sum())
    # at the tight tolerance the mixed run lands on the oracle's
    G2 = w.apply(StokesProblem(w.mesh))
    G2.locate()
    u8, p8, _ = G2.picard(w.picard, UzawaSolver(tolerance=1e-8, innerRtolFactor=0.01, maxIterations=20000,
                                                precision="mixed", inner="mg"))
    assert rel(u8, ut) <= 1e-6
    assert rel(p8 - p8.mean(), pt) <= 1e-5
