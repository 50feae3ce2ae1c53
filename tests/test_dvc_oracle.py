"""Discrete-Voronoi weights (DVCWeights) and population control (PCDVC) in the CPU
oracle: pinned to the reference's own known answers (no GPU needed)."""
import os

import numpy as np
import pytest

from gale_b200 import abi
from gale_b200.stokes import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("dim", [3, 2])
def test_dvc_matches_reference_known_answers(oracle_mod, dim):
    """DVCWeightsSuite_TestGetCentroids{,2D} (PICellerator/Weights/tests/DVCWeightsSuite.cxx):
    10 points, 10×10(×10) grid; the expected files print centroids and weights to 6
    decimals, and every weight is a cell count times the cell volume."""
    d = np.load(os.path.join(HERE, "golden", "dvc_suite.npz"))
    cent, w = oracle_mod.dvc_cell(dim, [10] * dim, d["points%d" % dim])
    da = 0.2 ** dim
    assert np.array_equal(np.rint(w / da), np.rint(d["weights%d" % dim] / da))
    assert np.abs(cent - d["centroids%d" % dim]).max() <= 5e-7 + 1e-12
    assert abs(w.sum() - 2.0 ** dim) < 1e-12


def test_dvc_partition_and_order_independence_of_distinct_points(oracle_mod):
    rng = np.random.default_rng(3)
    xi = rng.uniform(-1, 1, (27, 3))
    c, w = oracle_mod.dvc_cell(3, [10, 10, 10], xi)
    assert abs(w.sum() - 8.0) < 1e-12
    assert (w > 0).all()
    # each centroid lies inside the element
    assert (np.abs(c) < 1).all()


def _clustered_points(dim, n_el, seed):
    """Per element: 20 uniform points, or 4 (large regions → splits), or 20 with 8 packed
    near one corner (tiny regions → deletions); a second material in a few elements."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n_el
    pts, mat = [], []
    for idx in np.ndindex(*([n_el] * dim)):
        lo = np.array(idx) * h
        kind = rng.integers(0, 4)
        if kind == 0:
            p = lo + h * rng.uniform(0.05, 0.95, (4, dim))
        elif kind == 1:
            p = np.concatenate([lo + h * rng.uniform(0.05, 0.95, (12, dim)),
                                lo + h * (0.1 + 0.02 * rng.uniform(0, 1, (8, dim)))])
        else:
            p = lo + h * rng.uniform(0.05, 0.95, (20, dim))
        pts.append(p)
        m = np.zeros(len(p), dtype=np.int32)
        if rng.uniform() < 0.2:
            m[-1] = 1
        mat.append(m)
    return np.concatenate(pts), np.concatenate(mat)


@pytest.mark.parametrize("dim,n_el", [(2, 6), (3, 3)])
def test_population_control_oracle_invariants(oracle_mod, dim, n_el):
    mesh = Mesh(dim, [n_el] * dim)
    x, mat = _clustered_points(dim, n_el, 7)
    prm = oracle_mod.PcdvcParams(25.0, 0.6, 3, 2, 0, 0)
    out = oracle_mod.population_control(mesh, x, mat, None, prm, [10] * dim)
    assert out["splits"] > 0 and out["deletions"] > 0
    assert len(out["coords"]) == len(x) + out["splits"] - out["deletions"]
    # the weights of every element partition its reference volume (2^dim)
    cell = oracle_mod.locate(mesh, out["coords"])
    sums = np.bincount(cell, weights=out["weight"], minlength=n_el ** dim)
    assert np.allclose(sums, 2.0 ** dim, atol=1e-12)
    # the new points sit where their parents' regions had their centroids, inside the element
    assert (np.abs(out["xi"]) < 1).all()
    # interface elements (two materials) neither split nor delete by default
    cell0 = oracle_mod.locate(mesh, x)
    for e in range(n_el ** dim):
        if len(set(mat[cell0 == e])) > 1:
            assert (cell == e).sum() == (cell0 == e).sum()
