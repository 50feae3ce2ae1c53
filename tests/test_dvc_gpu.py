"""DVCWeights and PCDVC on the GPU against the CPU oracle (needs a B200).  Same
algorithm, same double roundings: the integration points, weights and the rebuilt point
set must agree bit for bit; the moments built from them to summation order."""
import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import GaleError, Mesh, StokesProblem, UzawaSolver

from test_dvc_oracle import _clustered_points

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: workloads.sinker_2d(n=16), lambda: workloads.creep_3d(n=8)],
                         ids=["2d", "3d"])
def test_dvc_weights_bit_exact(oracle_mod, make):
    w = make()
    G = w.apply(StokesProblem(w.mesh))
    G.set_weights("dvc", 10)
    G.locate()
    xi, wt = G.integration_points()
    cent, w_ref = oracle_mod.dvc_weights(w.mesh, w.coords, [10] * w.dim)
    assert np.array_equal(wt, w_ref)
    assert np.array_equal(xi, cent)
    assert np.allclose(np.bincount(oracle_mod.locate(w.mesh, w.coords), weights=wt), 2.0 ** w.dim, atol=1e-12)


@pytest.mark.parametrize("dim,n_el,seed", [(2, 6, 7), (2, 16, 8), (3, 3, 7), (3, 6, 9)])
def test_population_control_bit_exact(oracle_mod, dim, n_el, seed):
    mesh = Mesh(dim, [n_el] * dim)
    x, mat = _clustered_points(dim, n_el, seed)
    ps = np.linspace(0.0, 0.1, len(x))
    G = StokesProblem(mesh)
    G.set_points(x, mat, ps)
    G.set_weights("dvc", 10)
    G.locate()
    st = G.population_control()
    prm = oracle_mod.PcdvcParams(25.0, 0.6, 3, 2, 0, 0)
    ref = oracle_mod.population_control(mesh, x, mat, ps, prm, [10] * dim)
    assert st["splits"] == ref["splits"] and st["deletions"] == ref["deletions"]
    assert st["splits"] > 0 and st["deletions"] > 0
    assert st["points_after"] == len(ref["coords"])
    gx, gm, gps = G.points()
    assert np.array_equal(gx, ref["coords"])
    assert np.array_equal(gm, ref["material"])
    assert np.array_equal(gps, ref["plastic_strain"])
    xi, wt = G.integration_points()
    assert np.array_equal(wt, ref["weight"])
    assert np.array_equal(xi, ref["xi"])


def test_population_control_interface_flags(oracle_mod):
    mesh = Mesh(2, [8, 8])
    x, mat = _clustered_points(2, 8, 11)
    for flags in [(1, 0), (0, 1), (1, 1)]:
        G = StokesProblem(mesh)
        G.set_points(x, mat)
        G.set_weights("dvc", [12, 8])
        G.locate()
        st = G.population_control(upperT=20.0, lowerT=1.0, maxSplits=2, maxDeletions=3,
                                  splitInInterfaceCells=bool(flags[0]), deleteInInterfaceCells=bool(flags[1]))
        prm = oracle_mod.PcdvcParams(20.0, 1.0, 2, 3, flags[0], flags[1])
        ref = oracle_mod.population_control(mesh, x, mat, None, prm, [12, 8])
        assert (st["splits"], st["deletions"]) == (ref["splits"], ref["deletions"])
        gx, gm, _ = G.points()
        assert np.array_equal(gx, ref["coords"]) and np.array_equal(gm, ref["material"])


def test_build_with_dvc_weights_matches_oracle(oracle_mod):
    w = workloads.sinker_2d(n=16)
    G = w.apply(StokesProblem(w.mesh))
    G.set_weights("dvc", 10)
    G.locate()
    G.build_operator("mixed")
    xi, wt = G.integration_points()
    O = w.apply(oracle_mod.OracleProblem(w.mesh))
    O.set_integration_points(oracle_mod.locate(w.mesh, w.coords), xi, wt, w.material)
    O.assemble()
    m_g, m_o = G.moments(), O.moments()
    assert np.linalg.norm(m_g - m_o) <= 1e-12 * np.linalg.norm(m_o)
    u, p, st = G.solve(UzawaSolver(tolerance=1e-6, precision="mixed", inner="mg"))
    assert st["rel_residual"] <= 1e-6


def test_population_control_statuses():
    w = workloads.sinker_2d(n=8)
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    with pytest.raises(GaleError) as e:
        G.population_control()
    assert e.value.code == -8  # GG_ERR_STATE: needs the DVC weights
    G.set_weights("dvc", 10)
    G.locate()
    with pytest.raises(GaleError) as e:
        G.population_control(Inflow=True)
    assert e.value.code == -1
    with pytest.raises(GaleError):
        G.set_weights("dvc", 40)  # 40 × 40 > 1024 cells
