"""The multigrid hierarchy's dense coarse solve: the FP32 inverse that the blocked
Gauss–Jordan inversion (pivot blocks of 64, the last one ragged) writes against numpy's
inverse of the same FP64 operator (needs a B200)."""
import ctypes as C

import numpy as np
import pytest

from gale_b200 import workloads
from gale_b200.stokes import StokesProblem

pytestmark = pytest.mark.gpu


def coarse(G):
    n = C.c_int64(0)
    G._check(G.lib.gg_get_coarse_inverse(G.h, C.byref(n), None, None))
    m = n.value
    inv = np.zeros((m, m), np.float32)
    op = np.zeros((m, m), np.float64)
    G._check(G.lib.gg_get_coarse_inverse(G.h, C.byref(n), inv.ctypes.data_as(C.POINTER(C.c_float)),
                                         op.ctypes.data_as(C.POINTER(C.c_double))))
    return inv, op


# coarsest levels: 16³ → 8³ (2,187 dofs: 34 full blocks and one of 11), 64² → 32² (2,178
# dofs), 4³ → 2³ (81 dofs: a full block and one of 17), 8² → 4² (50 dofs: one block)
@pytest.mark.parametrize("make,n", [(lambda: workloads.creep_3d(n=16), 2187),
                                    (lambda: workloads.sinker_2d(n=64), 2178),
                                    (lambda: workloads.creep_3d(n=4), 81),
                                    (lambda: workloads.sinker_2d(n=8), 50)],
                         ids=["3d-2187", "2d-2178", "3d-81", "2d-50"])
def test_coarse_inverse_matches_numpy(make, n):
    w = make()
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("mixed")
    inv, op = coarse(G)
    assert inv.shape == (n, n)
    # Dirichlet rows and columns are the identity; the operator is symmetric
    assert np.allclose(op, op.T, rtol=0, atol=1e-12 * np.abs(op).max())
    ref = np.linalg.inv(op)
    # the FP64 elimination's own error is ~1e-16·cond; the FP32 rounding of each entry
    # bounds the rest at 2^-24 relative
    err = np.linalg.norm(inv.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, err
