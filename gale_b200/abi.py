"""ctypes mirror of ``include/gale_gpu.h`` and the loader of the sm_100a library.

The structures below are field-for-field copies of the C ABI structs; the loader
opens ``gale_b200/libgale_b200.so`` (built in-tree by ``gale_b200/build.py``) and
raises when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

GG_OK = 0
GG_ERR_INVALID = -1
GG_ERR_CUDA = -2
GG_ERR_NONFINITE = -3
GG_ERR_NOT_CONVERGED = -4
GG_ERR_STAGNATED = -5
GG_ERR_OUT_OF_DOMAIN = -6
GG_ERR_ZERO_FORCE = -7
GG_ERR_STATE = -8
GG_ERR_NO_DEVICE = -9
GG_ERR_EMPTY_CELL = -10

STATUS_NAMES = {
    0: "OK", -1: "INVALID", -2: "CUDA", -3: "NONFINITE", -4: "NOT_CONVERGED",
    -5: "STAGNATED", -6: "OUT_OF_DOMAIN", -7: "ZERO_FORCE", -8: "STATE",
    -9: "NO_DEVICE", -10: "EMPTY_CELL",
}

RHEO_MATERIAL_VISCOSITY = 1
RHEO_ARRHENIUS = 2
RHEO_FRANK_KAMENETSKII = 3
RHEO_VON_MISES = 4
RHEO_DRUCKER_PRAGER = 5
RHEO_BYERLEE = 6

PRECISION_FP64 = 0
PRECISION_MIXED = 1
INNER_JACOBI_CG = 0
INNER_MG_CG = 1
INNER_LEARNED_CG = 2
INNER_LEARNED_JACOBI_CG = 3
LEARN_BASE_MULTIGRID, LEARN_BASE_JACOBI = 0, 1

MAX_RHEOLOGIES = 4
MAX_MATERIALS = 16


class MeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("elements", C.c_int32 * 3),
                ("min", C.c_double * 3), ("max", C.c_double * 3)]


class VelocityBC(C.Structure):
    _fields_ = [("fixed", (C.c_uint8 * 3) * 6), ("value", (C.c_double * 3) * 6)]


class Rheology(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("strain_weakening", C.c_int32),
        ("eta0", C.c_double), ("activation_energy", C.c_double),
        ("activation_volume", C.c_double), ("reference_temp", C.c_double),
        ("theta", C.c_double), ("cohesion", C.c_double),
        ("cohesion_after_softening", C.c_double), ("friction_coefficient", C.c_double),
        ("friction_coefficient_after_softening", C.c_double),
        ("minimum_yield_stress", C.c_double), ("minimum_viscosity", C.c_double),
        ("max_strain_rate", C.c_double), ("depth_coefficient", C.c_double),
        ("strain_rate_softening", C.c_int32), ("pad", C.c_int32),
        ("boundary_cohesion", C.c_double), ("boundary_cohesion_after_softening", C.c_double),
        ("boundary_friction_coefficient", C.c_double),
        ("boundary_friction_coefficient_after_softening", C.c_double),
        ("boundary_walls", C.c_int32), ("hydrostatic_term", C.c_int32),
    ]


class StrainWeakening(C.Structure):
    _fields_ = [("initial_softening_strain", C.c_double),
                ("final_softening_strain", C.c_double), ("healing_rate", C.c_double)]


class Material(C.Structure):
    _fields_ = [("n_rheologies", C.c_int32), ("has_strain_weakening", C.c_int32),
                ("rheology", Rheology * MAX_RHEOLOGIES),
                ("strain_weakening", StrainWeakening),
                ("density", C.c_double), ("alpha", C.c_double)]


class BodyForce(C.Structure):
    _fields_ = [("gravity", C.c_double), ("g_hat", C.c_double * 3), ("rayleigh", C.c_double)]


class UzawaParams(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double), ("max_iterations", C.c_int32),
        ("min_iterations", C.c_int32), ("use_absolute_tolerance", C.c_int32),
        ("use_preconditioner", C.c_int32), ("inner", C.c_int32), ("precision", C.c_int32),
        ("inner_rtol_factor", C.c_double), ("inner_max_iterations", C.c_int32),
        ("reuse_pressure", C.c_int32), ("recycle_directions", C.c_int32), ("smoothing_degree", C.c_int32),
    ]


class UzawaStats(C.Structure):
    _fields_ = [
        ("outer_iterations", C.c_int32), ("inner_iterations", C.c_int32),
        ("inner_solves", C.c_int32), ("fallbacks", C.c_int32),
        ("rel_residual", C.c_double), ("abs_residual", C.c_double), ("div_u", C.c_double),
        ("momentum_residual", C.c_double), ("solve_ms", C.c_double),
        ("kernel_launches", C.c_int64),
        ("fused_launches", C.c_int32), ("fused_iterations", C.c_int32), ("fused_ms", C.c_double),
        ("fused_bytes_per_iteration", C.c_double), ("fused_barriers_per_iteration", C.c_int32),
        ("uzawa_fused", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PicardParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("min_iterations", C.c_int32),
                ("tolerance", C.c_double)]


class PicardStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("residual", C.c_double),
                ("outer_iterations", C.c_int32), ("inner_iterations", C.c_int32),
                ("solve_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LearnParams(C.Structure):
    _fields_ = [("level", C.c_int32), ("n_rhs", C.c_int32), ("iters_per_rhs", C.c_int32),
                ("epochs", C.c_int32), ("lr", C.c_float), ("seed", C.c_int32), ("base", C.c_int32)]


class LearnStats(C.Structure):
    _fields_ = [("samples", C.c_int32), ("loss_first", C.c_float), ("loss_last", C.c_float),
                ("train_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


WEIGHTS_CONSTANT, WEIGHTS_DVC = 0, 1


class Weights(C.Structure):
    _fields_ = [("mode", C.c_int32), ("resolution", C.c_int32 * 3)]


class PcdvcParams(C.Structure):
    _fields_ = [("upper_t", C.c_double), ("lower_t", C.c_double), ("max_splits", C.c_int32),
                ("max_deletions", C.c_int32), ("split_in_interface_cells", C.c_int32),
                ("delete_in_interface_cells", C.c_int32), ("inflow", C.c_int32)]


class PcdvcStats(C.Structure):
    _fields_ = [("points_before", C.c_int64), ("points_after", C.c_int64), ("splits", C.c_int64),
                ("deletions", C.c_int64), ("ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def ptr(a, ctype=C.c_double):
    """Pointer to a contiguous numpy array (None stays NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


# Exported C-ABI symbols with their argtypes; the header declares exactly these.
_P = C.c_void_p
_PD = C.POINTER(C.c_double)
_PI32 = C.POINTER(C.c_int32)
_PU32 = C.POINTER(C.c_uint32)
_PU8 = C.POINTER(C.c_uint8)
ABI_FUNCTIONS = {
    "gg_create": ([C.POINTER(MeshDesc), C.POINTER(_P)], C.c_int),
    "gg_destroy": ([_P], C.c_int),
    "gg_last_error": ([_P], C.c_char_p),
    "gg_version": ([], C.c_char_p),
    "gg_set_velocity_bc": ([_P, C.POINTER(VelocityBC)], C.c_int),
    "gg_set_velocity_bc_nodes": ([_P, _PU8, _PD], C.c_int),
    "gg_set_materials": ([_P, C.c_int32, C.POINTER(Material)], C.c_int),
    "gg_set_points": ([_P, C.c_int64, _PD, _PI32, _PD], C.c_int),
    "gg_set_temperature": ([_P, _PD], C.c_int),
    "gg_set_body_force": ([_P, C.POINTER(BodyForce)], C.c_int),
    "gg_locate": ([_P, _PU32], C.c_int),
    "gg_build_operator": ([_P, C.c_int32, C.c_int32, _PD, _PD], C.c_int),
    "gg_uzawa_solve": ([_P, C.POINTER(UzawaParams), _PD, _PD, C.POINTER(UzawaStats)], C.c_int),
    "gg_picard": ([_P, C.POINTER(PicardParams), C.POINTER(UzawaParams), _PD, _PD,
                   C.POINTER(PicardStats)], C.c_int),
    "gg_advect": ([_P, C.c_double, C.c_int32, _PD, _PD], C.c_int),
    "gg_courant_dt": ([_P, _PD, _PD], C.c_int),
    "gg_get_point_viscosity": ([_P, _PD], C.c_int),
    "gg_get_point_yield": ([_P, _PD, _PU8], C.c_int),
    "gg_get_moments": ([_P, _PD, _PI32], C.c_int),
    "gg_apply_K": ([_P, C.c_int32, _PD, _PD], C.c_int),
    "gg_apply_G": ([_P, _PD, _PD], C.c_int),
    "gg_apply_GT": ([_P, _PD, _PD], C.c_int),
    "gg_get_rhs": ([_P, _PD, _PD], C.c_int),
    "gg_get_diagonals": ([_P, _PD, _PD], C.c_int),
    "gg_time_apply": ([_P, C.c_int32, C.c_int32, _PD], C.c_int),
    "gg_get_coarse_inverse": ([_P, C.POINTER(C.c_int64), C.POINTER(C.c_float), _PD], C.c_int),
    "gg_time_grid_barrier": ([C.c_int32, C.c_int32, _PD], C.c_int),
    "gg_check_grid_barrier_timeout": ([C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "gg_locate_noalloc": ([C.POINTER(MeshDesc), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.POINTER(C.c_int64), C.c_void_p, C.POINTER(C.c_char_p)], C.c_int),
    "gg_solve_batch": ([C.c_int32, C.POINTER(_P), C.POINTER(UzawaParams), C.c_int32, C.POINTER(_PD),
                        C.POINTER(_PD), C.POINTER(UzawaStats), _PI32], C.c_int),
    "gg_set_weights": ([_P, C.POINTER(Weights)], C.c_int),
    "gg_population_control": ([_P, C.POINTER(PcdvcParams), C.POINTER(PcdvcStats)], C.c_int),
    "gg_point_count": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "gg_get_points": ([_P, _PD, _PI32, _PD], C.c_int),
    "gg_get_integration_points": ([_P, _PD, _PD], C.c_int),
    "gg_learned_train": ([_P, C.POINTER(LearnParams), C.POINTER(LearnStats)], C.c_int),
    "gg_learned_weights": ([_P, C.POINTER(C.c_float), _PI32], C.c_int),
    "gg_learned_set_weights": ([_P, C.c_int32, C.POINTER(C.c_float), C.c_int32], C.c_int),
    "gg_learned_eval": ([_P, C.c_int32, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                         C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), _PD, _PI32],
                        C.c_int),
}

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgale_b200.so")
_lib = None


def load_library(path: str = LIB_PATH):
    """Open the CUDA library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"gale_b200 CUDA library not found at {path}; run "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, (argtypes, restype) in ABI_FUNCTIONS.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = restype
    _lib = lib
    return lib
