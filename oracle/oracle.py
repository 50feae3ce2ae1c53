"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module,
always as the checker or the CPU baseline, never as the product path.  The oracle is
an FP64 C restatement of the reference (see oracle/gale_oracle.c for the per-function
citations); ``oracle/Makefile`` builds ``liboracle``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gale_b200 import abi
from gale_b200.abi import ptr, f64

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libgale_oracle.so")
_lib = None

_P = C.c_void_p
_PD = C.POINTER(C.c_double)
_PI32 = C.POINTER(C.c_int32)
_PI64 = C.POINTER(C.c_int64)
_PU32 = C.POINTER(C.c_uint32)
_PU8 = C.POINTER(C.c_uint8)
_SIG = {
    "or_locate": ([C.POINTER(abi.MeshDesc), C.c_int64, _PD, _PU32], C.c_int64),
    "or_local_coords": ([C.POINTER(abi.MeshDesc), C.c_int64, _PD, _PU32, _PD], None),
    "or_cell_lists": ([C.c_int64, _PU32, C.c_int64, _PI64, _PI64], None),
    "or_create": ([C.POINTER(abi.MeshDesc)], _P),
    "or_destroy": ([_P], None),
    "or_set_threads": ([C.c_int], C.c_int),
    "or_set_velocity_bc": ([_P, C.POINTER(abi.VelocityBC)], C.c_int),
    "or_set_materials": ([_P, C.c_int32, C.POINTER(abi.Material)], C.c_int),
    "or_set_temperature": ([_P, _PD], C.c_int),
    "or_set_body_force": ([_P, C.POINTER(abi.BodyForce)], C.c_int),
    "or_set_points": ([_P, C.c_int64, _PD, _PI32, _PD], C.c_int),
    "or_set_integration_points": ([_P, C.c_int64, _PU32, _PD, _PD, _PI32], C.c_int),
    "or_assemble": ([_P, C.c_int32, _PD, _PD], C.c_int),
    "or_dense_K": ([_P, _PD], C.c_int),
    "or_apply_K": ([_P, _PD, _PD], C.c_int),
    "or_apply_G": ([_P, _PD, _PD], C.c_int),
    "or_apply_GT": ([_P, _PD, _PD], C.c_int),
    "or_get_rhs": ([_P, _PD, _PD], C.c_int),
    "or_get_diagonals": ([_P, _PD, _PD], C.c_int),
    "or_point_viscosity": ([_P, _PD], C.c_int),
    "or_point_yield": ([_P, _PD, _PU8], C.c_int),
    "or_moments": ([_P, _PD, _PI32], C.c_int),
    "or_monomials": ([C.c_int32, _PI32], C.c_int),
    "or_uzawa": ([_P, C.POINTER(abi.UzawaParams), _PD, _PD, C.POINTER(abi.UzawaStats)], C.c_int),
    "or_picard": ([_P, C.POINTER(abi.PicardParams), C.POINTER(abi.UzawaParams), _PD, _PD,
                   C.POINTER(abi.PicardStats)], C.c_int),
    "or_inner_solve": ([_P, _PD, _PD, C.c_double, C.c_int32], C.c_int),
    "or_advect": ([_P, C.c_double, C.c_int32, _PD, _PD], C.c_int),
    "or_courant_dt": ([_P, _PD, _PD], C.c_int),
    "or_last_error": ([], C.c_char_p),
}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        for k, (a, r) in _SIG.items():
            f = getattr(L, k)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle status {code} ({abi.STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


def _check(rc):
    if rc != 0:
        raise OracleError(rc, lib().or_last_error().decode())


def set_threads(n: int) -> int:
    return lib().or_set_threads(int(n))


def locate(mesh: abi.MeshDesc, coords: np.ndarray) -> np.ndarray:
    coords = f64(coords)
    n = coords.shape[0]
    cell = np.empty(n, dtype=np.uint32)
    lib().or_locate(C.byref(mesh), n, ptr(coords), ptr(cell, C.c_uint32))
    return cell


def local_coords(mesh, coords, cell):
    coords = f64(coords)
    xi = np.empty_like(coords)
    lib().or_local_coords(C.byref(mesh), coords.shape[0], ptr(coords),
                          ptr(np.ascontiguousarray(cell, dtype=np.uint32), C.c_uint32), ptr(xi))
    return xi


def monomials(dim: int) -> np.ndarray:
    ex = np.zeros((27, 3), dtype=np.int32)
    n = lib().or_monomials(dim, ptr(ex, C.c_int32))
    return ex[:n]


class OracleProblem:
    """One Stokes problem on the CPU oracle; mirrors gale_b200.StokesProblem."""

    def __init__(self, mesh: abi.MeshDesc):
        self.mesh = mesh
        self.dim = mesh.dim
        self.nel = int(np.prod([mesh.elements[i] for i in range(mesh.dim)]))
        self.nnode = int(np.prod([mesh.elements[i] + 1 for i in range(mesh.dim)]))
        self.h = lib().or_create(C.byref(mesh))
        if not self.h:
            raise OracleError(-1, "or_create")

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_velocity_bc(self, bc):
        _check(lib().or_set_velocity_bc(self.h, C.byref(bc)))

    def set_materials(self, mats):
        arr = (abi.Material * len(mats))(*mats)
        _check(lib().or_set_materials(self.h, len(mats), arr))

    def set_temperature(self, T):
        self._T = f64(T)
        _check(lib().or_set_temperature(self.h, ptr(self._T)))

    def set_body_force(self, bf):
        _check(lib().or_set_body_force(self.h, C.byref(bf)))

    def set_points(self, coords, material=None, plastic_strain=None):
        coords = f64(coords)
        self.np = coords.shape[0]
        mat = None if material is None else np.ascontiguousarray(material, dtype=np.int32)
        ps = f64(plastic_strain)
        _check(lib().or_set_points(self.h, self.np, ptr(coords), ptr(mat, C.c_int32), ptr(ps)))

    def set_integration_points(self, cell, xi, weight, material=None):
        cell = np.ascontiguousarray(cell, dtype=np.uint32)
        xi = f64(xi)
        weight = f64(weight)
        self.np = cell.shape[0]
        mat = None if material is None else np.ascontiguousarray(material, dtype=np.int32)
        _check(lib().or_set_integration_points(self.h, self.np, ptr(cell, C.c_uint32), ptr(xi),
                                               ptr(weight), ptr(mat, C.c_int32)))

    def assemble(self, previous_solution_exists=False, u=None, p=None):
        u = f64(u)
        p = f64(p)
        _check(lib().or_assemble(self.h, int(previous_solution_exists), ptr(u), ptr(p)))

    def dense_K(self):
        nd = self.nnode * self.dim
        K = np.zeros((nd, nd))
        _check(lib().or_dense_K(self.h, ptr(K)))
        return K

    def apply_K(self, x):
        x = f64(x)
        y = np.zeros_like(x)
        _check(lib().or_apply_K(self.h, ptr(x), ptr(y)))
        return y

    def apply_G(self, p):
        p = f64(p)
        y = np.zeros(self.nnode * self.dim)
        _check(lib().or_apply_G(self.h, ptr(p), ptr(y)))
        return y

    def apply_GT(self, u):
        u = f64(u)
        q = np.zeros(self.nel)
        _check(lib().or_apply_GT(self.h, ptr(u), ptr(q)))
        return q

    def rhs(self):
        f = np.zeros(self.nnode * self.dim)
        h = np.zeros(self.nel)
        _check(lib().or_get_rhs(self.h, ptr(f), ptr(h)))
        return f, h

    def diagonals(self):
        kd = np.zeros(self.nnode * self.dim)
        sd = np.zeros(self.nel)
        _check(lib().or_get_diagonals(self.h, ptr(kd), ptr(sd)))
        return kd, sd

    def point_viscosity(self):
        eta = np.zeros(self.np)
        _check(lib().or_point_viscosity(self.h, ptr(eta)))
        return eta

    def point_yield(self):
        inc = np.zeros(self.np)
        y = np.zeros(self.np, dtype=np.uint8)
        _check(lib().or_point_yield(self.h, ptr(inc), ptr(y, C.c_uint8)))
        return inc, y

    def moments(self):
        n = C.c_int32(0)
        _check(lib().or_moments(self.h, None, C.byref(n)))
        m = np.zeros((n.value, self.nel))
        _check(lib().or_moments(self.h, ptr(m), None))
        return m

    def inner_solve(self, b, rtol, maxit=10000):
        b = f64(b)
        x = np.zeros_like(b)
        it = lib().or_inner_solve(self.h, ptr(b), ptr(x), rtol, maxit)
        return x, it

    def uzawa(self, params, p0=None):
        u = np.zeros(self.nnode * self.dim)
        p = np.zeros(self.nel) if p0 is None else f64(p0).copy()
        st = abi.UzawaStats()
        _check(lib().or_uzawa(self.h, C.byref(params), ptr(u), ptr(p), C.byref(st)))
        return u, p, st.as_dict()

    def picard(self, pic, params):
        u = np.zeros(self.nnode * self.dim)
        p = np.zeros(self.nel)
        st = abi.PicardStats()
        _check(lib().or_picard(self.h, C.byref(pic), C.byref(params), ptr(u), ptr(p),
                               C.byref(st)))
        return u, p, st.as_dict()

    def advect(self, dt, u, order=2):
        u = f64(u)
        out = np.zeros((self.np, self.dim))
        _check(lib().or_advect(self.h, dt, order, ptr(u), ptr(out)))
        return out

    def courant_dt(self, u):
        u = f64(u)
        dt = C.c_double(0)
        _check(lib().or_courant_dt(self.h, ptr(u), C.byref(dt)))
        return dt.value
