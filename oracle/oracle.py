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
    "or_set_velocity_bc_nodes": ([_P, _PU8, _PD], C.c_int),
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
    "or_local_to_global": ([C.POINTER(abi.MeshDesc), C.c_int64, _PU32, _PD, _PD], None),
    "od_dvc_cell": ([C.c_int32, _PI32, C.c_int32, _PD, _PD, _PI32], C.c_int),
    "od_dvc_cell_volume": ([C.c_int32, _PI32], C.c_double),
}


class PcdvcParams(C.Structure):
    """od_pcdvc_params (oracle/dvc_oracle.h)."""
    _fields_ = [("upper_t", C.c_double), ("lower_t", C.c_double), ("max_splits", C.c_int32),
                ("max_deletions", C.c_int32), ("split_in_interface_cells", C.c_int32),
                ("delete_in_interface_cells", C.c_int32)]


_SIG["od_pcdvc_cell"] = ([C.c_int32, _PI32, C.POINTER(PcdvcParams), C.c_int32, _PD, _PI32, _PI64, _PI32, _PD, _PD,
                          _PD, _PI32, _PI32, _PI32], C.c_int)


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

    def set_velocity_bc_nodes(self, fixed, values):
        """fixed [nodes] (bit c: component c fixed), values [nodes, dim] node-major."""
        self._bcf = np.ascontiguousarray(fixed, dtype=np.uint8)
        self._bcv = f64(values)
        _check(lib().or_set_velocity_bc_nodes(self.h, ptr(self._bcf, C.c_uint8), ptr(self._bcv)))

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


# ---- A13: discrete-Voronoi weights and population control --------------------------
def dvc_cell(dim, res, xi):
    """Voronoi centroids [n][dim] and weights [n] of one element's points xi [n][dim]."""
    xi = f64(xi).reshape(-1, dim)
    n = xi.shape[0]
    r = np.ascontiguousarray(list(res) + [1] * (3 - len(res)), dtype=np.int32)
    cent = np.zeros((n, dim))
    cnt = np.zeros(n, dtype=np.int32)
    rc = lib().od_dvc_cell(dim, ptr(r, C.c_int32), n, ptr(xi), ptr(cent), ptr(cnt, C.c_int32))
    if rc:
        raise OracleError(rc, "od_dvc_cell")
    return cent, cnt * lib().od_dvc_cell_volume(dim, ptr(r, C.c_int32))


def _cells_of(mesh, coords):
    cell = locate(mesh, coords)
    nel = int(np.prod([mesh.elements[d] for d in range(mesh.dim)]))
    offs = np.zeros(nel + 1, dtype=np.int64)
    order = np.zeros(len(cell), dtype=np.int64)
    lib().or_cell_lists(len(cell), ptr(cell, C.c_uint32), nel, ptr(offs, C.c_int64), ptr(order, C.c_int64))
    xi = np.zeros((len(cell), mesh.dim))
    lib().or_local_coords(C.byref(mesh), len(cell), ptr(f64(coords)), ptr(cell, C.c_uint32), ptr(xi))
    return cell, offs, order, xi


def dvc_weights(mesh, coords, res):
    """DVCWeights on every element: per point (input order) the integration position (the
    centroid of its Voronoi region) and weight (its volume)."""
    dim = mesh.dim
    cell, offs, order, xi = _cells_of(mesh, coords)
    cent = np.zeros((len(cell), dim))
    w = np.zeros(len(cell))
    for e in range(len(offs) - 1):
        idx = order[offs[e]:offs[e + 1]]
        if len(idx):
            c, ww = dvc_cell(dim, res, xi[idx])
            cent[idx], w[idx] = c, ww
    return cent, w


def population_control(mesh, coords, material, plastic_strain, params, res):
    """PCDVC (Inflow off) over all elements in element order, then the new point set:
    points that survive in input order, followed by the new points (element order, then
    their parents' order in the element list), each with its integration position and
    weight from its element's final Voronoi diagram.  Returns a dict."""
    dim = mesh.dim
    coords = f64(coords).reshape(-1, dim)
    material = np.ascontiguousarray(material, dtype=np.int32)
    ps = np.zeros(len(coords)) if plastic_strain is None else f64(plastic_strain)
    cell, offs, order, xi = _cells_of(mesh, coords)
    r = np.ascontiguousarray(list(res) + [1] * (3 - len(res)), dtype=np.int32)
    keep = np.zeros(len(coords), dtype=bool)
    cent = np.zeros((len(coords), dim))
    w = np.zeros(len(coords))
    new_parent, new_cell, new_xi, new_cent, new_w = [], [], [], [], []
    nsplit = ndel = 0
    prm = params
    for e in range(len(offs) - 1):
        idx = order[offs[e]:offs[e + 1]]
        n = len(idx)
        if n == 0:
            continue
        cap = n + prm.max_splits + 1
        src = np.zeros(cap, dtype=np.int32)
        oxi = np.zeros((cap, dim))
        oc = np.zeros((cap, dim))
        ow = np.zeros(cap)
        no, ns, nd = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        exi = np.ascontiguousarray(xi[idx])
        emat = np.ascontiguousarray(material[idx])
        eidx = np.ascontiguousarray(idx, dtype=np.int64)
        rc = lib().od_pcdvc_cell(dim, ptr(r, C.c_int32), C.byref(prm), n, ptr(exi), ptr(emat, C.c_int32),
                                 ptr(eidx, C.c_int64), ptr(src, C.c_int32), ptr(oxi), ptr(oc), ptr(ow),
                                 C.byref(no), C.byref(ns), C.byref(nd))
        if rc:
            raise OracleError(rc, f"od_pcdvc_cell (element {e})")
        nsplit += ns.value
        ndel += nd.value
        news = []
        for k in range(no.value):
            if src[k] >= 0:
                p = idx[src[k]]
                keep[p] = True
                cent[p], w[p] = oc[k], ow[k]
            else:
                news.append((-1 - src[k], k))
        for slot, k in sorted(news):
            new_parent.append(idx[slot])
            new_cell.append(e)
            new_xi.append(oxi[k])
            new_cent.append(oc[k])
            new_w.append(ow[k])
    surv = np.nonzero(keep)[0]
    m = len(new_parent)
    if m:
        nxi = np.ascontiguousarray(np.array(new_xi).reshape(m, dim))
        ncell = np.ascontiguousarray(new_cell, dtype=np.uint32)
        ncoords = np.zeros((m, dim))
        lib().or_local_to_global(C.byref(mesh), m, ptr(ncell, C.c_uint32), ptr(nxi), ptr(ncoords))
        par = np.array(new_parent, dtype=np.int64)
    else:
        ncoords = np.zeros((0, dim))
        par = np.zeros(0, dtype=np.int64)
    return {
        "coords": np.concatenate([coords[surv], ncoords]),
        "material": np.concatenate([material[surv], material[par]]).astype(np.int32),
        "plastic_strain": np.concatenate([ps[surv], ps[par]]),
        "xi": np.concatenate([cent[surv], np.array(new_cent).reshape(m, dim)]),
        "weight": np.concatenate([w[surv], np.array(new_w)]),
        "splits": nsplit, "deletions": ndel,
    }
