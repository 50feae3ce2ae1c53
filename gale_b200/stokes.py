"""Host-side mirror of Gale's Stokes component interface over the sm_100a C ABI.

The constructors take the XML parameter names of the reference components, so an
input deck translates field for field:

=====================================  =============================================
reference component (XML ``Type``)      here
=====================================  =============================================
MaterialViscosity / Arrhenius /         ``MaterialViscosity(eta0=…)`` etc. → ``gg_rheology``
FrankKamenetskii / VonMises /
DruckerPrager / Byerlee
StrainWeakening                         ``StrainWeakening(…)``
RheologyMaterial (+ density, alpha)     ``RheologyMaterial([...], density=…, alpha=…)``
WallVC velocityBCs                      ``VelocityBC`` / ``free_slip(dim)``
BuoyancyForceTerm /                     ``BodyForce(gravity=…, gHat=…, rayleighNumber=…)``
ThermalBuoyancyForceTerm
Stokes_SLE_UzawaSolver                  ``UzawaSolver(tolerance=…, maxIterations=…)``
Stokes_SLE (+ Picard)                   ``StokesProblem.solve`` / ``.picard``
SwarmAdvector + TimeIntegrator          ``StokesProblem.advect``
=====================================  =============================================

Errors come back as :class:`GaleError` carrying the C status (the reference aborts
through Journal_Firewall instead).  There is no CPU fallback: constructing a problem
without the CUDA library or a GPU raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .abi import f64, ptr


class GaleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gale_b200 status {code} ({abi.STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


# ---------------------------------------------------------------- rheologies ----
def _rheo(kind, **kw) -> abi.Rheology:
    r = abi.Rheology()
    r.kind = kind
    for k, v in kw.items():
        setattr(r, k, v)
    return r


def MaterialViscosity(eta0: float = 1.0) -> abi.Rheology:
    """Underworld/Rheology/src/MaterialViscosity.cxx:129-149."""
    return _rheo(abi.RHEO_MATERIAL_VISCOSITY, eta0=eta0)


def Arrhenius(eta0=1.0, activationEnergy=0.0, activationVolume=0.0,
              referenceTemperature=1.0) -> abi.Rheology:
    """Underworld/Rheology/src/Arrhenius.cxx:130-220 (XML defaults)."""
    return _rheo(abi.RHEO_ARRHENIUS, eta0=eta0, activation_energy=activationEnergy,
                 activation_volume=activationVolume, reference_temp=referenceTemperature)


def FrankKamenetskii(eta0=1.0, theta=0.0) -> abi.Rheology:
    """Underworld/Rheology/src/FrankKamenetskii.cxx:125-161."""
    return _rheo(abi.RHEO_FRANK_KAMENETSKII, eta0=eta0, theta=theta)


def VonMises(cohesion=0.0, cohesionAfterSoftening=0.0, minimumViscosity=0.0,
             strainRateSoftening=False, strainWeakening=False) -> abi.Rheology:
    """Underworld/Rheology/src/VonMises.cxx:150-289."""
    return _rheo(abi.RHEO_VON_MISES, cohesion=cohesion,
                 cohesion_after_softening=cohesionAfterSoftening,
                 minimum_viscosity=minimumViscosity,
                 strain_rate_softening=int(strainRateSoftening),
                 strain_weakening=int(strainWeakening))


def DruckerPrager(cohesion=0.0, cohesionAfterSoftening=0.0, frictionCoefficient=0.0,
                  frictionCoefficientAfterSoftening=0.0, minimumYieldStress=0.0,
                  minimumViscosity=0.0, maxStrainRate=0.0,
                  strainWeakening=False, boundaryCohesion=0.0, boundaryCohesionAfterSoftening=0.0,
                  boundaryFrictionCoefficient=0.0, boundaryFrictionCoefficientAfterSoftening=0.0,
                  boundaryLeft=False, boundaryRight=False, boundaryBottom=False, boundaryTop=False,
                  boundaryBack=False, boundaryFront=False, HydrostaticTerm=None) -> abi.Rheology:
    """Underworld/Rheology/src/DruckerPrager.cxx:225-490 (XML defaults).  Elements in the
    first or last layer along a wall flagged boundary<Wall> use the boundary cohesion and
    friction (:341-361).  A HydrostaticTerm is refused by the library (GG_ERR_INVALID)."""
    walls = sum(1 << i for i, on in enumerate((boundaryLeft, boundaryRight, boundaryBottom, boundaryTop,
                                               boundaryBack, boundaryFront)) if on)
    return _rheo(abi.RHEO_DRUCKER_PRAGER, cohesion=cohesion,
                 cohesion_after_softening=cohesionAfterSoftening,
                 friction_coefficient=frictionCoefficient,
                 friction_coefficient_after_softening=frictionCoefficientAfterSoftening,
                 minimum_yield_stress=minimumYieldStress, minimum_viscosity=minimumViscosity,
                 max_strain_rate=maxStrainRate, strain_weakening=int(strainWeakening),
                 boundary_cohesion=boundaryCohesion,
                 boundary_cohesion_after_softening=boundaryCohesionAfterSoftening,
                 boundary_friction_coefficient=boundaryFrictionCoefficient,
                 boundary_friction_coefficient_after_softening=boundaryFrictionCoefficientAfterSoftening,
                 boundary_walls=walls, hydrostatic_term=int(HydrostaticTerm is not None))


def Byerlee(cohesion=0.0, depthCoefficient=0.0, minimumViscosity=0.0) -> abi.Rheology:
    """Underworld/Rheology/src/Byerlee.cxx:140-187."""
    return _rheo(abi.RHEO_BYERLEE, cohesion=cohesion, depth_coefficient=depthCoefficient,
                 minimum_viscosity=minimumViscosity)


@dataclass
class StrainWeakening:
    """Underworld/Rheology/src/StrainWeakening.cxx:250-275."""
    initialSofteningStrain: float = 0.0
    finalSofteningStrain: float = float("inf")
    healingRate: float = 0.0


def RheologyMaterial(rheologies: Sequence[abi.Rheology], density: float = 0.0,
                     alpha: float = 0.0,
                     strainWeakening: Optional[StrainWeakening] = None) -> abi.Material:
    """A RheologyMaterial with its rheology list (run in order) and buoyancy data."""
    if len(rheologies) > abi.MAX_RHEOLOGIES:
        raise ValueError("too many rheologies")
    m = abi.Material()
    m.n_rheologies = len(rheologies)
    for i, r in enumerate(rheologies):
        m.rheology[i] = r
    m.density = density
    m.alpha = alpha
    if strainWeakening is not None:
        m.has_strain_weakening = 1
        m.strain_weakening.initial_softening_strain = strainWeakening.initialSofteningStrain
        m.strain_weakening.final_softening_strain = strainWeakening.finalSofteningStrain
        m.strain_weakening.healing_rate = strainWeakening.healingRate
    return m


# ------------------------------------------------------------ BCs / forces ----
WALLS = ("left", "right", "bottom", "top", "back", "front")


def VelocityBC(**walls) -> abi.VelocityBC:
    """WallVC list: ``VelocityBC(left={'vx': 0}, bottom={'vy': 0}, ...)``."""
    bc = abi.VelocityBC()
    for name, comps in walls.items():
        w = WALLS.index(name)
        for cname, val in comps.items():
            c = "xyz".index(cname[-1])
            bc.fixed[w][c] = 1
            bc.value[w][c] = float(val)
    return bc


def free_slip(dim: int) -> abi.VelocityBC:
    """velocityBCs.freeslip.xml: normal velocity zero on every wall."""
    kw = {"left": {"vx": 0}, "right": {"vx": 0}, "bottom": {"vy": 0}, "top": {"vy": 0}}
    if dim == 3:
        kw.update(back={"vz": 0}, front={"vz": 0})
    return VelocityBC(**kw)


def BodyForce(gravity=0.0, gHat=(0.0, -1.0, 0.0), rayleighNumber=0.0) -> abi.BodyForce:
    b = abi.BodyForce()
    b.gravity = gravity
    for i, g in enumerate(gHat):
        b.g_hat[i] = g
    b.rayleigh = rayleighNumber
    return b


def Mesh(dim, elements, minCoord=None, maxCoord=None) -> abi.MeshDesc:
    """elementResI/J/K, minX/… maxX/… of the CartesianGenerator."""
    m = abi.MeshDesc()
    m.dim = dim
    for i in range(3):
        m.elements[i] = int(elements[i]) if i < dim else 1
        m.min[i] = (minCoord[i] if minCoord is not None else 0.0) if i < dim else 0.0
        m.max[i] = (maxCoord[i] if maxCoord is not None else 1.0) if i < dim else 0.0
    return m


def UzawaSolver(tolerance=1e-5, maxIterations=1000, minIterations=1,
                useAbsoluteTolerance=False, preconditioner=True, inner="jacobi",
                precision="fp64", innerRtolFactor=0.1, innerMaxIterations=10000,
                reusePressure=False, recycle=None, smoothingDegree=0) -> abi.UzawaParams:
    """Stokes_SLE_UzawaSolver XML parameters (Stokes_SLE_UzawaSolver.cxx:241-264).
    recycle (default: on for the mixed path) starts each inner solve from β u*_prev;
    smoothingDegree (2..4, 0 = 2) is the multigrid Chebyshev degree of each fine-level sweep;
    coarser levels use min(smoothingDegree, 2)."""
    p = abi.UzawaParams()
    p.tolerance = tolerance
    p.max_iterations = maxIterations
    p.min_iterations = minIterations
    p.use_absolute_tolerance = int(useAbsoluteTolerance)
    p.use_preconditioner = int(preconditioner)
    p.inner = {"jacobi": abi.INNER_JACOBI_CG, "mg": abi.INNER_MG_CG, "learned": abi.INNER_LEARNED_CG,
               "learned_jacobi": abi.INNER_LEARNED_JACOBI_CG}[inner]
    p.precision = {"fp64": abi.PRECISION_FP64, "mixed": abi.PRECISION_MIXED}[precision]
    p.inner_rtol_factor = innerRtolFactor
    p.inner_max_iterations = innerMaxIterations
    p.reuse_pressure = int(reusePressure)
    p.recycle_directions = int(precision == "mixed" if recycle is None else recycle)
    p.smoothing_degree = int(smoothingDegree)
    return p


def Picard(nonLinearMaxIterations=20, nonLinearTolerance=1e-5,
           nonLinearMinIterations=1) -> abi.PicardParams:
    p = abi.PicardParams()
    p.max_iterations = nonLinearMaxIterations
    p.min_iterations = nonLinearMinIterations
    p.tolerance = nonLinearTolerance
    return p


# -------------------------------------------------------------------- problem ----
class StokesProblem:
    """One PIC Q1-P0 Stokes problem resident on the GPU (one C-ABI handle)."""

    def __init__(self, mesh: abi.MeshDesc):
        self.lib = abi.load_library()
        self.mesh = mesh
        self.dim = mesh.dim
        self.nel = int(np.prod([mesh.elements[i] for i in range(mesh.dim)]))
        self.nnode = int(np.prod([mesh.elements[i] + 1 for i in range(mesh.dim)]))
        h = C.c_void_p()
        rc = self.lib.gg_create(C.byref(mesh), C.byref(h))
        if rc != 0:
            raise GaleError(rc, "gg_create")
        self.h = h
        self.np = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.gg_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise GaleError(rc, self.lib.gg_last_error(self.h).decode())

    # inputs
    def set_velocity_bc(self, bc):
        self._check(self.lib.gg_set_velocity_bc(self.h, C.byref(bc)))

    def set_velocity_bc_nodes(self, fixed, values):
        """Per-node velocity BCs (a condition function evaluated at the nodes): fixed
        [nodes] with bit c = component c fixed, values [nodes, dim] node-major."""
        self._bcf = np.ascontiguousarray(fixed, dtype=np.uint8)
        self._bcv = f64(values)
        self._check(self.lib.gg_set_velocity_bc_nodes(self.h, ptr(self._bcf, C.c_uint8), ptr(self._bcv)))

    def set_materials(self, mats: List[abi.Material]):
        arr = (abi.Material * len(mats))(*mats)
        self._check(self.lib.gg_set_materials(self.h, len(mats), arr))

    def set_points(self, coords, material=None, plastic_strain=None):
        coords = f64(coords)
        self.np = coords.shape[0]
        self._mat = None if material is None else np.ascontiguousarray(material, dtype=np.int32)
        self._ps = f64(plastic_strain)
        self._check(self.lib.gg_set_points(self.h, self.np, ptr(coords), ptr(self._mat, C.c_int32),
                                           ptr(self._ps)))

    def set_temperature(self, T):
        self._T = f64(T)
        self._check(self.lib.gg_set_temperature(self.h, ptr(self._T)))

    def set_body_force(self, bf):
        self._check(self.lib.gg_set_body_force(self.h, C.byref(bf)))

    # integration weights and population control (DVCWeights / PCDVC)
    def set_weights(self, mode="constant", resolution=10):
        """mode "constant" (ConstantWeights) or "dvc" (DVCWeights with `resolution` cells
        per element axis, an int or a per-axis sequence); call locate() afterwards."""
        w = abi.Weights()
        w.mode = {"constant": abi.WEIGHTS_CONSTANT, "dvc": abi.WEIGHTS_DVC}[mode]
        res = [resolution] * 3 if np.isscalar(resolution) else list(resolution) + [1] * (3 - len(resolution))
        for d in range(3):
            w.resolution[d] = int(res[d])
        self._check(self.lib.gg_set_weights(self.h, C.byref(w)))

    def population_control(self, upperT=25.0, lowerT=0.6, maxSplits=3, maxDeletions=2,
                           splitInInterfaceCells=False, deleteInInterfaceCells=False, Inflow=False):
        """PCDVC with the reference's XML parameter names (PCDVC.cxx:233-276 defaults)."""
        p = abi.PcdvcParams()
        p.upper_t, p.lower_t = upperT, lowerT
        p.max_splits, p.max_deletions = maxSplits, maxDeletions
        p.split_in_interface_cells = int(splitInInterfaceCells)
        p.delete_in_interface_cells = int(deleteInInterfaceCells)
        p.inflow = int(Inflow)
        st = abi.PcdvcStats()
        self._check(self.lib.gg_population_control(self.h, C.byref(p), C.byref(st)))
        self.np = st.points_after
        return st.as_dict()

    def points(self):
        n = C.c_int64(0)
        self._check(self.lib.gg_point_count(self.h, C.byref(n)))
        x = np.zeros((n.value, self.dim))
        m = np.zeros(n.value, dtype=np.int32)
        ps = np.zeros(n.value)
        self._check(self.lib.gg_get_points(self.h, ptr(x), ptr(m, C.c_int32), ptr(ps)))
        return x, m, ps

    def integration_points(self):
        n = C.c_int64(0)
        self._check(self.lib.gg_point_count(self.h, C.byref(n)))
        xi = np.zeros((n.value, self.dim))
        w = np.zeros(n.value)
        self._check(self.lib.gg_get_integration_points(self.h, ptr(xi), ptr(w)))
        return xi, w

    # pipeline
    def locate(self) -> np.ndarray:
        cell = np.empty(self.np, dtype=np.uint32)
        self._check(self.lib.gg_locate(self.h, ptr(cell, C.c_uint32)))
        return cell

    def build_operator(self, precision="fp64", previous_solution=None):
        prec = {"fp64": abi.PRECISION_FP64, "mixed": abi.PRECISION_MIXED}[precision]
        if previous_solution is None:
            self._check(self.lib.gg_build_operator(self.h, prec, 0, None, None))
        else:
            u, p = (f64(v) for v in previous_solution)
            self._check(self.lib.gg_build_operator(self.h, prec, 1, ptr(u), ptr(p)))

    def solve(self, params: abi.UzawaParams, p0=None):
        u = np.zeros(self.nnode * self.dim)
        p = np.zeros(self.nel) if p0 is None else f64(p0).copy()
        st = abi.UzawaStats()
        rc = self.lib.gg_uzawa_solve(self.h, C.byref(params), ptr(u), ptr(p), C.byref(st))
        if rc != 0:
            err = GaleError(rc, self.lib.gg_last_error(self.h).decode())
            err.stats = st.as_dict()  # how far the solve got
            raise err
        return u, p, st.as_dict()

    def picard(self, picard: abi.PicardParams, params: abi.UzawaParams):
        u = np.zeros(self.nnode * self.dim)
        p = np.zeros(self.nel)
        st = abi.PicardStats()
        self._check(self.lib.gg_picard(self.h, C.byref(picard), C.byref(params), ptr(u), ptr(p),
                                       C.byref(st)))
        return u, p, st.as_dict()

    def advect(self, dt, u=None, order=2):
        out = np.zeros((self.np, self.dim))
        uu = f64(u)
        self._check(self.lib.gg_advect(self.h, dt, order, ptr(uu), ptr(out)))
        return out

    def courant_dt(self, u):
        dt = C.c_double(0)
        self._check(self.lib.gg_courant_dt(self.h, ptr(f64(u)), C.byref(dt)))
        return dt.value

    @staticmethod
    def solve_batch(problems, params: abi.UzawaParams, workers: int = 16):
        """locate → build → Uzawa for every problem (inputs set), `workers` host threads
        feeding one GPU.  Returns [(u, p, stats)] and raises on the first failure."""
        n = len(problems)
        lib = problems[0].lib
        hs = (C.c_void_p * n)(*[pr.h for pr in problems])
        us = [np.zeros(pr.nnode * pr.dim) for pr in problems]
        ps = [np.zeros(pr.nel) for pr in problems]
        up = (C.POINTER(C.c_double) * n)(*[ptr(u) for u in us])
        pp = (C.POINTER(C.c_double) * n)(*[ptr(p) for p in ps])
        st = (abi.UzawaStats * n)()
        status = np.zeros(n, dtype=np.int32)
        rc = lib.gg_solve_batch(n, hs, C.byref(params), workers, up, pp, st, ptr(status, C.c_int32))
        if rc != 0:
            bad = int(np.flatnonzero(status)[0])
            raise GaleError(rc, f"problem {bad}: " + lib.gg_last_error(problems[bad].h).decode())
        return [(us[i], ps[i], st[i].as_dict()) for i in range(n)]

    # learned coarse correction
    def train_learned(self, level=2, n_rhs=4, iters_per_rhs=6, epochs=60, lr=2e-3, seed=1, base="multigrid"):
        """Train the coarse-correction network on pairs the solver generates for the current
        operator; base "multigrid" (for inner="learned") or "jacobi" (inner="learned_jacobi")
        is the preconditioner whose leftover error it learns to correct."""
        p = abi.LearnParams(level, n_rhs, iters_per_rhs, epochs, lr, seed,
                            {"multigrid": abi.LEARN_BASE_MULTIGRID, "jacobi": abi.LEARN_BASE_JACOBI}[base])
        st = abi.LearnStats()
        self._check(self.lib.gg_learned_train(self.h, C.byref(p), C.byref(st)))
        return st.as_dict()

    def learned_param_count(self):
        n = C.c_int32(0)
        self._check(self.lib.gg_learned_weights(self.h, None, C.byref(n)))
        return n.value

    def learned_weights(self):
        n = C.c_int32(0)
        self._check(self.lib.gg_learned_weights(self.h, None, C.byref(n)))
        w = np.zeros(n.value, dtype=np.float32)
        self._check(self.lib.gg_learned_weights(self.h, ptr(w, C.c_float), None))
        return w

    def set_learned_weights(self, w, level=2):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self.lib.gg_learned_set_weights(self.h, level, ptr(w, C.c_float), w.size))

    def learned_eval(self, inputs, targets, weights, level=2):
        """Forward + backward of a batch (inputs [B][1+dim][N], targets [B][dim][N])."""
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        y = np.zeros_like(t)
        g = np.zeros_like(w)
        loss = C.c_double(0)
        nodes = C.c_int32(x.shape[2])  # checked against the level before the buffers are used
        self._check(self.lib.gg_learned_eval(self.h, level, x.shape[0], ptr(x, C.c_float), ptr(t, C.c_float),
                                             ptr(w, C.c_float), ptr(y, C.c_float), ptr(g, C.c_float),
                                             C.byref(loss), C.byref(nodes)))
        return y, g, loss.value

    # diagnostics / operator access
    def point_viscosity(self):
        eta = np.zeros(self.np)
        self._check(self.lib.gg_get_point_viscosity(self.h, ptr(eta)))
        return eta

    def point_yield(self):
        inc = np.zeros(self.np)
        y = np.zeros(self.np, dtype=np.uint8)
        self._check(self.lib.gg_get_point_yield(self.h, ptr(inc), ptr(y, C.c_uint8)))
        return inc, y

    def moments(self):
        n = C.c_int32(0)
        self._check(self.lib.gg_get_moments(self.h, None, C.byref(n)))
        m = np.zeros((n.value, self.nel))
        self._check(self.lib.gg_get_moments(self.h, ptr(m), None))
        return m

    def apply_K(self, x, precision="fp64"):
        prec = {"fp64": abi.PRECISION_FP64, "mixed": abi.PRECISION_MIXED}[precision]
        x = f64(x)
        y = np.zeros_like(x)
        self._check(self.lib.gg_apply_K(self.h, prec, ptr(x), ptr(y)))
        return y

    def apply_G(self, p):
        y = np.zeros(self.nnode * self.dim)
        self._check(self.lib.gg_apply_G(self.h, ptr(f64(p)), ptr(y)))
        return y

    def apply_GT(self, u):
        q = np.zeros(self.nel)
        self._check(self.lib.gg_apply_GT(self.h, ptr(f64(u)), ptr(q)))
        return q

    def rhs(self):
        f = np.zeros(self.nnode * self.dim)
        hv = np.zeros(self.nel)
        self._check(self.lib.gg_get_rhs(self.h, ptr(f), ptr(hv)))
        return f, hv

    def diagonals(self):
        kd = np.zeros(self.nnode * self.dim)
        sd = np.zeros(self.nel)
        self._check(self.lib.gg_get_diagonals(self.h, ptr(kd), ptr(sd)))
        return kd, sd
