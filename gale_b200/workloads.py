"""Seeded synthetic inputs for the Stokes configurations this library is measured on.

The reference measures nothing on public datasets for this path; these generators
stand in for its XML input decks with the shapes, sizes and value distributions of
each configuration.  Every workload is deterministic for a given seed.

* ``sinker_2d``      2D Q1-P0 sinker, 64×64, 20 points per element, free slip
* ``creep_3d``       3D temperature-dependent creep, 64³, 27 points per element
* ``extension_2d``   2D viscoplastic extension, 256×64 on [0,4]×[0,1], 40 per element
* ``batch_sinkers``  uneven batch of 2D sinkers (n ∈ {32,48,64,96,128})
* ``subduction_3d``  3D slab, 128×128×64, 27 per element
* ``viscous_suite``  the 10×10 Gauss-swarm assembly of the reference's ViscousSuite
* ``lid_driven_pic2d`` the reference's LidDrivenPIC2D regression model (20×20, PCDVC, 10 steps)
* ``rayleigh_taylor_benchmark`` the reference's RayleighTaylorBenchmark regression model (64×64)
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, List, Optional

import numpy as np

from . import abi
from .stokes import (Arrhenius, BodyForce, Byerlee, DruckerPrager, FrankKamenetskii, MaterialViscosity,
                     Mesh, RheologyMaterial, StrainWeakening, UzawaSolver, VelocityBC, VonMises, free_slip,
                     Picard)


@dataclass
class Workload:
    name: str
    mesh: abi.MeshDesc
    bc: abi.VelocityBC
    materials: List[abi.Material]
    force: abi.BodyForce
    coords: np.ndarray
    material: np.ndarray
    plastic_strain: Optional[np.ndarray] = None
    temperature: Optional[np.ndarray] = None
    uzawa: Any = None
    picard: Any = None
    meta: dict = field(default_factory=dict)
    bc_nodes: Any = None  # (fixed [nodes] uint8, values [nodes, dim]) when BCs are functions

    @property
    def dim(self):
        return self.mesh.dim

    @property
    def nel(self):
        return int(np.prod([self.mesh.elements[i] for i in range(self.dim)]))

    @property
    def nnode(self):
        return int(np.prod([self.mesh.elements[i] + 1 for i in range(self.dim)]))

    def apply(self, prob):
        """Load the inputs into a StokesProblem (GPU) or an oracle problem (CPU)."""
        if self.bc_nodes is not None:
            prob.set_velocity_bc_nodes(*self.bc_nodes)
        else:
            prob.set_velocity_bc(self.bc)
        prob.set_materials(self.materials)
        prob.set_body_force(self.force)
        if self.temperature is not None:
            prob.set_temperature(self.temperature)
        prob.set_points(self.coords, self.material, self.plastic_strain)
        return prob


def vertex_coords(mesh: abi.MeshDesc, d: int) -> np.ndarray:
    """CartesianGenerator_CalcGeom vertex coordinates along axis d."""
    n = mesh.elements[d]
    i = np.arange(n + 1, dtype=np.float64)
    x = mesh.min[d] + (i / n) * (mesh.max[d] - mesh.min[d])
    x[0] = mesh.min[d]
    x[-1] = mesh.max[d]
    return x


def node_coords(mesh: abi.MeshDesc) -> np.ndarray:
    """[nnode, dim] coordinates, x fastest."""
    axes = [vertex_coords(mesh, d) for d in range(mesh.dim)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]
    return np.stack([g.reshape(-1) for g in grids], axis=1)


def random_points(mesh: abi.MeshDesc, ppc: int, rng: np.random.Generator, shuffle=True):
    """ppc points per element at uniform-random local coordinates ξ ∈ (-1,1)^dim."""
    dim = mesh.dim
    nel_axes = [mesh.elements[d] for d in range(dim)]
    nel = int(np.prod(nel_axes))
    e = np.repeat(np.arange(nel), ppc)
    xi = rng.uniform(-1.0, 1.0, size=(nel * ppc, dim))
    coords = np.empty((nel * ppc, dim))
    rem = e.copy()
    for d in range(dim):
        idx = rem % nel_axes[d]
        rem //= nel_axes[d]
        v = vertex_coords(mesh, d)
        lo, hi = v[idx], v[idx + 1]
        coords[:, d] = lo + 0.5 * (xi[:, d] + 1.0) * (hi - lo)
    if shuffle:
        perm = rng.permutation(nel * ppc)
        coords = coords[perm]
    return np.ascontiguousarray(coords)


def sinker_2d(n=64, ppc=20, seed=13, eta_inclusion=100.0, rho_inclusion=1.01, radius=0.1,
              centre=(0.5, 0.75), tolerance=1e-5) -> Workload:
    """2D Q1-P0 Stokes sinker on the unit square with free-slip walls: a circular
    inclusion (η=100, ρ=1.01) in a matrix (η=1, ρ=1), gravity −y, constant weights."""
    rng = np.random.default_rng(seed)
    mesh = Mesh(2, (n, n), (0.0, 0.0), (1.0, 1.0))
    coords = random_points(mesh, ppc, rng)
    r2 = (coords[:, 0] - centre[0]) ** 2 + (coords[:, 1] - centre[1]) ** 2
    material = (r2 < radius * radius).astype(np.int32)
    mats = [RheologyMaterial([MaterialViscosity(1.0)], density=1.0),
            RheologyMaterial([MaterialViscosity(eta_inclusion)], density=rho_inclusion)]
    return Workload("sinker_2d", mesh, free_slip(2), mats, BodyForce(gravity=1.0), coords, material,
                    uzawa=UzawaSolver(tolerance=tolerance), meta={"n": n, "ppc": ppc, "seed": seed})


def creep_3d(n=64, ppc=27, seed=2024, noise=0.05, theta=9.21, rayleigh=1e6, tolerance=1e-6) -> Workload:
    """3D temperature-dependent creep in a free-slip box: T = (1 − y) + N(0, σ=0.05) at the
    nodes (y vertical), η = exp(θ(0.5 − T)) (FrankKamenetskii with η0 = e^{θ/2}), thermal
    buoyancy f_y = Ra·T with Ra = 1e6."""
    rng = np.random.default_rng(seed)
    mesh = Mesh(3, (n, n, n), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    coords = random_points(mesh, ppc, rng)
    nodes = node_coords(mesh)
    T = (1.0 - nodes[:, 1]) + rng.normal(0.0, noise, size=nodes.shape[0])
    mats = [RheologyMaterial([FrankKamenetskii(eta0=float(np.exp(0.5 * theta)), theta=theta)])]
    material = np.zeros(coords.shape[0], dtype=np.int32)
    return Workload("creep_3d", mesh, free_slip(3), mats, BodyForce(rayleighNumber=rayleigh), coords,
                    material, temperature=np.ascontiguousarray(T), uzawa=UzawaSolver(tolerance=tolerance),
                    meta={"n": n, "ppc": ppc, "seed": seed})


def velic_solcx(n=64, ppc=20, eta_a=100.0, eta_b=1.0, xc=0.5, nz=2, nx=1, tolerance=1e-5) -> Workload:
    """Underworld's Velic solCx benchmark (testVelicSolCx.xml, Analytic plugin
    Underworld/SysTest/AnalyticPlugins/Velic_solCx): unit square, free-slip walls, a viscosity
    step at x = xc (η_A = 100 left, η_B = 1 right, two MaterialViscosity materials assigned
    by point position), driven by the thermal buoyancy f_y = Ra·T with Ra = 1 and the nodal
    temperature T = sin(n_z π y) cos(n_x π x) (StandardConditionFunctions' VelicTemperatureIC,
    wavenumberY = 2, wavenumberX = 1).  Points and weights as the deck's PIC components
    (PICellerator/Apps/PIC_Components/MaterialPointSwarm.xml): SpaceFillerParticleLayout
    with 20 points per element, PCDVC weights at resolution 10 (lowerT 0.6, upperT 25,
    3 splits, 3 deletions)."""
    mesh = Mesh(2, (n, n), (0.0, 0.0), (1.0, 1.0))
    from .layouts import space_filler
    coords = space_filler(mesh, ppc)
    material = (coords[:, 0] >= xc).astype(np.int32)
    nodes = node_coords(mesh)
    T = np.sin(nz * np.pi * nodes[:, 1]) * np.cos(nx * np.pi * nodes[:, 0])
    mats = [RheologyMaterial([MaterialViscosity(eta_a)]), RheologyMaterial([MaterialViscosity(eta_b)])]
    return Workload("velic_solcx", mesh, free_slip(2), mats, BodyForce(rayleighNumber=1.0), coords, material,
                    temperature=np.ascontiguousarray(T), uzawa=UzawaSolver(tolerance=tolerance),
                    meta={"n": n, "ppc": ppc, "eta_a": eta_a, "eta_b": eta_b, "xc": xc, "nz": nz, "nx": nx,
                          "weights_resolution": 10,
                          "pcdvc": dict(upperT=25.0, lowerT=0.6, maxSplits=3, maxDeletions=3)})


def extension_2d(nx=256, ny=64, ppc=40, seed=7, width=4.0, picard_its=20, tolerance=1e-5) -> Workload:
    """2D viscoplastic extension on [0,4]×[0,1] (domain assumed: square elements).
    Layers: mantle y<0.5 (η=1), lower crust 0.5≤y<0.75 (η=1e2), upper crust y≥0.75
    (η=1e3 + Drucker-Prager C=1, μ=0.6, cohesion softening to 0.1 over plastic strain
    0.5, initial plastic strain U(0,0.1)).  vx = −1 / +1 on the left / right walls, vy = 0
    at the bottom, free top; gravity −y with unit density."""
    rng = np.random.default_rng(seed)
    mesh = Mesh(2, (nx, ny), (0.0, 0.0), (width, 1.0))
    coords = random_points(mesh, ppc, rng)
    y = coords[:, 1]
    material = np.where(y >= 0.75, 2, np.where(y >= 0.5, 1, 0)).astype(np.int32)
    ps = np.where(material == 2, rng.uniform(0.0, 0.1, size=y.shape[0]), 0.0)
    sw = StrainWeakening(initialSofteningStrain=0.0, finalSofteningStrain=0.5)
    mats = [RheologyMaterial([MaterialViscosity(1.0)], density=1.0),
            RheologyMaterial([MaterialViscosity(1e2)], density=1.0),
            RheologyMaterial([MaterialViscosity(1e3),
                              DruckerPrager(cohesion=1.0, cohesionAfterSoftening=0.1,
                                            frictionCoefficient=0.6,
                                            frictionCoefficientAfterSoftening=0.6,
                                            strainWeakening=True)],
                             density=1.0, strainWeakening=sw)]
    bc = VelocityBC(left={"vx": -1.0}, right={"vx": 1.0}, bottom={"vy": 0.0})
    return Workload("extension_2d", mesh, bc, mats, BodyForce(gravity=1.0), coords, material,
                    plastic_strain=np.ascontiguousarray(ps), uzawa=UzawaSolver(tolerance=tolerance),
                    picard=Picard(nonLinearMaxIterations=picard_its, nonLinearTolerance=1e-5),
                    meta={"nx": nx, "ny": ny, "ppc": ppc, "seed": seed})


def batch_sinkers(count=512, ppc=20, seed=99, sizes=(32, 48, 64, 96, 128)) -> List[Workload]:
    """Uneven batch of 2D sinkers: n per axis uniform from `sizes`, inclusion viscosity
    contrast log-uniform in [1, 1e4], radius uniform in [0.05, 0.2]."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        n = int(rng.choice(sizes))
        eta = float(10 ** rng.uniform(0.0, 4.0))
        r = float(rng.uniform(0.05, 0.2))
        w = sinker_2d(n=n, ppc=ppc, seed=int(rng.integers(1 << 30)), eta_inclusion=eta, radius=r)
        w.name = f"sinker_{b}"
        out.append(w)
    return out


def subduction_3d(nx=128, ny=64, nz=128, ppc=27, seed=5, tolerance=1e-6) -> Workload:
    """3D subduction-like model on [0,2]×[0,1]×[0,2] (y vertical): a slab (η=1e4, Δρ=0.01)
    dipping at 45° through an η=1 mantle, with a weak η=1e-2 channel on its top surface,
    free-slip walls, gravity −y."""
    rng = np.random.default_rng(seed)
    mesh = Mesh(3, (nx, ny, nz), (0.0, 0.0, 0.0), (2.0, 1.0, 2.0))
    coords = random_points(mesh, ppc, rng)
    x, y = coords[:, 0], coords[:, 1]
    # signed distance from the slab's top surface: plane through (0.8, 1.0) dipping 45°
    d = ((x - 0.8) + (y - 1.0)) / np.sqrt(2.0)
    slab = (d <= 0.0) & (d > -0.1) & (y > 0.3)
    channel = (d > 0.0) & (d <= 0.02) & (y > 0.3)
    material = np.where(slab, 1, np.where(channel, 2, 0)).astype(np.int32)
    mats = [RheologyMaterial([MaterialViscosity(1.0)], density=1.0),
            RheologyMaterial([MaterialViscosity(1e4)], density=1.01),
            RheologyMaterial([MaterialViscosity(1e-2)], density=1.0)]
    return Workload("subduction_3d", mesh, free_slip(3), mats, BodyForce(gravity=1.0), coords, material,
                    uzawa=UzawaSolver(tolerance=tolerance), meta={"ppc": ppc, "seed": seed})


def partial_lid_top_layer(mesh: abi.MeshDesc, x: np.ndarray) -> np.ndarray:
    """StgFEM_StandardConditionFunctions_PartialLid_TopLayer (StgFEM/plugins/
    StandardConditionFunctions/StandardConditionFunctions.cxx:547-568): 1 where
    min + margin < x < max − margin, else 0, margin = 1.1 × the minimum element separation."""
    sep = min((mesh.max[d] - mesh.min[d]) / mesh.elements[d] for d in range(mesh.dim))
    margin = sep * 1.1
    return ((x < mesh.max[0] - margin) & (x > mesh.min[0] + margin)).astype(np.float64)


def lid_driven_pic2d() -> Workload:
    """PICellerator's regression model LidDrivenPIC2D (PICellerator/SysTest/RegressionTests/
    LidDrivenPIC2D.xml with lidDrivenVelocityBCs.xml and the PIC_Components it includes):
    2D unit square, 20×20 Q1-P0 elements, one material of viscosity 1
    (IsoviscousStressTensorTerm, no body force), 36 points per cell from
    SpaceFillerParticleLayout, PCDVC weights (resolution 10, lowerT 0.6, upperT 25,
    maxDeletions 3, maxSplits 3), Uzawa tolerance 1e-5 / maxIterations 5000, RK2 advection,
    10 time steps.  BCs: vy = 0 on the bottom, vx = 0 on the left and right walls,
    vx = PartialLid_TopLayer(x) and vy = 0 on the top."""
    mesh = Mesh(2, (20, 20), (0.0, 0.0), (1.0, 1.0))
    from .layouts import space_filler
    coords = space_filler(mesh, 36)
    nodes = node_coords(mesh)
    nx = mesh.elements[0] + 1
    ix = np.arange(nodes.shape[0]) % nx
    iy = np.arange(nodes.shape[0]) // nx
    fixed = np.zeros(nodes.shape[0], dtype=np.uint8)
    values = np.zeros((nodes.shape[0], 2))
    fixed[iy == 0] |= 2                         # bottom: vy
    fixed[(ix == 0) | (ix == nx - 1)] |= 1      # left, right: vx
    top = iy == mesh.elements[1]
    fixed[top] |= 3                             # top: vx (function), vy
    values[top, 0] = partial_lid_top_layer(mesh, nodes[top, 0])
    mats = [RheologyMaterial([MaterialViscosity(1.0)])]
    return Workload("lid_driven_pic2d", mesh, abi.VelocityBC(), mats, BodyForce(), coords,
                    np.zeros(coords.shape[0], dtype=np.int32),
                    uzawa=UzawaSolver(tolerance=1e-5, maxIterations=5000),
                    bc_nodes=(fixed, values),
                    meta={"steps": 10, "order": 2, "weights_resolution": 10,
                          "pcdvc": dict(upperT=25.0, lowerT=0.6, maxSplits=3, maxDeletions=3)})


def below_cosine_plane(coords: np.ndarray, offset=0.5, amplitude=0.1, wavelength=2 * np.pi,
                       phase=0.0) -> np.ndarray:
    """Stg_Shape BelowCosinePlane (StgDomain/Shape/src/BelowCosinePlane.cxx:196-213) with no
    centre or rotation: inside where y < offset + amplitude·cos(2πx / wavelength + phase)."""
    x, y = coords[:, 0], coords[:, 1]
    return y < offset + amplitude * np.cos((2 * np.pi * x / wavelength) + phase)


def rayleigh_taylor_benchmark() -> Workload:
    """Underworld's regression model RayleighTaylorBenchmark (Underworld/SysTest/
    RegressionTests/RayleighTaylorBenchmark.xml on BaseApps/RayleighTaylor.xml and
    LidDrivenPIC.xml; van Keken et al. 1997): 64×64 Q1-P0 elements on [0, 0.9142]×[0, 1],
    a light layer (density 0, viscosity 1) below y = 0.2 + 0.02 cos(2πx/1.8284) under a
    background of density 1 and viscosity 1, gravity 1 (BuoyancyForceTerm), free-slip sides
    and no-slip top and bottom, 20 points per cell from SpaceFillerParticleLayout, PCDVC
    weights (resolution 10, lowerT 0.6, upperT 25, maxDeletions 3, maxSplits 3), Uzawa
    tolerance 1e-5, RK2 advection.  Materials are set by shape in material order (the light
    layer, defined second, wins where both shapes hold)."""
    mesh = Mesh(2, (64, 64), (0.0, 0.0), (0.9142, 1.0))
    from .layouts import space_filler
    coords = space_filler(mesh, 20)
    material = below_cosine_plane(coords, offset=0.2, amplitude=0.02, wavelength=1.8284,
                                  phase=0.0).astype(np.int32)
    mats = [RheologyMaterial([MaterialViscosity(1.0)], density=1.0),
            RheologyMaterial([MaterialViscosity(1.0)], density=0.0)]
    bc = VelocityBC(bottom={"vx": 0, "vy": 0}, top={"vx": 0, "vy": 0}, left={"vx": 0}, right={"vx": 0})
    return Workload("rayleigh_taylor_benchmark", mesh, bc, mats, BodyForce(gravity=1.0), coords, material,
                    uzawa=UzawaSolver(tolerance=1e-5, maxIterations=5000),
                    meta={"steps": 10, "order": 2, "weights_resolution": 10,
                          "pcdvc": dict(upperT=25.0, lowerT=0.6, maxSplits=3, maxDeletions=3)})


def viscous_suite(rheology: str):
    """Inputs of the reference's ViscousSuite golden-matrix tests
    (Underworld/Rheology/tests/input/test{MaterialViscosity,Arrhenius,FrankKamenetskii}2D.xml):
    10×10 elements on the unit square, a 2×2 Gauss swarm with unit weights, no velocity
    BCs, nodal temperature from LinearWithSinusoidalPerturbation
    (StgFEM/plugins/StandardConditionFunctions/StandardConditionFunctions.cxx:714-760)."""
    mesh = Mesh(2, (10, 10), (0.0, 0.0), (1.0, 1.0))
    g = 1.0 / np.sqrt(3.0)
    nel = 100
    cell = np.repeat(np.arange(nel, dtype=np.uint32), 4)
    q = np.tile(np.arange(4), nel)
    xi = np.stack([np.where(q & 1, g, -g), np.where(q & 2, g, -g)], axis=1)
    w = np.ones(nel * 4)
    nodes = node_coords(mesh)
    # topLayerBC=0, bottomLayerBC=1, amplitude 0.1, wave numbers 1
    rel_y = nodes[:, 1]
    T = 0.0 + 1.0 * (1.0 - rel_y) + 0.1 * (np.cos(np.pi * nodes[:, 0]) * np.sin(np.pi * rel_y))
    rheo = {"MaterialViscosity": MaterialViscosity(1.0),
            "Arrhenius": Arrhenius(eta0=1.0e-6, activationEnergy=27.63102112),
            "FrankKamenetskii": FrankKamenetskii(eta0=1.0e6, theta=13.815510558)}[rheology]
    return mesh, cell, xi, w, T, [RheologyMaterial([rheo])]


def gauss_points(mesh: abi.MeshDesc, per_dim=2) -> np.ndarray:
    """GaussParticleLayout (StgDomain/Swarm/src/GaussParticleLayout.cxx:175-180, default two
    points per axis): the Gauss–Legendre abscissae of every element, element by element,
    x fastest inside an element, mapped to global coordinates."""
    if per_dim != 2:
        raise ValueError("two Gauss points per axis only")
    g = 1.0 / np.sqrt(3.0)
    dim = mesh.dim
    n = [mesh.elements[d] for d in range(dim)]
    nel = int(np.prod(n))
    e = np.repeat(np.arange(nel), 2 ** dim)
    q = np.tile(np.arange(2 ** dim), nel)
    idx = [e % n[0], (e // n[0]) % n[1]] + ([e // (n[0] * n[1])] if dim == 3 else [])
    coords = np.empty((nel * 2 ** dim, dim))
    for d in range(dim):
        v = vertex_coords(mesh, d)
        lo, hi = v[idx[d]], v[idx[d] + 1]
        xi = np.where((q >> d) & 1, g, -g)
        coords[:, d] = lo + 0.5 * (xi + 1.0) * (hi - lo)
    return np.ascontiguousarray(coords)


def yield_criterion_2d(kind: str, width=3.0, height=1.0) -> Workload:
    """The model of the reference's yielding suites (Underworld/Rheology/tests/input/
    testYieldCriterion.xml with testVonMisesYieldCriterion.xml or
    testByerleeYieldCriterion.xml): 30×10 elements on [0, width]×[0, height], one material
    of MaterialViscosity η = 3.4 followed by the yield rheology, a 2×2 Gauss particle layout,
    Uzawa tolerance 1e-4 (VonMises deck) or 1e-5, and the IncompressibleExtensionBC
    velocities: vx = +0.5 on the left wall and −0.5 on the right, vy = 0 on the bottom and
    vy = height·(0.5 − (−0.5))/width on the top (Underworld/plugins/IncompressibleExtensionBC/
    IncompressibleExtensionBC.cxx GetTopWallVelocity / GetBottomWallVelocity with
    constantHeight 0), a pure-shear shortening whose stress invariant is 2·3.4/width.
    VonMises: cohesion 3.0222222 (the whole box yields once width < 2.25); Byerlee: cohesion
    2, depthCoefficient 0.533333333333333 (the upper half yields at width 3)."""
    mesh = Mesh(2, (30, 10), (0.0, 0.0), (width, height))
    left, right = 0.5, -0.5
    top = -height * (right - left) / width
    bc = VelocityBC(left={"vx": left}, right={"vx": right}, top={"vy": top}, bottom={"vy": 0.0})
    if kind == "VonMises":
        yr, tol = VonMises(cohesion=3.0222222), 1e-4
    elif kind == "Byerlee":
        yr, tol = Byerlee(cohesion=2.0, depthCoefficient=0.533333333333333), 1e-5
    else:
        raise ValueError(kind)
    coords = gauss_points(mesh)
    mats = [RheologyMaterial([MaterialViscosity(3.4), yr])]
    return Workload(f"yield_criterion_{kind}", mesh, bc, mats, BodyForce(), coords,
                    np.zeros(coords.shape[0], dtype=np.int32), uzawa=UzawaSolver(tolerance=tol),
                    picard=Picard(nonLinearMaxIterations=500, nonLinearTolerance=0.01),
                    meta={"width": width, "height": height})
