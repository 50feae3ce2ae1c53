"""Slab decomposition of one Stokes problem over ranks (one process per GPU).

The reference's only parallelism is domain decomposition: each MPI rank owns part of the
mesh, exchanges the shared nodes' values with its neighbours (StGermain/Base/Automation/
src/Comm.cxx:206-306), sums the Krylov dot products over ranks, and hands material points
to the rank whose domain they enter (StgDomain/Swarm/src/ParticleMovementHandler.cxx:
345-487).  Here the mesh is cut into slabs of whole element layers along its last axis
(z in 3D, y in 2D); rank r owns element layers [k0_r, k1_r) and holds the node layers
k0_r … k1_r, so the node plane between two slabs lives on both ranks:

- element terms (K, G, the force vector, the Jacobi diagonal) are summed per rank over
  its own elements, then the two copies of each interface plane exchange their partial
  sums and add them (a one-plane halo, `SlabComm.halo_add`), so both copies hold the
  global value;
- Gᵀu and the element data (pressure, Ĝ) are local;
- dot products sum each node once (the lower rank's copy of an interface plane does not
  count) and all-reduce;
- points belong to the rank owning their element; after advection the points that
  crossed a slab face move to the neighbouring rank (`SlabProblem.migrate`).

The solve is the reference's: Uzawa (Stokes_SLE_UzawaSolver.cxx:393-938) around the
PETSc CG + Jacobi inner solve with its preconditioned-norm stopping rule, in FP64, with
every vector operation and dot product as above.  Collectives are torch.distributed
(NCCL between GPUs, gloo on the CPU); the per-slab operators are any problem object with
the StokesProblem interface (the GPU library through gale_b200.stokes, or a CPU problem of
the same interface).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

from . import abi
from .stokes import Mesh

WALLS = ("left", "right", "bottom", "top", "back", "front")


def slab_bounds(n_layers: int, world: int) -> List[Tuple[int, int]]:
    """Element layers [k0, k1) of each rank: contiguous, sizes differing by at most one."""
    if world < 1 or n_layers < world:
        raise ValueError("every rank needs at least one element layer")
    base, extra = divmod(n_layers, world)
    out, k = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((k, k + n))
        k += n
    return out


def vertex_coord(mesh: abi.MeshDesc, d: int, i: int) -> float:
    """CartesianGenerator vertex coordinate of index i along axis d (the library's
    vert_coord_d: min, max exactly at the ends, min + (i/n)(max − min) between)."""
    n = mesh.elements[d]
    if i == 0:
        return float(mesh.min[d])
    if i == n:
        return float(mesh.max[d])
    return float(mesh.min[d]) + (float(i) / float(n)) * (float(mesh.max[d]) - float(mesh.min[d]))


def slab_mesh(mesh: abi.MeshDesc, k0: int, k1: int) -> abi.MeshDesc:
    """The mesh of element layers [k0, k1) along the last axis."""
    dim = mesh.dim
    ax = dim - 1
    el = [mesh.elements[d] for d in range(dim)]
    el[ax] = k1 - k0
    lo = [float(mesh.min[d]) for d in range(dim)]
    hi = [float(mesh.max[d]) for d in range(dim)]
    lo[ax], hi[ax] = vertex_coord(mesh, ax, k0), vertex_coord(mesh, ax, k1)
    return Mesh(dim, tuple(el), tuple(lo), tuple(hi))


def node_bc_arrays(mesh: abi.MeshDesc, bc: abi.VelocityBC) -> Tuple[np.ndarray, np.ndarray]:
    """Per-node fixed mask (bit c: component c) and values [nodes, dim] of a wall BC set:
    a node on several walls takes the value of the last wall in the order left, right,
    bottom, top, back, front that fixes the component (the library's rule)."""
    dim = mesh.dim
    nn = [mesh.elements[d] + 1 for d in range(dim)]
    idx = np.indices(nn[::-1]).reshape(dim, -1)[::-1]  # idx[d] = node index along axis d
    fixed = np.zeros(int(np.prod(nn)), dtype=np.uint8)
    values = np.zeros((fixed.shape[0], dim))
    for w in range(2 * dim):
        d, hi = w // 2, w % 2
        on = idx[d] == (nn[d] - 1 if hi else 0)
        for c in range(dim):
            if bc.fixed[w][c]:
                fixed[on] |= np.uint8(1 << c)
                values[on, c] = bc.value[w][c]
    return fixed, values


class SlabComm:
    """The collectives of one rank: interface-plane halo sums and owned dot products."""

    def __init__(self, rank: int, world: int, plane_nodes: int, dim: int, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank, self.world = rank, world
        self.plane = plane_nodes * dim  # values of one node plane (node-major layout)
        self.dim = dim
        self.device = device

    def _t(self, a: np.ndarray):
        return self.torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def halo_add(self, y: np.ndarray) -> np.ndarray:
        """Both copies of each interface plane get the sum of the two ranks' partials."""
        if self.world == 1:
            return y
        P = self.plane
        dist = self.dist
        reqs, recv_lo, recv_hi = [], None, None
        if self.rank > 0:
            recv_lo = self._t(np.empty(P))
            reqs.append(dist.isend(self._t(y[:P]), self.rank - 1))
            reqs.append(dist.irecv(recv_lo, self.rank - 1))
        if self.rank < self.world - 1:
            recv_hi = self._t(np.empty(P))
            reqs.append(dist.isend(self._t(y[-P:]), self.rank + 1))
            reqs.append(dist.irecv(recv_hi, self.rank + 1))
        for q in reqs:
            q.wait()
        y = y.copy()
        if recv_lo is not None:
            y[:P] += recv_lo.cpu().numpy()
        if recv_hi is not None:
            y[-P:] += recv_hi.cpu().numpy()
        return y

    def owned(self, n: int) -> slice:
        """Node-major values this rank counts in a dot product: its top interface plane
        belongs to the rank above."""
        return slice(0, n - self.plane) if self.rank < self.world - 1 else slice(0, n)

    def allreduce(self, v: float) -> float:
        if self.world == 1:
            return float(v)
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t)
        return float(t.item())

    def dot_nodal(self, a: np.ndarray, b: np.ndarray) -> float:
        s = self.owned(a.shape[0])
        return self.allreduce(float(np.dot(a[s], b[s])))

    def dot_elem(self, a: np.ndarray, b: np.ndarray) -> float:
        return self.allreduce(float(np.dot(a, b)))

    def send_points(self, to: int, arr: np.ndarray):
        return self.dist.isend(self._t(arr), to)


class SlabProblem:
    """One rank's slab of a Stokes problem: builds the slab's problem object from the
    global inputs and runs the distributed operators, the Uzawa solve and the point
    migration.

    make_problem(mesh) -> a problem object with set_velocity_bc_nodes, set_materials,
    set_body_force, set_temperature, set_points, assemble, apply_K, apply_G, apply_GT,
    rhs, diagonals, advect (node-major host arrays).  locate(mesh, coords) -> global
    element of every point (the bit-exact search)."""

    def __init__(self, w, rank: int, world: int, make_problem: Callable, locate: Callable, device=None):
        self.w, self.rank, self.world = w, rank, world
        mesh = w.mesh
        self.dim = dim = mesh.dim
        ax = dim - 1
        self.bounds = slab_bounds(mesh.elements[ax], world)
        self.k0, self.k1 = self.bounds[rank]
        self.mesh = slab_mesh(mesh, self.k0, self.k1)
        self.locate = locate
        nn = [mesh.elements[d] + 1 for d in range(dim)]
        self.plane_nodes = int(np.prod(nn[:ax]))
        self.comm = SlabComm(rank, world, self.plane_nodes, dim, device)
        # global per-node BCs, restricted to this slab's node layers
        if w.bc_nodes is not None:
            fixed, values = w.bc_nodes
        else:
            fixed, values = node_bc_arrays(mesh, w.bc)
        lo, hi = self.k0 * self.plane_nodes, (self.k1 + 1) * self.plane_nodes
        self.node_range = (lo, hi)
        self._make_problem = make_problem
        self.P = make_problem(self.mesh)
        self.P.set_velocity_bc_nodes(np.ascontiguousarray(fixed[lo:hi]), np.ascontiguousarray(values[lo:hi]))
        self.fixed = np.ascontiguousarray(fixed[lo:hi])
        self.P.set_materials(w.materials)
        self.P.set_body_force(w.force)
        if w.temperature is not None:
            self.P.set_temperature(np.ascontiguousarray(w.temperature[lo:hi]))
        # the points of this slab's elements
        cell = locate(mesh, w.coords)
        layer = cell // self.plane_elements(mesh)
        keep = (layer >= self.k0) & (layer < self.k1)
        self.coords = np.ascontiguousarray(w.coords[keep])
        self.material = np.ascontiguousarray(w.material[keep])
        self.plastic = None if w.plastic_strain is None else np.ascontiguousarray(w.plastic_strain[keep])
        self.ids = np.flatnonzero(keep)  # global point indices, for gathering results
        self.P.set_points(self.coords, self.material, self.plastic)
        self.nel_global = int(np.prod([mesh.elements[d] for d in range(dim)]))

    @staticmethod
    def plane_elements(mesh) -> int:
        return int(np.prod([mesh.elements[d] for d in range(mesh.dim - 1)]))

    # ---- distributed operators (node-major nodal vectors of this slab) -----------------
    def assemble(self):
        self.P.assemble()
        f, h = self.P.rhs()
        kd, sd = self.P.diagonals()
        self.f = self.comm.halo_add(f)
        self.h = h
        self.kdiag = self.comm.halo_add(kd)
        self.sdiag = sd
        self.free = np.repeat(self.fixed[:, None], self.dim, axis=1).reshape(-1)
        self.free = ((self.free >> np.tile(np.arange(self.dim), self.fixed.shape[0])) & 1) == 0

    def apply_K(self, x):
        return self.comm.halo_add(self.P.apply_K(x))

    def apply_G(self, p):
        return self.comm.halo_add(self.P.apply_G(p))

    def apply_GT(self, u):
        return self.P.apply_GT(u)

    # ---- the solve ---------------------------------------------------------------------
    def jacobi_cg(self, b, rtol, maxit):
        """PETSc CG + PCJACOBI, zero guess, preconditioned norm, KSPConvergedDefault."""
        c = self.comm
        fr = self.free
        x = np.zeros_like(b)
        r = np.where(fr, b, 0.0)
        z = np.where(fr, r / self.kdiag, 0.0)
        rnorm0 = np.sqrt(c.dot_nodal(z, z))
        ttol = max(rtol * rnorm0, 1e-50)
        if rnorm0 <= ttol:
            return x, 0
        beta, betaold = c.dot_nodal(z, r), 0.0
        p = None
        for it in range(1, maxit + 1):
            p = z.copy() if it == 1 else z + (beta / betaold) * p
            betaold = beta
            Ap = self.apply_K(p)
            a = beta / c.dot_nodal(p, Ap)
            x += a * p
            r -= a * Ap
            z = np.where(fr, r / self.kdiag, 0.0)
            dp = np.sqrt(c.dot_nodal(z, z))
            if dp <= ttol:
                return x, it
            if not np.isfinite(dp):
                raise FloatingPointError("inner CG: non-finite residual")
            beta = c.dot_nodal(z, r)
        raise RuntimeError("inner CG: iteration limit")

    def uzawa(self, params: abi.UzawaParams):
        """_Stokes_SLE_UzawaSolver_Solve (Stokes_SLE_UzawaSolver.cxx:393-938), distributed.
        Returns (u free part + BC values, node-major; element pressure; stats)."""
        c = self.comm
        tol = params.tolerance
        maxit = params.inner_max_iterations or 10000
        scaleq = np.sqrt(self.nel_global)
        q = np.zeros(self.h.shape[0])
        its = 0
        vstar, k = self.jacobi_cg(self.f, tol, maxit)
        its += k
        qtmp = self.apply_GT(vstar) - self.h
        rhs_scale = np.sqrt(c.dot_elem(qtmp, qtmp)) / scaleq
        inner = params.inner_rtol_factor * tol
        u, k = self.jacobi_cg(self.f - self.apply_G(q), inner, maxit)
        its += k
        r = self.apply_GT(u) - self.h
        zr_prev, relres, absres, it = 1.0, 0.0, 0.0, 0
        s = None
        while True:
            z = r / self.sdiag if params.use_preconditioner else r.copy()
            zr = c.dot_elem(z, r)
            s = z.copy() if it == 0 else z + (zr / zr_prev) * s
            vstar, k = self.jacobi_cg(self.apply_G(s), inner, maxit)
            its += k
            qtmp = self.apply_GT(vstar)
            alpha = zr / c.dot_elem(s, qtmp)
            q += alpha * s
            u -= alpha * vstar
            r -= alpha * qtmp
            zr_prev = zr
            absres = np.sqrt(c.dot_elem(r, r)) / scaleq
            relres = absres / rhs_scale
            if not (it < params.max_iterations):
                raise RuntimeError("Uzawa: iteration limit")
            it += 1
            chosen = absres if params.use_absolute_tolerance else relres
            if not (chosen > tol or it < params.min_iterations):
                break
        fixed_vals = self._bc_values()
        u_full = np.where(self.free, u, fixed_vals)
        return u_full, q, {"outer_iterations": it, "inner_iterations": its, "rel_residual": relres}

    def _bc_values(self):
        w = self.w
        if w.bc_nodes is not None:
            values = w.bc_nodes[1]
        else:
            values = node_bc_arrays(w.mesh, w.bc)[1]
        lo, hi = self.node_range
        return np.ascontiguousarray(values[lo:hi]).reshape(-1)

    # ---- advection and migration ---------------------------------------------------------
    def advect_and_migrate(self, dt: float, u_full: np.ndarray, order: int = 2, make_problem: Callable = None):
        """RK2 advection of this slab's points, then every point whose element now lies in a
        neighbouring slab moves to that rank (a point crosses at most one slab face per
        Courant-limited step).  The midpoint stage may fall in the neighbour's first element
        layer, so the advection runs on the slab widened by one element layer on each
        interior side, with the velocity of the extra node layers from the neighbours (the
        reference's shadow layer, shadowDepth 1).  Returns the new point count."""
        ax = self.dim - 1
        n_ax = self.w.mesh.elements[ax]
        e0, e1 = max(self.k0 - 1, 0), min(self.k1 + 1, n_ax)
        if getattr(self, "_adv_bounds", None) != (e0, e1):
            self.Padv = (make_problem or self._make_problem)(slab_mesh(self.w.mesh, e0, e1))
            self.Padv.set_materials(self.w.materials)
            self._adv_bounds = (e0, e1)
        u_ext = self._widen(u_full, e0 < self.k0, e1 > self.k1)
        # one marker point at the centre of every shadow element (a located swarm has no
        # empty element); markers are advected with the rest and dropped
        markers = self._shadow_markers(e0, e1)
        pts = np.ascontiguousarray(np.concatenate([self.coords, markers])) if markers.shape[0] else self.coords
        mats = np.concatenate([self.material, np.zeros(markers.shape[0], dtype=np.int32)])
        self.Padv.set_points(pts, np.ascontiguousarray(mats), None)
        new = self.Padv.advect(dt, u_ext, order)[:self.coords.shape[0]]
        cell = self.locate(self.w.mesh, new)
        layer = cell // self.plane_elements(self.w.mesh)
        down = layer < self.k0
        up = layer >= self.k1
        stay = ~(down | up)
        if (down & (self.rank == 0)).any() or (up & (self.rank == self.world - 1)).any():
            raise RuntimeError("a point left the mesh")
        payload = lambda m: np.concatenate([new[m], self.material[m][:, None].astype(np.float64),
                                            self.ids[m][:, None].astype(np.float64)], axis=1)
        outgoing = {self.rank - 1: payload(down), self.rank + 1: payload(up)}
        incoming = self._exchange(outgoing)
        keep = [np.concatenate([new[stay], self.material[stay][:, None].astype(np.float64),
                                self.ids[stay][:, None].astype(np.float64)], axis=1)] + incoming
        allp = np.concatenate(keep, axis=0)
        order_ = np.argsort(allp[:, -1], kind="stable")  # the global input order
        allp = allp[order_]
        self.coords = np.ascontiguousarray(allp[:, :self.dim])
        self.material = np.ascontiguousarray(allp[:, self.dim].astype(np.int32))
        self.ids = allp[:, self.dim + 1].astype(np.int64)
        self.P.set_points(self.coords, self.material, None)
        return self.coords.shape[0]

    def _shadow_markers(self, e0: int, e1: int) -> np.ndarray:
        mesh = self.w.mesh
        dim = self.dim
        ax = dim - 1
        layers = [k for k in (e0, e1 - 1) if k < self.k0 or k >= self.k1]
        if not layers:
            return np.zeros((0, dim))
        centres = []
        for d in range(ax):
            v = np.array([vertex_coord(mesh, d, i) for i in range(mesh.elements[d] + 1)])
            centres.append(0.5 * (v[:-1] + v[1:]))
        grids = np.meshgrid(*centres, indexing="ij") if ax else []
        base = np.stack([g.reshape(-1) for g in grids], axis=1) if ax else np.zeros((1, 0))
        out = []
        for k in layers:
            zc = 0.5 * (vertex_coord(mesh, ax, k) + vertex_coord(mesh, ax, k + 1))
            out.append(np.concatenate([base, np.full((base.shape[0], 1), zc)], axis=1))
        return np.concatenate(out)

    def _widen(self, u: np.ndarray, below: bool, above: bool) -> np.ndarray:
        """u with the neighbours' node layer k0−1 prepended and k1+1 appended."""
        c = self.comm
        torch, dist = c.torch, c.dist
        P = c.plane
        reqs, lo, hi = [], None, None
        if below:  # rank − 1 holds layer k0 − 1 as its second-to-last plane
            lo = torch.zeros(P, dtype=torch.float64, device=c.device)
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(u[P:2 * P])).to(c.device), self.rank - 1))
            reqs.append(dist.irecv(lo, self.rank - 1))
        if above:
            hi = torch.zeros(P, dtype=torch.float64, device=c.device)
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(u[-2 * P:-P])).to(c.device), self.rank + 1))
            reqs.append(dist.irecv(hi, self.rank + 1))
        for q in reqs:
            q.wait()
        parts = ([lo.cpu().numpy()] if below else []) + [u] + ([hi.cpu().numpy()] if above else [])
        return np.ascontiguousarray(np.concatenate(parts))

    def _exchange(self, outgoing) -> List[np.ndarray]:
        """Counts first, then the rows, with each neighbour."""
        c = self.comm
        torch, dist = c.torch, c.dist
        cols = self.dim + 2
        got = []
        for nb in (self.rank - 1, self.rank + 1):
            if nb < 0 or nb >= self.world:
                continue
            out = outgoing[nb]
            cnt_in = torch.zeros(1, dtype=torch.int64, device=c.device)
            reqs = [dist.isend(torch.tensor([out.shape[0]], dtype=torch.int64, device=c.device), nb),
                    dist.irecv(cnt_in, nb)]
            for q in reqs:
                q.wait()
            n_in = int(cnt_in.item())
            buf = torch.zeros(max(n_in, 1) * cols, dtype=torch.float64, device=c.device)
            reqs = []
            if out.shape[0]:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(out.reshape(-1))).to(c.device), nb))
            if n_in:
                reqs.append(dist.irecv(buf, nb))
            for q in reqs:
                q.wait()
            if n_in:
                got.append(buf.cpu().numpy()[:n_in * cols].reshape(n_in, cols))
        return got


def gather_nodal(sp: SlabProblem, y: np.ndarray) -> np.ndarray:
    """The global node-major vector from every rank's slab vector (rank 0 gets it)."""
    import torch
    import torch.distributed as dist
    c = sp.comm
    own = y[c.owned(y.shape[0])]
    parts = [torch.zeros(0)] * sp.world
    sizes = [0] * sp.world
    t = torch.tensor([own.shape[0]], dtype=torch.int64)
    allsz = [torch.zeros(1, dtype=torch.int64) for _ in range(sp.world)]
    dist.all_gather(allsz, t)
    sizes = [int(s.item()) for s in allsz]
    mx = max(sizes)
    buf = torch.zeros(mx, dtype=torch.float64)
    buf[:own.shape[0]] = torch.from_numpy(own)
    parts = [torch.zeros(mx, dtype=torch.float64) for _ in range(sp.world)]
    dist.all_gather(parts, buf)
    return np.concatenate([parts[r].numpy()[:sizes[r]] for r in range(sp.world)])


def gather_elem(sp: SlabProblem, q: np.ndarray) -> np.ndarray:
    """The global element vector (element layers are contiguous per rank)."""
    import torch
    import torch.distributed as dist
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(sp.world)]
    dist.all_gather(sizes, torch.tensor([q.shape[0]], dtype=torch.int64))
    sizes = [int(s.item()) for s in sizes]
    mx = max(sizes)
    buf = torch.zeros(mx, dtype=torch.float64)
    buf[:q.shape[0]] = torch.from_numpy(np.ascontiguousarray(q))
    parts = [torch.zeros(mx, dtype=torch.float64) for _ in range(sp.world)]
    dist.all_gather(parts, buf)
    return np.concatenate([parts[r].numpy()[:sizes[r]] for r in range(sp.world)])
