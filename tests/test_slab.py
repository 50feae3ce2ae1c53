"""Slab decomposition of one problem (gale_b200/slab.py) with gloo ranks on the CPU, on the
oracle's arithmetic (each rank's slab is an oracle problem; the halo sums, the owned dot
products, the distributed Uzawa/CG and the point migration are the module's).  Checked
against the single-domain oracle on the same inputs:

- distributed K x, G p, Gᵀ u, force vector and Jacobi diagonal equal the single-domain ones
  to rounding (≤ 1e-13 relative);
- the distributed Uzawa solve at tight tolerance lands on the single-domain solution: the
  two runs sum their dot products in different orders, so they agree to the level at which
  both sit on the discrete solution (Uzawa 1e-10 → ≤ 1e-8 on the 3D case; 1e-8 → ≤ 1e-6 on
  the three-rank 2D case);
- after an RK2 step long enough to carry points across the slab faces, the migrated point
  sets, gathered, are the points the single-domain oracle advects with the same velocity
  (≤ 1e-13), each point on the rank that owns its new element.
"""
import os
import socket

import numpy as np
import pytest

from gale_b200.slab import node_bc_arrays, slab_bounds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_slab_bounds_cover_every_layer():
    for n, world in ((8, 2), (16, 3), (64, 8), (5, 5)):
        b = slab_bounds(n, world)
        assert b[0][0] == 0 and b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        assert max(k1 - k0 for k0, k1 in b) - min(k1 - k0 for k0, k1 in b) <= 1
    with pytest.raises(ValueError):
        slab_bounds(2, 3)


def test_node_bc_arrays_follow_the_wall_order():
    from gale_b200.stokes import Mesh, VelocityBC
    m = Mesh(2, (2, 2))
    fixed, values = node_bc_arrays(m, VelocityBC(left={"vx": 1.0}, bottom={"vx": 2.0, "vy": 0.0}))
    # node 0 (bottom-left): left fixes vx = 1, bottom (later) overrides it with 2
    assert fixed[0] == 3 and values[0, 0] == 2.0
    assert fixed[3] == 1 and values[3, 0] == 1.0  # left wall, middle
    assert fixed[4] == 0


def _make(name):
    from gale_b200 import workloads
    return {"creep": lambda: workloads.creep_3d(n=6), "sinker": lambda: workloads.sinker_2d(n=12)}[name]()


TOL = {"creep": 1e-10, "sinker": 1e-8}  # Uzawa tolerance of the distributed solve (inner ×0.01)
BOUND = {"creep": 1e-8, "sinker": 1e-6}


def _worker(rank, world, port, name, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    from gale_b200.slab import SlabProblem, gather_elem, gather_nodal
    from gale_b200.stokes import UzawaSolver
    from oracle import oracle
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    oracle.set_threads(max(1, (os.cpu_count() or 2) // world))
    try:
        w = _make(name)
        sp = SlabProblem(w, rank, world, lambda m: oracle.OracleProblem(m), oracle.locate)
        sp.assemble()
        lo, hi = sp.node_range
        dim = w.dim
        rng = np.random.default_rng(11)
        xg = rng.standard_normal(w.nnode * dim)
        pg = rng.standard_normal(w.nel)
        ne_plane = sp.plane_elements(w.mesh)
        x = np.ascontiguousarray(xg[lo * dim:hi * dim])
        p = np.ascontiguousarray(pg[sp.k0 * ne_plane:sp.k1 * ne_plane])
        out = {"Kx": gather_nodal(sp, sp.apply_K(x)), "Gp": gather_nodal(sp, sp.apply_G(p)),
               "GTu": gather_elem(sp, sp.apply_GT(x)), "f": gather_nodal(sp, sp.f),
               "kdiag": gather_nodal(sp, sp.kdiag)}
        prm = UzawaSolver(tolerance=TOL[name], innerRtolFactor=0.01, maxIterations=5000, innerMaxIterations=200000)
        u, pres, st = sp.uzawa(prm)
        out["u"] = gather_nodal(sp, u)
        out["p"] = gather_elem(sp, pres)
        out["stats"] = st
        # an advection step of several Courant steps carries points across the slab faces
        hmin = min((w.mesh.max[d] - w.mesh.min[d]) / w.mesh.elements[d] for d in range(dim))
        dt = 4.0 * 0.5 * hmin / np.abs(out["u"]).max()
        n_after = sp.advect_and_migrate(dt, u, 2)
        out["dt"] = dt
        out["points"] = (sp.ids.copy(), sp.coords.copy())
        cell = oracle.locate(w.mesh, sp.coords)
        layer = cell // sp.plane_elements(w.mesh)
        out["owned_layers_ok"] = bool(((layer >= sp.k0) & (layer < sp.k1)).all())
        out["n_after"] = n_after
        dist.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _run(name, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    import queue
    res = {}
    while len(res) < world:
        try:
            r, out = q.get(timeout=5)
            res[r] = out
        except queue.Empty:
            assert all(p.is_alive() or p.exitcode == 0 for p in procs), "a rank failed"
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return res


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name,world", [("creep", 2), ("sinker", 3)])
def test_slab_matches_single_domain(oracle_mod, name, world):
    res = _run(name, world)
    w = _make(name)
    O = w.apply(oracle_mod.OracleProblem(w.mesh))
    O.assemble()
    rng = np.random.default_rng(11)
    xg = rng.standard_normal(w.nnode * w.dim)
    pg = rng.standard_normal(w.nel)
    r0 = res[0]
    f, _ = O.rhs()
    kd, _ = O.diagonals()
    assert rel(r0["Kx"], O.apply_K(xg)) < 1e-13
    assert rel(r0["Gp"], O.apply_G(pg)) < 1e-13
    assert rel(r0["GTu"], O.apply_GT(xg)) < 1e-13
    assert rel(r0["f"], f) < 1e-13
    assert rel(r0["kdiag"], kd) < 1e-13
    from gale_b200.stokes import UzawaSolver
    uo, po, so = O.uzawa(UzawaSolver(tolerance=TOL[name], innerRtolFactor=0.01, maxIterations=5000,
                                     innerMaxIterations=200000))
    assert rel(r0["u"], uo) < BOUND[name]
    pc, poc = r0["p"] - r0["p"].mean(), po - po.mean()
    assert rel(pc, poc) < BOUND[name]
    # migration: every point once, on its owner, at the single-domain advected position
    xo = O.advect(r0["dt"], r0["u"])  # the same velocity: the difference is the decomposition
    ids = np.concatenate([res[r]["points"][0] for r in range(world)])
    xs = np.concatenate([res[r]["points"][1] for r in range(world)])
    assert np.array_equal(np.sort(ids), np.arange(w.coords.shape[0]))
    assert all(res[r]["owned_layers_ok"] for r in range(world))
    assert np.max(np.abs(xs - xo[ids])) < 1e-13
    moved = sum(res[r]["n_after"] for r in range(world))
    assert moved == w.coords.shape[0]
