"""Checkpoint files in the reference's layout (host side, numpy + h5lite; no libhdf5).

Gale checkpoints step n as one HDF5 file per object in the output directory:
- `VelocityField.%05d.h5` / `PressureField.%05d.h5` (`_FeVariable_SaveToFile`,
  StgFEM/Discretisation/src/FeVariable.cxx:1986-2140): dataset "/data", one row per node
  (per element for the P0 pressure) holding its dof values; root attributes
  "checkpoint file version" (2), "dimensions" and, for fields on the regular velocity mesh,
  "mesh resolution", all 32-bit big-endian integers;
- `materialSwarm.%05d.h5` (`SwarmDump`, StgDomain/Swarm/src/SwarmDump.cxx:304): one dataset
  per swarm variable ("/Position" [n, dim], "/MaterialIndex" [n, 1]) and the root attribute
  "Swarm Particle Count";
- `timeInfo.%05d.h5` (`_AbstractContext_SaveTimeInfo`): "/currentTime", "/Dt", "/nproc";
- `Mesh.%05d.h5` (`FiniteElementContext.cxx:582-830`): "/min", "/max", "/vertices" and
  "/connectivity", with each element's nodes in Gale's element order except that nodes 2
  and 3 (and 6 and 7) are swapped, so that every face runs counter-clockwise.

`save` writes exactly those objects from this library's arrays; `load` reads them back as
numpy arrays, Gale's own files included, in the current format (version 2) and in the older
version 1 (no attributes, the node number in column 0 of each field row, swarm variables
named "<swarm>-<variable>").
"""
from __future__ import annotations

import os
from typing import Dict

import numpy as np

from . import abi, h5lite

VERSION = 2


def _i32be(v) -> np.ndarray:
    return np.atleast_1d(np.asarray(v, dtype=">i4"))


def _resolution(mesh: abi.MeshDesc):
    return [int(mesh.elements[d]) for d in range(mesh.dim)]


def vertices(mesh: abi.MeshDesc) -> np.ndarray:
    """Node coordinates [nodes, dim] in Gale's node order (x fastest), computed as the
    CartesianGenerator does: min + (i / n)·(max − min), with the walls exact."""
    dim = mesh.dim
    axes = []
    for d in range(dim):
        n = int(mesh.elements[d])
        lo, hi = float(mesh.min[d]), float(mesh.max[d])
        c = lo + (np.arange(n + 1) / n) * (hi - lo)
        c[0], c[-1] = lo, hi
        axes.append(c)
    grids = np.meshgrid(*axes, indexing="ij")
    return np.stack([g.ravel(order="F") for g in grids], axis=1)


def connectivity(mesh: abi.MeshDesc) -> np.ndarray:
    """Element → node table [elements, 2^dim] as Gale's Mesh checkpoint writes it."""
    dim = mesh.dim
    n = _resolution(mesh)
    nn = [k + 1 for k in n]
    idx = np.indices(n[::-1]).reshape(dim, -1)[::-1]  # i (fastest), j, k per element
    corners = []
    for a in range(1 << dim):
        node = np.zeros(idx.shape[1], dtype=np.int64)
        stride = 1
        for d in range(dim):
            node += (idx[d] + ((a >> d) & 1)) * stride
            stride *= nn[d]
        corners.append(node)
    order = [0, 1, 3, 2] if dim == 2 else [0, 1, 3, 2, 4, 5, 7, 6]
    return np.stack([corners[o] for o in order], axis=1).astype(np.int32)


def save(directory: str, step: int, mesh: abi.MeshDesc, u: np.ndarray, p: np.ndarray, coords: np.ndarray,
         material: np.ndarray, current_time: float, dt: float, nproc: int = 1) -> Dict[str, str]:
    """Write the five checkpoint files of step `step` into `directory`; returns their paths.
    u: nodal velocity [nodes*dim] or [nodes, dim] (node-major, BC values included);
    p: element pressure [elements]; coords/material: the material points."""
    dim = mesh.dim
    os.makedirs(directory, exist_ok=True)
    tag = f"{step:05d}"
    paths = {k: os.path.join(directory, f"{k}.{tag}.h5")
             for k in ("VelocityField", "PressureField", "materialSwarm", "timeInfo", "Mesh")}
    res = _resolution(mesh)
    common = {"checkpoint file version": _i32be(VERSION), "dimensions": _i32be(dim)}
    h5lite.write(paths["VelocityField"], {"data": np.asarray(u, dtype=np.float64).reshape(-1, dim)},
                 dict(common, **{"mesh resolution": _i32be(res)}))
    h5lite.write(paths["PressureField"], {"data": np.asarray(p, dtype=np.float64).reshape(-1, 1)}, common)
    coords = np.asarray(coords, dtype=np.float64).reshape(-1, dim)
    h5lite.write(paths["materialSwarm"],
                 {"Position": coords,
                  "MaterialIndex": np.asarray(material, dtype=np.int32).reshape(-1, 1)},
                 {"Swarm Particle Count": _i32be(len(coords))})
    h5lite.write(paths["timeInfo"], {"currentTime": np.array([float(current_time)]), "Dt": np.array([float(dt)]),
                                     "nproc": np.array([int(nproc)], dtype=np.int32)})
    h5lite.write(paths["Mesh"],
                 {"min": np.array([float(mesh.min[d]) for d in range(dim)]),
                  "max": np.array([float(mesh.max[d]) for d in range(dim)]),
                  "vertices": vertices(mesh), "connectivity": connectivity(mesh)},
                 dict(common, **{"mesh resolution": _i32be(res)}))
    return paths


def _rows(f: "h5lite.File", key: str) -> np.ndarray:
    """Rows of a field dataset.  Version 2 files (root attribute "checkpoint file version")
    hold one row per node in node order; version 1 files (no attributes,
    FeVariable.cxx:2236-2240) put the global node number in column 0."""
    data = f[key]
    if "checkpoint file version" in f.attrs():
        return data
    order = np.argsort(data[:, 0], kind="stable")
    return data[order, 1:]


def _swarm_var(f: "h5lite.File", name: str) -> np.ndarray:
    """Swarm variable `name`; older dumps prefix it with the swarm's name ("materialSwarm-")."""
    for k in f.keys():
        if k == name or k.endswith("-" + name):
            return f[k]
    raise KeyError(name)


def load(directory: str, step: int) -> Dict[str, np.ndarray]:
    """Read a checkpoint (this library's or Gale's, version 1 or 2) as flat arrays: velocity
    [nodes, dim], pressure [elements], positions, material_index, current_time, dt,
    vertices, connectivity (None in version 1) and mesh_resolution (None in version 1)."""
    tag = f"{step:05d}"
    f = {k: h5lite.File(os.path.join(directory, f"{k}.{tag}.h5"))
         for k in ("VelocityField", "PressureField", "materialSwarm", "timeInfo", "Mesh")}
    mesh = f["Mesh"]
    v2 = "vertices" in mesh.keys()
    return {
        "velocity": _rows(f["VelocityField"], "data"),
        "pressure": _rows(f["PressureField"], "data").ravel(),
        "positions": _swarm_var(f["materialSwarm"], "Position"),
        "material_index": _swarm_var(f["materialSwarm"], "MaterialIndex").ravel(),
        "current_time": float(f["timeInfo"]["currentTime"][0]),
        "dt": float(f["timeInfo"]["Dt"][0]),
        "vertices": mesh["vertices"] if v2 else _rows(mesh, "data"),
        "connectivity": mesh["connectivity"] if v2 else None,
        "mesh_resolution": f["VelocityField"].attrs().get("mesh resolution"),
    }
