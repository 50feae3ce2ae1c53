"""Checkpoint I/O in the reference's HDF5 layout (gale_b200/h5lite.py, gale_b200/checkpoint.py).

No HDF5 library exists in this environment, so the writer is checked three ways:
- round trips through the reader, every supported element type;
- against the reference's own checkpoint files: the same datasets and root attributes
  (names, big-endian types, values), and dataspace / datatype / fill-value messages that are
  byte for byte those the HDF5 library wrote;
- the mesh tables (vertices, connectivity with Gale's face order) equal the reference's.
"""
import os

import numpy as np
import pytest

from conftest import reference_dir
from gale_b200 import checkpoint, h5lite, workloads
from gale_b200.stokes import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "lid_driven_pic2d.npz")
LID_CKPT = os.path.join("PICellerator", "SysTest", "RegressionTests", "expected", "LidDrivenPIC2D.xml")


def test_round_trip_every_type(tmp_path):
    rng = np.random.default_rng(3)
    ds = {"f8": rng.random((17, 3)), "f4": rng.random(5).astype(np.float32),
          "i4": rng.integers(-9, 9, (6, 1)).astype(np.int32), "i8": np.arange(4, dtype=np.int64),
          "u1": np.arange(3, dtype=np.uint8), "be": np.arange(3, dtype=">i4"), "one": np.array([0.5])}
    at = {"checkpoint file version": np.array([2], dtype=">i4"), "scale": np.array([1.5, 2.5])}
    p = str(tmp_path / "t.h5")
    h5lite.write(p, ds, at)
    f = h5lite.File(p)
    assert sorted(f.keys()) == sorted(ds)
    for k, v in ds.items():
        r = f[k]
        assert r.dtype == v.dtype and np.array_equal(r, v), k
    a = f.attrs()
    assert a["checkpoint file version"].dtype == np.dtype(">i4") and a["checkpoint file version"][0] == 2
    assert np.array_equal(a["scale"], at["scale"])


def test_mesh_tables_are_the_reference_tables():
    g = dict(np.load(GOLDEN))
    w = workloads.lid_driven_pic2d()
    assert np.array_equal(checkpoint.vertices(w.mesh), g["vertices"])
    assert np.array_equal(checkpoint.connectivity(w.mesh), g["connectivity"])
    # 3D: bottom face then top face, each counter-clockwise
    c = checkpoint.connectivity(Mesh(3, (2, 2, 2)))
    assert c[0].tolist() == [0, 1, 4, 3, 9, 10, 13, 12]


def test_save_load_round_trip(tmp_path):
    g = dict(np.load(GOLDEN))
    w = workloads.lid_driven_pic2d()
    checkpoint.save(str(tmp_path), 10, w.mesh, g["velocity"], g["pressure"], g["positions"], g["material_index"],
                    float(g["current_time"][0]), float(g["dt"][0]))
    o = checkpoint.load(str(tmp_path), 10)
    for k in ("velocity", "pressure", "positions", "material_index", "vertices", "connectivity"):
        assert np.array_equal(o[k], g[k]), k
    assert o["current_time"] == g["current_time"][0] and o["dt"] == g["dt"][0]
    assert o["mesh_resolution"].tolist() == [20, 20]


def test_written_files_match_the_reference_files(tmp_path):
    REF_CKPT = os.path.join(reference_dir(), LID_CKPT)
    g = checkpoint.load(REF_CKPT, 10)
    w = workloads.lid_driven_pic2d()
    checkpoint.save(str(tmp_path), 10, w.mesh, g["velocity"], g["pressure"], g["positions"], g["material_index"],
                    g["current_time"], g["dt"])
    for name in ("VelocityField", "PressureField", "materialSwarm", "timeInfo", "Mesh"):
        a = h5lite.File(str(tmp_path / f"{name}.00010.h5"))
        b = h5lite.File(os.path.join(REF_CKPT, f"{name}.00010.h5"))
        assert sorted(a.keys()) == sorted(b.keys()), name
        aa, ba = a.attrs(), b.attrs()
        assert aa.keys() == ba.keys(), name
        for k in aa:
            assert aa[k].dtype == ba[k].dtype and np.array_equal(aa[k], ba[k]), (name, k)
        for k in a.keys():
            assert np.array_equal(a[k], b[k]) and a[k].dtype == b[k].dtype, (name, k)
            ma = {t: body for t, _, body in a._r.messages(a._links[k])}
            mb = {t: body for t, _, body in b._r.messages(b._links[k])}
            for t in (0x01, 0x03, 0x05):  # dataspace, datatype, fill value
                assert ma[t] == mb[t], (name, k, hex(t))


def test_reads_every_reference_hdf5_file():
    """Every HDF5 file the reference ships (266 regression checkpoints, both checkpoint
    format versions, layout messages of version 2 and 3) parses: datasets, groups, attributes."""
    import glob
    files = sorted(glob.glob(os.path.join(reference_dir(), "**", "*.h5"), recursive=True))
    for path in files:
        f = h5lite.File(path)
        f.attrs()
        for k in f.keys():
            v = f[k]
            if isinstance(v, h5lite.File):
                for kk in v.keys():
                    assert isinstance(v[kk], (np.ndarray, h5lite.File)), (path, k, kk)
            else:
                assert isinstance(v, np.ndarray), (path, k)
    assert len(files) >= 200
