"""The StGermain side of the plugin (gale_b200/host/stokes_gpu_plugin.c) compiled against a
declaration stub of the StGermain / StgFEM / PICellerator / Underworld / PETSc headers
(tests/c/stub) and driven as Gale drives a solver (tests/c/plugin_driver.c):

- Underworld_StokesGPU_Register(PluginsManager*) submits the codelet and adds the
  Stokes_SLE_UzawaSolverGPU type (Plugin.cxx:55,97; Multigrid.cxx:139-143);
- the constructor the component register hands back builds the solver, its AssignFromXML
  reads the Stokes_SLE_UzawaSolver keys (Stokes_SLE_UzawaSolver.cxx:241-264);
- _solverSetup / _solve run through the SLE_Solver function pointers
  (SLE_Solver.h:61-62) on a Stokes_SLE (Stokes_SLE.h:63-81) and write u and p into the
  FeVariables and the SolutionVectors' Vecs.

Without a GPU the solve ends in the reference's failure mode, Journal_Firewall, with the
library's status; on a GPU its result is the Python host's, bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gale_b200")


def build_plugin_driver(tmp):
    exe = os.path.join(tmp, "plugin_driver")
    c = os.path.join(ROOT, "tests", "c")
    cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-Werror",
           os.path.join(c, "plugin_driver.c"), os.path.join(c, "stub", "stub_runtime.c"),
           os.path.join(ROOT, "gale_b200", "host", "stokes_gpu_plugin.c"),
           os.path.join(ROOT, "gale_b200", "host", "stokes_gpu_host.c"),
           "-I", os.path.join(c, "stub"), "-I", os.path.join(ROOT, "include"),
           "-L", LIBDIR, "-lgale_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def write_input(w, path):
    with open(path, "wb") as f:
        np.array([w.mesh.elements[0]], dtype=np.int32).tofile(f)
        np.array([w.coords.shape[0]], dtype=np.int64).tofile(f)
        w.coords.astype(np.float64).tofile(f)
        w.material.astype(np.int32).tofile(f)


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_plugin_registers_and_fails_like_the_reference_without_a_device(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libgale_b200.so")):
        pytest.skip("library not built")
    if have_gpu():
        pytest.skip("a device is present (the GPU test covers the solve)")
    from gale_b200 import workloads
    exe = build_plugin_driver(str(tmp_path))
    w = workloads.sinker_2d(n=8)
    inp = os.path.join(tmp_path, "in.bin")
    write_input(w, inp)
    r = subprocess.run([exe, inp, os.path.join(tmp_path, "out.bin")], capture_output=True, text=True)
    assert "plugin Underworld_StokesGPU solver-type registered" in r.stdout
    # Journal_Firewall with the library's status
    from gale_b200 import abi
    assert r.returncode == 3, (r.stdout, r.stderr)
    assert "Journal_Firewall" in r.stderr and f"status {abi.GG_ERR_NO_DEVICE}" in r.stderr


@pytest.mark.gpu
def test_plugin_solve_matches_python_host(tmp_path):
    from gale_b200 import workloads
    from gale_b200.stokes import StokesProblem
    exe = build_plugin_driver(str(tmp_path))
    w = workloads.sinker_2d(n=16)
    inp, out = os.path.join(tmp_path, "in.bin"), os.path.join(tmp_path, "out.bin")
    write_input(w, inp)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    nn, ne = w.nnode * 2, w.nel
    uc, pc, ufree = data[:nn], data[nn:nn + ne], data[nn + ne:]
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("fp64")
    up, pp, st = G.solve(w.uzawa)
    fields = r.stdout.split("outer")[1].split()
    assert int(fields[0]) == st["outer_iterations"]
    assert np.array_equal(uc, up) and np.array_equal(pc, pp)
    # the SolutionVector holds the free dofs in node order
    fixed = np.zeros((w.nnode, 2), dtype=bool)
    ix, iy = np.arange(w.nnode) % 17, np.arange(w.nnode) // 17
    fixed[:, 0] = (ix == 0) | (ix == 16)
    fixed[:, 1] = (iy == 0) | (iy == 16)
    assert np.array_equal(ufree, up.reshape(-1, 2)[~fixed])
