"""The plugin's C host side (gale_b200/host) compiles with plain gcc against the C ABI
and, on a GPU, produces the same solution as the Python host mirror."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gale_b200")


def build_driver(tmp):
    exe = os.path.join(tmp, "stokes_driver")
    cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-Werror",
           os.path.join(ROOT, "tests", "c", "stokes_driver.c"),
           os.path.join(ROOT, "gale_b200", "host", "stokes_gpu_host.c"),
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lgale_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_c_host_compiles(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libgale_b200.so")):
        pytest.skip("library not built")
    build_driver(str(tmp_path))


@pytest.mark.gpu
def test_c_host_solves_like_python(tmp_path):
    from gale_b200 import workloads
    from gale_b200.stokes import StokesProblem
    exe = build_driver(str(tmp_path))
    w = workloads.sinker_2d(n=16)
    inp, out = os.path.join(tmp_path, "in.bin"), os.path.join(tmp_path, "out.bin")
    with open(inp, "wb") as f:
        np.array([16], dtype=np.int32).tofile(f)
        np.array([w.coords.shape[0]], dtype=np.int64).tofile(f)
        w.coords.astype(np.float64).tofile(f)
        w.material.astype(np.int32).tofile(f)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    uc, pc = data[:w.nnode * 2], data[w.nnode * 2:]
    G = w.apply(StokesProblem(w.mesh))
    G.locate()
    G.build_operator("fp64")
    up, pp, st = G.solve(w.uzawa)
    outer = int(r.stdout.split()[1])
    # the same library call on the same inputs from C and from Python: the FP64 path sums
    # in a fixed order, so the two solves are the same bits
    assert outer == st["outer_iterations"]
    assert np.array_equal(uc, up)
    assert np.array_equal(pc, pp)
