"""The C-ABI library loads and exports every entry point include/gale_gpu.h declares.
No compute call is made; on a machine without a GPU gg_create reports GG_ERR_NO_DEVICE."""
import ctypes as C
import os
import re

import pytest

from gale_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gale_gpu.h")


def header_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:GG_API\s+)?(?:int|const char\*)\s+(gg_\w+)\s*\(", txt, re.M)))


def test_header_declares_the_mirrored_functions():
    assert header_functions() == sorted(abi.ABI_FUNCTIONS)


def test_library_exports_every_symbol():
    if not os.path.exists(abi.LIB_PATH):
        pytest.skip("library not built")
    lib = C.CDLL(abi.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header():
    # sizes of the ABI structs as the C compiler lays them out
    import subprocess, tempfile
    src = r'''
#include <stdio.h>
#include "gale_gpu.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(gg_mesh_desc), sizeof(gg_velocity_bc),
 sizeof(gg_rheology), sizeof(gg_material), sizeof(gg_body_force), sizeof(gg_uzawa_params),
 sizeof(gg_uzawa_stats), sizeof(gg_picard_params), sizeof(gg_picard_stats)); return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        sizes = [int(v) for v in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    py = [C.sizeof(t) for t in (abi.MeshDesc, abi.VelocityBC, abi.Rheology, abi.Material, abi.BodyForce,
                                 abi.UzawaParams, abi.UzawaStats, abi.PicardParams, abi.PicardStats)]
    assert sizes == py


def test_create_without_device_or_invalid_mesh():
    if not os.path.exists(abi.LIB_PATH):
        pytest.skip("library not built")
    lib = abi.load_library()
    bad = abi.MeshDesc()
    bad.dim = 4
    h = C.c_void_p()
    assert lib.gg_create(C.byref(bad), C.byref(h)) == abi.GG_ERR_INVALID
    import torch
    if not torch.cuda.is_available():
        from gale_b200.stokes import Mesh
        m = Mesh(2, (4, 4))
        assert lib.gg_create(C.byref(m), C.byref(h)) == abi.GG_ERR_NO_DEVICE


def test_inspection_entries_refuse_null_handles():
    # argument checks come before any device call
    if not os.path.exists(abi.LIB_PATH):
        pytest.skip("library not built")
    lib = abi.load_library()
    n = C.c_int64(-1)
    assert lib.gg_get_coarse_inverse(None, C.byref(n), None, None) == abi.GG_ERR_INVALID
    assert lib.gg_get_coarse_inverse(C.c_void_p(1), None, None, None) == abi.GG_ERR_INVALID
    assert n.value == -1
