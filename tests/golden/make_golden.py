"""Convert the reference's golden stiffness matrices into compact numpy fixtures.

Reads the PETSc binary matrices the reference's ViscousSuite compares against
(Underworld/Rheology/tests/expected/test*2D.matrix; format: big-endian int32 classid
1211216, rows, cols, nnz, row lengths, column indices, then float64 values) and writes
tests/golden/viscous_suite_K.npz with one CSR triple per rheology.  Run here, where the
reference is mounted; the .npz travels with the tests.

    python tests/golden/make_golden.py /root/reference
"""
import os
import struct
import sys

import numpy as np

NAMES = ["testMaterialViscosity2D", "testArrhenius2D", "testFrankKamenetskii2D"]


def read_petsc_matrix(path):
    b = open(path, "rb").read()
    classid, m, n, nnz = struct.unpack(">4i", b[:16])
    assert classid == 1211216, "not a PETSc Mat"
    rl = np.frombuffer(b, dtype=">i4", count=m, offset=16).astype(np.int64)
    off = 16 + 4 * m
    cols = np.frombuffer(b, dtype=">i4", count=nnz, offset=off).astype(np.int32)
    off += 4 * nnz
    vals = np.frombuffer(b, dtype=">f8", count=nnz, offset=off).astype(np.float64)
    rowptr = np.concatenate([[0], np.cumsum(rl)]).astype(np.int64)
    return m, n, rowptr, cols, vals


def main(ref):
    src = os.path.join(ref, "Underworld", "Rheology", "tests", "expected")
    out = {}
    for name in NAMES:
        m, n, rp, c, v = read_petsc_matrix(os.path.join(src, name + ".matrix"))
        out[name + "_shape"] = np.array([m, n])
        out[name + "_rowptr"] = rp
        out[name + "_cols"] = c
        out[name + "_vals"] = v
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "viscous_suite_K.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
