"""Extract the reference's discrete-Voronoi known-answer data into a numpy fixture.

The reference's DVCWeightsSuite (PICellerator/Weights/tests/DVCWeightsSuite.cxx) builds the
Voronoi weights of 10 hard-coded points on a 10×10(×10) element grid and compares them
with PICellerator/Weights/tests/expected/DVCWeightsSuite_testGetCentroids{,2D}.txt.  This
script reads the point coordinates from the suite's source (the `data->pList[i].x = …`
lines) and the expected centroids and weights from the two text files, and writes
tests/golden/dvc_suite.npz.  Run here, where the reference is mounted:

    python tests/golden/make_dvc_golden.py /root/reference
"""
import os
import re
import sys

import numpy as np


def coords(src, name, axes):
    out = {}
    for ax in axes:
        vals = re.findall(r"data->%s\[i\]\.%s\s*=\s*([-+0-9.eE]+)\s*;" % (name, ax), src)
        out[ax] = [float(v) for v in vals]
    return np.array([out[a] for a in axes]).T


def expected(path, dim):
    txt = open(path).read()
    num = r"([-+]?[0-9.]+)"
    if dim == 3:
        c = re.findall(r"centroids: \(cx, cy, cz\) = \(%s, %s, %s\)" % (num, num, num), txt)
    else:
        c = re.findall(r"centroids: \(cx, cy\) = \(%s, %s\)" % (num, num), txt)
    w = re.findall(r"weight = %s" % num, txt)
    return np.array(c, dtype=float), np.array(w, dtype=float)


def main(ref):
    base = os.path.join(ref, "PICellerator", "Weights", "tests")
    src = open(os.path.join(base, "DVCWeightsSuite.cxx")).read()
    p3 = coords(src, "pList", "xyz")
    p2 = coords(src, "pList2D", "xy")
    c3, w3 = expected(os.path.join(base, "expected", "DVCWeightsSuite_testGetCentroids.txt"), 3)
    c2, w2 = expected(os.path.join(base, "expected", "DVCWeightsSuite_testGetCentroids2D.txt"), 2)
    assert p3.shape == (10, 3) and p2.shape == (10, 2) and c3.shape == (10, 3) and c2.shape == (10, 2)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dvc_suite.npz")
    np.savez(out, points3=p3, centroids3=c3, weights3=w3, points2=p2, centroids2=c2, weights2=w2,
             resolution=np.array([10, 10, 10]))
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
