"""Convert the reference's LidDrivenPIC2D regression checkpoint (step 10) into the fixture
tests/golden/lid_driven_pic2d.npz.

Source: PICellerator/SysTest/RegressionTests/expected/LidDrivenPIC2D.xml/{VelocityField,
PressureField,materialSwarm,timeInfo,Mesh}.00010.h5 of the reference, read with
gale_b200.h5lite (no libhdf5).  Run from the repository root:

    python tests/golden/make_lid_driven_golden.py /root/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from gale_b200 import h5lite  # noqa: E402

REL = "PICellerator/SysTest/RegressionTests/expected/LidDrivenPIC2D.xml"


def load(ref_root: str) -> dict:
    d = os.path.join(ref_root, REL)
    vel = h5lite.File(os.path.join(d, "VelocityField.00010.h5"))
    pre = h5lite.File(os.path.join(d, "PressureField.00010.h5"))
    swm = h5lite.File(os.path.join(d, "materialSwarm.00010.h5"))
    tim = h5lite.File(os.path.join(d, "timeInfo.00010.h5"))
    msh = h5lite.File(os.path.join(d, "Mesh.00010.h5"))
    return {
        "velocity": vel["data"],                       # [441, 2] node-major
        "pressure": pre["data"].ravel(),               # [400]
        "positions": swm["Position"],                  # [14104, 2], swarm order
        "material_index": swm["MaterialIndex"].ravel(),
        "current_time": tim["currentTime"],
        "dt": tim["Dt"],
        "vertices": msh["vertices"],
        "connectivity": msh["connectivity"],
        "mesh_resolution": vel.attrs()["mesh resolution"],
        "swarm_particle_count": swm.attrs()["Swarm Particle Count"],
    }


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    np.savez_compressed(os.path.join(HERE, "lid_driven_pic2d.npz"), **load(ref))
    print("wrote", os.path.join(HERE, "lid_driven_pic2d.npz"))
