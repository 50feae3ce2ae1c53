"""gale_b200: B200-native (sm_100a) particle-in-cell Q1-P0 Stokes path of Gale.

The compute path is the CUDA library ``libgale_b200.so`` behind the C ABI of
``include/gale_gpu.h``; this package is its Python host mirror.  See
:mod:`gale_b200.stokes` for the component-level interface and
:mod:`gale_b200.workloads` for the seeded synthetic inputs.
"""
from .abi import load_library, LIB_PATH  # noqa: F401
from .stokes import (Arrhenius, BodyForce, Byerlee, DruckerPrager, FrankKamenetskii,  # noqa: F401
                     GaleError, MaterialViscosity, Mesh, Picard, RheologyMaterial, StokesProblem,
                     StrainWeakening, UzawaSolver, VelocityBC, VonMises, free_slip)

__version__ = "0.1.0"
