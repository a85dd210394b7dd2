"""B200-native particle-mesh step of the CUBE cosmological N-body code.

The CUDA library libcube_b200.so (built from csrc/ for sm_100a) exports the
C-ABI declared in include/cube_gpu.h; `Cube` mirrors the reference's step
routines on top of it.  Importing this package does not need a GPU; creating a
`Cube` does, and raises if the library is missing.
"""
from .abi import CubeParams, CubeScalars, make_params  # noqa: F401
from .cube import Cube, CubeError, expansion, load_library, scalars_from_ic  # noqa: F401

__all__ = ["Cube", "CubeError", "CubeParams", "CubeScalars", "make_params", "expansion", "load_library",
           "scalars_from_ic"]
