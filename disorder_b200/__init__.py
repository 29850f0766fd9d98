"""B200-native (sm_100a) DISORDER aligned-reconstruction hot path.

The compute runs in libdisorder.so (CUDA kernels behind the C ABI declared
in include/disorder.h); this package is the host-side mirror of the
reference's MATLAB call surface (encode, decode, encodedecode, CGsolver,
LMsolver, sincRigidTransform, sincRigidTransformGradient, computeEnergy, and
CSsolver with its shearlet system and trace estimates).
Importing the package does not touch the GPU; the first operator call loads
the library and fails loudly if it is missing.
"""

from .api import (CGsolver, Context, DeviceArray, Grids, LMsolver, Plan, Struct, computeEnergy, decode,  # noqa: F401
                  default_context, encode, encodedecode, generateTransformGrids,
                  precomputeFactorsSincRigidTransform, sincRigidTransform, sincRigidTransformGradient,
                  compressCoils, gather_samples, precondition_weights, resampling)
from ._lib import DisorderError  # noqa: F401
from .cs import CSsolver, ShearletSystem, traceEstimation  # noqa: F401
