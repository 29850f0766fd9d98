"""CPU oracle for the DISORDER aligned-reconstruction hot path.

TEST INFRASTRUCTURE ONLY. This package is a NumPy restatement of the
reference MATLAB functions on the hot path (sincRigidTransform and its
gradient, encode/decode/encodedecode, CGsolver, LMsolver, computeEnergy and
the data-preparation helpers around them). Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it, and only as the checker or as the timed CPU baseline; the product path
(``disorder_b200``) never calls into it.

Parity status: UNPINNED by the reference. The reference is MATLAB code with
no tests, no golden vectors and no datasets, and neither MATLAB nor Octave is
available, so its outputs cannot be produced here. The oracle is instead
pinned by known-answer tests derived from the mathematics of the reference
algorithm (identity at zero motion, integer translations equal circular
shifts, exact 90-degree rotations, unitarity, adjointness, finite-difference
gradients, literal-versus-fast encoding agreement); see tests/test_oracle.py.

Every function cites the reference file and lines it restates. Arrays follow
the reference's MATLAB dimension order (axis 0 is MATLAB dim 1): volumes are
``(N1, N2, N3)`` with dims 1-2 the phase encodes and dim 3 the readout, coils
are axis 3 and motion states axis 4.
"""

from . import grids, transform, encoding, solvers, prep  # noqa: F401
