import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libdisorder.so")


def make_problem(N=(16, 16, 12), C=4, S=4, seed=1, rot_deg=3.0, trans=2.0, snr=30.0,
                 n_ell=6, dtype=np.complex128, zero_motion=False):
    """A small synthetic scan plus the oracle's E structure for it."""
    from disorder_b200 import synth
    from oracle.grids import generateTransformGrids
    from oracle.encoding import Struct

    sc = synth.make_scan(N, C, S, rot_deg, trans, snr, n_ell, seed, dtype)
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    g = generateTransformGrids(N, N, cent, sh=1)
    T = np.zeros_like(sc.T_gt) if zero_motion else sc.T_gt
    E = Struct(Tr=T, NMs=S, NSe=S + 1, Sf=sc.S.astype(dtype), ky=sc.ky, kz=sc.kz, nEc=sc.nEc,
               mSt=sc.mSt, grids=g, cent=cent)
    return sc, E


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
