"""The scanner acquisition order -> motion states (disorder_b200.recio, the
acquisition-structure block of Reconstruction/solveXT.m:74-142) against a
loop-by-loop restatement (oracle/recio.py), and end to end against the
DISORDER trajectory generator: the shot map recovered from the scanner's
profile order is the generator's own."""

import numpy as np
import pytest

from disorder_b200 import recio, sampling
from oracle import recio as orec


def _same(a, b):
    for k in ("NEchos", "NShots", "NProfs", "NSweeps", "steady_state"):
        assert a[k] == b[k], k
    for k in ("kTraj", "kShift", "kSize", "kIndex", "sweepSample", "timeIndex", "H"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def _grid(N):
    c = [np.arange(n) - n // 2 for n in N]
    a, b = np.meshgrid(c[0], c[1], indexing="ij")
    return a.ravel(), b.ravel(), (int(c[0][0]), int(c[0][-1])), (int(c[1][0]), int(c[1][-1]))


def test_shots_from_a_random_order():
    N = (12, 10)
    k1, k2, r1, r2 = _grid(N)
    rng = np.random.default_rng(0)
    p = rng.permutation(k1.size)
    z3, z2 = k1[p], k2[p]
    a = recio.acquisition_structure(z2, z3, r2, r1, TFEfactor=20)
    b = orec.acquisition_structure(z2, z3, r2, r1, TFEfactor=20)
    _same(a, b)
    assert a["NShots"] == 6 and not a["steady_state"] and a["H"].min() == 1 and a["H"].max() == 6
    # the DC of the grid is the first element of H (ifftshifted)
    dc = np.flatnonzero((z3 == 0) & (z2 == 0))[0]
    assert a["H"][0, 0] == dc // 20 + 1


def test_repeats_and_revisited_points():
    N = (8, 6)
    k1, k2, r1, r2 = _grid(N)
    rng = np.random.default_rng(1)
    # 72 profiles over 48 points: some points twice, some not at all
    idx = rng.integers(0, k1.size, 72)
    z3, z2 = k1[idx], k2[idx]
    for NRepeats in (1, 2, 3):
        a = recio.acquisition_structure(z2, z3, r2, r1, TFEfactor=12, NRepeats=NRepeats)
        b = orec.acquisition_structure(z2, z3, r2, r1, TFEfactor=12, NRepeats=NRepeats)
        _same(a, b)
    # more repeats than shots: the trajectory repeats (solveXT.m:85-90)
    a = recio.acquisition_structure(z2[:12], z3[:12], r2, r1, TFEfactor=12, NRepeats=4)
    b = orec.acquisition_structure(z2[:12], z3[:12], r2, r1, TFEfactor=12, NRepeats=4)
    _same(a, b)
    assert a["NShots"] == 4 and a["NProfs"] == 48


def test_steady_state_sweeps():
    # one long train (NEchos = NProfs: a single shot) that passes over the
    # whole grid 8 times, a raster forwards then backwards: both coordinates
    # oscillate with the sweeps, which solveXT.m:115-123 reads off the
    # trajectory's DCT (the lowest peak of the two coordinates)
    N = (16, 12)
    raster = [(i, j if i % 2 == 0 else N[1] - 1 - j) for i in range(N[0]) for j in range(N[1])]
    rows = np.array([p for s in range(8) for p in (raster if s % 2 == 0 else raster[::-1])])
    z3 = rows[:, 0] - N[0] // 2
    z2 = rows[:, 1] - N[1] // 2
    r1, r2 = (-N[0] // 2, N[0] - N[0] // 2 - 1), (-N[1] // 2, N[1] - N[1] // 2 - 1)
    a = recio.acquisition_structure(z2, z3, r2, r1, TFEfactor=1)
    b = orec.acquisition_structure(z2, z3, r2, r1, TFEfactor=1)
    _same(a, b)
    assert a["steady_state"] and a["NShots"] == 1 and a["NSweeps"] == 8
    assert np.array_equal(np.bincount(a["sweepSample"])[1:], np.full(8, len(raster)))
    # grouping sweeps in pairs halves them
    g = recio.acquisition_structure(z2, z3, r2, r1, TFEfactor=1, groupSweeps=2)
    _same(g, orec.acquisition_structure(z2, z3, r2, r1, TFEfactor=1, groupSweeps=2))
    assert g["NSweeps"] == 4
    # a staircase in one coordinate has no sweep period below the length
    stair = np.array([(i, j) for i in range(N[0]) for j in range(N[1])])
    st = recio.acquisition_structure(stair[:, 1] - 6, stair[:, 0] - 8, r2, r1, TFEfactor=1)
    assert st["NSweeps"] == 1


def test_the_dct_is_fct():
    """The product's orthonormal DCT-II (scipy) against Methods/fct.m's FFT form."""
    x = np.random.default_rng(2).standard_normal((37, 2))
    assert np.allclose(recio._dct_ortho(x), orec.fct(x), atol=1e-12)
    x = np.random.default_rng(3).standard_normal((40, 3))
    assert np.allclose(recio._dct_ortho(x), orec.fct(x), atol=1e-12)


def test_scans_the_reconstruction_skips():
    k1, k2, r1, r2 = _grid((8, 8))
    with pytest.raises(recio.AcquisitionError):  # separable trajectories (solveXT.m:77)
        recio.acquisition_structure(k2, k1[:-1], r2, r1, TFEfactor=8)
    with pytest.raises(recio.AcquisitionError):  # interrupted scan (:83)
        recio.acquisition_structure(k2[:60], k1[:60], r2, r1, TFEfactor=8)
    with pytest.raises(recio.AcquisitionError):  # outside the grid
        recio.acquisition_structure(k2 + 8, k1, r2, r1, TFEfactor=8)


@pytest.mark.parametrize("order", ["RandomCheckered", "Checkered"])
def test_disorder_trajectory_round_trip(order):
    """A DISORDER trajectory (Acquisition/samplingDISORDER.m) acquired shot by
    shot, echo by echo: the shot map solveXT.m recovers from the profile
    order is the generator's shot map, the one the driver reconstructs with."""
    N = (16, 16)
    pts = sampling.cartesian_points(N)
    _, NP, _, _, Shot, Echo = sampling.samplingDISORDER(pts, (4, 4), order, "AlternatingZigZag",
                                                        rng=np.random.default_rng(4))
    z2, z3 = recio.profile_order(Shot, Echo, N)
    r = (-N[0] // 2, N[0] - N[0] // 2 - 1)
    a = recio.acquisition_structure(z2, z3, r, r, TFEfactor=NP // 16)
    _same(a, orec.acquisition_structure(z2, z3, r, r, TFEfactor=NP // 16))
    assert a["NShots"] == 16
    assert np.array_equal(a["H"], sampling.shot_map(Shot))
