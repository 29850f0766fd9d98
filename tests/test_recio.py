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


def test_roi_against_the_while_loops():
    rng = np.random.default_rng(5)
    for _ in range(15):
        M = np.zeros((int(rng.integers(9, 20)), int(rng.integers(5, 12)), int(rng.integers(4, 9))))
        sl = tuple(slice(int(rng.integers(0, s // 2)), int(rng.integers(s // 2 + 1, s + 1))) for s in M.shape)
        M[sl] = rng.uniform(0.5, 1.0)
        for sy in ([0, 0, 0], [1, 0, 1]):
            for ev in ([0, 0, 0], [1, 1, 1]):
                for ext in (0, 2):
                    assert np.array_equal(recio.compute_roi(M, ext, sy, ev), orec.computeROI(M, ext, sy, ev))
        R = recio.compute_roi(M, 1, [0, 0, 0], [1, 0, 0])
        for dims in (1, [1, 3], None):
            crop = recio.extract_roi(M, R, 1, dims)  # ext = 1 crops, ext = 0 puts back
            assert np.array_equal(crop, orec.extractROI(M, R, 1, dims))
            back = recio.extract_roi(crop, R, 0, dims)
            assert np.array_equal(back, orec.extractROI(crop, R, 0, dims))
            assert back.shape == M.shape and np.array_equal(back * (M != 0), M)
    with pytest.raises(ValueError):
        recio.compute_roi(np.zeros((4, 4, 4)))


def test_tukey_window():
    for N, sp, g in (((16,), [1], [0.5]), ((9, 12, 7), [10, 10, 1], [0.0, 0.0, 0.1]), ((20, 11, 8), [1, 2, 1], [0.3])):
        a = recio.tukey_filter(N, sp, g)
        b = orec.buildFilter_tukey(list(N), sp, g)
        assert np.allclose(a, b, rtol=0, atol=1e-12)
    # one dimension, no taper: 1 up to the band edge, 0 at k = pi (the most
    # negative frequency of an even length), DC first after fftshift
    w = np.fft.ifftshift(recio.tukey_filter((8,), [1], [0.0]))
    assert w[0] == 0 and np.all(w[1:] == 1)
    w = np.fft.ifftshift(recio.tukey_filter((8,), [1], [0.5]))
    assert np.allclose(w, [0, 0.5, 1, 1, 1, 1, 1, 0.5])


def test_prepare_rec_against_the_oracle():
    rng = np.random.default_rng(6)
    Nr, Ny, Nz, C = 24, 10, 8, 3
    M = np.zeros((Nr, Ny, Nz))
    M[5:18, 1:9, 2:7] = 1
    y = (rng.standard_normal((Nr, Ny, Nz, C, 2, 2)) + 1j * rng.standard_normal((Nr, Ny, Nz, C, 2, 2)))
    S = rng.standard_normal((Nr, Ny, Nz, C)) + 1j * rng.standard_normal((Nr, Ny, Nz, C))
    a = recio.prepare_rec(y, S, M, (0.5, 1.0, 2.0), apod=(0.1, 0.0, 0.0))
    b = orec.prepare_rec(y, S, M, (0.5, 1.0, 2.0), apod=(0.1, 0.0, 0.0))
    # the readout ROI of the mask is 13 samples, evened to 12 (ev = [1 0 0])
    assert list(a["ROI"][0, :4]) == [7, 18, 24, 12]
    assert a["y"].shape == (Nz, Ny, 12, C, 4) and a["S"].shape == (Nz, Ny, 12, C) and a["M"].shape == (Nz, Ny, 12)
    assert a["voxSiz"] == (2.0, 1.0, 0.5) and a["NY"] == (Nz, Ny, 12, C, 4)
    for k in ("y", "S", "M"):
        assert np.allclose(a[k], b[k], rtol=0, atol=1e-12)
    assert np.array_equal(a["ROI"], b["ROI"])
