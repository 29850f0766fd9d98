"""Host logic of the reconstruction driver: motion binning
(Methods/compressMotion.m) and the pyramid plan (Methods/pyramidPlan.m)."""

import math

import numpy as np
import pytest

from disorder_b200 import recon


@pytest.mark.parametrize("n", [64, 37, 16, 5, 3, 2])
def test_haar_round_trip(n):
    x = np.random.default_rng(n).standard_normal(n)
    C, L = recon._haar_dec(x, int(math.floor(math.log2(n))))
    assert L[0] == n and len(C) == len(L)
    assert np.allclose(recon._haar_rec(C, L), x, atol=1e-13)


def test_haar_matches_the_definition_on_an_even_pair():
    C, L = recon._haar_dec(np.array([3.0, 1.0]), 1)
    s = math.sqrt(0.5)
    assert np.allclose(C[0], [4 * s]) and np.allclose(C[1], [2 * s])


def _offsets(n, per=10, outer=7):
    return np.concatenate([[0], np.cumsum(np.full(n, per)), [n * per + outer]]).astype(np.int64)


def test_piecewise_constant_motion_bins_by_run():
    rng = np.random.default_rng(1)
    T = np.zeros((64, 6), np.float32)
    for k in range(4):
        T[16 * k:16 * (k + 1)] = rng.uniform(-3, 3, 6)
    nEc = _offsets(64)
    Tb, off, bins = recon.compressMotion(T, nEc, math.sqrt(2))
    assert Tb.shape == (4, 6)
    assert np.allclose(Tb, T[::16], atol=1e-6)
    assert list(off) == [0, 160, 320, 480, 640, 647]
    assert list(bins) == list(np.repeat(np.arange(4), 16))


def test_zero_motion_is_one_bin():
    Tb, off, _ = recon.compressMotion(np.zeros((64, 6)), _offsets(64), math.sqrt(2))
    assert Tb.shape == (1, 6) and not Tb.any() and list(off) == [0, 640, 647]


def test_distinct_motion_keeps_every_state_within_the_limits():
    rng = np.random.default_rng(2)
    T = np.zeros((64, 6), np.float32)
    T[:, :3] = rng.uniform(-5, 5, (64, 3))
    T[:, 3:] = np.radians(rng.uniform(-5, 5, (64, 3)))
    res = math.sqrt(2)
    Tb, off, _ = recon.compressMotion(T, _offsets(64), res)
    assert Tb.shape == (64, 6) and np.array_equal(off, _offsets(64))
    # zeroing coefficients below the limit moves a parameter by at most
    # (number of levels + 1) times the limit
    lim = 7 * np.array([0.05 * res] * 3 + [math.radians(0.02 * res)] * 3)
    assert np.all(np.abs(Tb - T) <= lim)


def test_binned_structure_for_the_image_update():
    from disorder_b200.api import Struct
    T = np.zeros((8, 6), np.float32)
    T[4:] = 1.0
    nEc = _offsets(8, per=3, outer=2)
    E = Struct(Tr=T, NMs=8, NSe=9, nEc=nEc, ky=np.zeros(26, np.int32), kz=np.zeros(26, np.int32),
               mSt=np.repeat(np.arange(9), np.diff(nEc)).astype(np.int32))
    Eb = recon.binned(E, 1.0)
    assert Eb.NMs == 2 and Eb.NSe == 3 and list(Eb.nEc) == [0, 12, 24, 26]
    assert list(np.bincount(Eb.mSt)) == [12, 12, 2]
    assert E.NMs == 8  # the motion update keeps the unbinned structure


def test_pyramid_plan_of_the_benchmark_scan():
    resPyr, L, estT, resIso = recon.pyramidPlan((1.0, 1.0, 1.0), 4.0, 1, (1, 0))
    assert L == 3 and list(resPyr) == [0.25, 0.5, 1.0] and list(estT) == [1, 1, 0]
    assert np.allclose(resIso, math.sqrt(2) * np.array([4, 2, 1]))
