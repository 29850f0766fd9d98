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


# ---------------------------------------------------------------- outlier rejection
def test_prctile_is_the_midpoint_rule():
    x = np.array([4.0, 1.0, 3.0, 2.0])
    # MATLAB prctile: sorted values sit at 100*(i-0.5)/n, linear in between, clamped
    assert np.percentile(x, 50, method="hazen") == 2.5
    assert np.percentile(x, 10, method="hazen") == 1.0
    assert np.percentile(x, 25, method="hazen") == 1.5


def _shot_residuals(rng, n_shots=64, per=64, bad=()):
    Re = np.exp(rng.normal(0.0, 0.3, n_shots * per))
    sweeps = np.repeat(np.arange(n_shots), per)
    for b in bad:
        Re[sweeps == b] *= 50.0
    return Re, sweeps


def test_no_outliers_keep_unit_weights():
    Re, sw = _shot_residuals(np.random.default_rng(3))
    We = recon.outlier_weights(Re, sw, 64, leff=1)
    assert We.shape == (64,) and np.all(We == 1.0)


def test_corrupted_shots_are_down_weighted():
    Re, sw = _shot_residuals(np.random.default_rng(4), bad=(5, 40))
    sw = np.concatenate([sw, np.full(30, 64)])  # outer samples are ignored
    Re = np.concatenate([Re, np.full(30, 1e6)])
    We = recon.outlier_weights(Re, sw, 64, leff=1)
    assert We[5] < 1e-3 and We[40] < 1e-3
    assert np.all(np.delete(We, [5, 40]) == 1.0)


@pytest.mark.gpu
def test_sample_energies_match_oracle():
    import disorder_b200 as db
    from conftest import make_problem
    from oracle import encoding as oe
    from oracle.encoding import Struct as OStruct
    N, C, S = (24, 20, 16), 3, 4
    sc, Eo = make_problem(N, C, S, seed=21, rot_deg=4.0, trans=2.0)
    rng = np.random.default_rng(22)
    y = (oe.encode(sc.x_gt.astype(np.complex128), Eo)
         + 0.01 * (rng.standard_normal((int(sc.nEc[-1]), N[2], C)) + 0j)).astype(np.complex64)
    x = (sc.x_gt * 0.9).astype(np.complex64)
    Mb = rng.uniform(0.5, 1.0, N[2]).astype(np.float32)
    Mbe = (np.arange(N[2]) < 11).astype(np.float32)
    ctx = db.Context(0)
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    E = db.Struct(Tr=sc.T_gt, NMs=S, NSe=S + 1, Sf=ctx.upload(sc.S.astype(np.complex64)),
                  grids=db.generateTransformGrids(N, N, cent, sh=1), ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    got = db.api.sampleEnergies(y, x, E, db.Struct(Mb=Mb, Mbe=ctx.upload(Mbe)), ctx=ctx)
    ref = oe.computeEnergy(y.astype(np.complex128), x.astype(np.complex128), Eo, EH=OStruct(Mb=Mb, Mbe=Mbe),
                           per_sample=True)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


def test_shot_weights_map_to_samples_and_outer_samples_keep_one():
    mSt = np.array([0, 0, 1, 2, 2, 3, 3], np.int32)  # 3 shots, then the outer segment
    w = recon._sample_weights(np.array([1.0, 0.25, 0.5]), mSt, 3)
    assert w.dtype == np.float32 and list(w) == [1.0, 1.0, 0.25, 0.5, 0.5, 1.0, 1.0]
