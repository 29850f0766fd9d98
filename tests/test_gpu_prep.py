"""GPU tests of the data-preparation entry points and of the aligned
reconstruction driver on a small scan with known motion."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    return db.Context(0)


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize("Nin,Nout", [((16, 12, 10), (8, 6, 5)), ((15, 16, 9), (30, 20, 11)),
                                      ((64, 64, 44), (128, 128, 88)), ((128, 96, 20), (64, 48, 20))])
def test_resampling(ctx, Nin, Nout):
    import disorder_b200 as db
    from oracle.prep import resampling
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(Nin) + 1j * rng.standard_normal(Nin)).astype(np.complex64)
    r = db.resampling(x, Nout, ctx=ctx)
    ro = resampling(x.astype(np.complex128), Nout)
    assert rel(r, ro) < 1e-5


def test_compress_coils(ctx):
    import disorder_b200 as db
    from oracle.prep import compressCoils
    from disorder_b200 import synth
    rng = np.random.default_rng(4)
    N = (24, 20, 16)
    S = synth.coil_maps(N, 12, rng)
    S = S + 0.05 * (rng.standard_normal(S.shape) + 1j * rng.standard_normal(S.shape)).astype(np.complex64)
    y = (rng.standard_normal((300, 16, 12)) + 1j * rng.standard_normal((300, 16, 12))).astype(np.complex64)
    So, yo, C, D, U = db.compressCoils(S, 0.95, y, ctx=ctx)
    So_o, yo_o, Co, Do, Uo, P = compressCoils(S.astype(np.complex128), [0.95], y.astype(np.complex128))
    assert C == Co[0]
    assert np.allclose(D, Do, rtol=1e-4, atol=1e-6 * Do[0])
    # the kept subspace is unique; the phases of the singular vectors are not
    Pk = U[:, :C] @ U[:, :C].conj().T
    Po = Uo[:, :C] @ Uo[:, :C].conj().T
    assert np.max(np.abs(Pk - Po)) < 1e-4
    # compressed data are A S with A = U(:,1:C)^H
    A = U[:, :C].conj().T
    assert rel(So, np.tensordot(S, A, axes=([3], [1]))) < 1e-5
    assert rel(yo, np.tensordot(y, A, axes=([2], [1]))) < 1e-5


def test_precondition_and_gather(ctx):
    import disorder_b200 as db
    rng = np.random.default_rng(6)
    S = (rng.standard_normal((8, 6, 4, 3)) + 1j * rng.standard_normal((8, 6, 4, 3))).astype(np.complex64)
    Se = db.precondition_weights(S, 1e-9, ctx=ctx)
    assert rel(Se, 1.0 / (np.sum(np.abs(S) ** 2, axis=3) + 1e-9)) < 1e-6
    y = (rng.standard_normal((50, 7, 3)) + 1j * rng.standard_normal((50, 7, 3))).astype(np.complex64)
    idx = np.array([3, 0, 49, 7], np.int32)
    g = db.gather_samples(y, idx, 0.5, ctx=ctx)
    assert rel(g, 0.5 * y[idx]) < 1e-7


def test_level_sampling_matches_centred_crop():
    from disorder_b200 import recon, synth
    rng = np.random.default_rng(2)
    H = synth.random_checkered((32, 32), 16, rng)
    ky, kz, nEc, mSt, src = recon.level_sampling(H, 16, (16, 16))
    kyf, kzf, nEcf, mStf, iSt = synth.sample_lists(H, 16)
    # every level sample maps to a full sample of the same shot and of the same
    # signed frequency
    sf = lambda j, n: ((j + n // 2) % n) - n // 2  # noqa: E731
    assert np.array_equal(mStf[src], mSt)
    assert np.array_equal([sf(a, 32) for a in kyf[src]], [sf(a, 16) for a in ky])
    assert np.array_equal([sf(a, 32) for a in kzf[src]], [sf(a, 16) for a in kz])
    assert len(src) == 16 * 16


def test_aligned_reconstruction_recovers_motion(ctx):
    import disorder_b200 as db
    from disorder_b200 import recon, synth
    N, C, S = (32, 32, 24), 8, 16
    sc = synth.make_scan(N, C, S, 4.0, 2.0, 40.0, 8, seed=123)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    Sd = ctx.upload(sc.S)
    E = db.Struct(Tr=sc.T_gt, NMs=S, NSe=S + 1, Sf=Sd, grids=db.generateTransformGrids(N, N, cent), ky=sc.ky,
                  kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    y = db.encode(sc.x_gt, E, ctx=ctx)
    y = synth.add_noise(y, sc.sigma, sc.noise_seed)
    yd = ctx.upload(y)
    # motion-corrected reconstruction
    x, T, log = recon.aligned_reconstruction(ctx, Sd, yd, sc.H, S, N, perc=C, resolMax=2.0)
    err = np.linalg.norm(x.numpy() - sc.x_gt) / np.linalg.norm(sc.x_gt)
    # uncorrected reconstruction for comparison
    E0 = E.copy(Tr=np.zeros_like(sc.T_gt))
    xu, _, _ = db.CGsolver(y, E0, None, None, None, None, None, 40, "Energy", 1e-4, ctx=ctx)
    err_u = np.linalg.norm(xu - sc.x_gt) / np.linalg.norm(sc.x_gt)
    assert err < 0.5 * err_u, (err, err_u)
    assert np.max(np.abs(T - sc.T_gt)[:, :3]) < 0.3
    assert np.degrees(np.max(np.abs(T - sc.T_gt)[:, 3:])) < 1.0
