"""GPU parity against the FP64 oracle at the shapes the benchmark runs.

The reconstruction benchmark runs 256x256x176 (final level), 128x128x88 and
64x64x44 with 16 coils and 64 shots; the kernels compiled for those line
lengths (256 = 16x16, 176 = 16x11, 128, 88, 64, 44) and the coil-stage passes
at 16 coils are compared here with the oracle on random inputs. At the full
size two motion states of a 64-shot random-checkered sampling are used, so
every segment has the benchmark's 1,024 samples per shot; the kernels are the
same for any state count. Tolerance: 1e-5 relative L2 for the operators (the
FP32 bar), 1e-4 for solver outputs.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_SOLVER = 1e-4


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    return db.Context(0)


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    # the oracle's FFTs on all host threads (same arithmetic as one thread)
    import os
    from oracle import grids as og
    old = og.WORKERS
    og.WORKERS = os.cpu_count() or 1
    yield
    og.WORKERS = old


def _problem(ctx, N, C, n_shots, n_keep, seed, rot=5.0, tr=5.0):
    """Random image and coils, the first n_keep shots of an n_shots
    random-checkered sampling as motion states; (device E, oracle E, x)."""
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle.encoding import Struct as OStruct
    from oracle.grids import generateTransformGrids as ogrids
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    S = (rng.standard_normal(N + (C,)) + 1j * rng.standard_normal(N + (C,))).astype(np.complex64)
    H = synth.random_checkered(N[:2], n_shots, rng)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, n_shots)
    nEc = nEc[:n_keep + 1]
    ky, kz, mSt = ky[:nEc[-1]], kz[:nEc[-1]], mSt[:nEc[-1]]
    T = synth.motion(n_keep, rot, tr, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    Ed = db.Struct(Tr=T, NMs=n_keep, NSe=n_keep, Sf=ctx.upload(S), grids=db.generateTransformGrids(N, N, cent),
                   ky=ky, kz=kz, nEc=nEc, mSt=mSt)
    Eo = OStruct(Tr=T, NMs=n_keep, NSe=n_keep, Sf=S.astype(np.complex128), ky=ky, kz=kz, nEc=nEc, mSt=mSt,
                 grids=ogrids(N, N, cent, sh=1), cent=cent)
    return Ed, Eo, x


@pytest.mark.parametrize("N,S", [((256, 256, 176), 2), ((128, 128, 88), 4), ((64, 64, 44), 8)])
def test_transform_at_benchmark_sizes(ctx, N, S):
    """Forward transform of one volume to S states and the inverse with the
    state sum (the 256-point and 176-point line passes at full size)."""
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle.grids import generateTransformGrids as ogrids
    from oracle.transform import precomputeFactorsSincRigidTransform as opf
    from oracle.transform import sincRigidTransform as ost
    rng = np.random.default_rng(sum(N))
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    T = synth.motion(S, 5.0, 5.0, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = db.generateTransformGrids(N, N, cent)
    et, _ = db.precomputeFactorsSincRigidTransform(grids, T, 1)
    y, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    og = ogrids(N, N, cent, sh=1)
    oet, _ = opf(og, T, 1, 0)
    yo = ost(x.astype(np.complex128).reshape(N + (1, 1)), oet, 1)[:, :, :, 0, :]
    assert rel(y, yo) < TOL
    eti, _ = db.precomputeFactorsSincRigidTransform(grids, T, 0)
    u = (rng.standard_normal(N + (S,)) + 1j * rng.standard_normal(N + (S,))).astype(np.complex64)
    back, _ = db.sincRigidTransform(u, eti, 0, sumR=1, ctx=ctx)
    oeti, _ = opf(og, T, 0, 0)
    backo = ost(u.astype(np.complex128)[:, :, :, None, :], oeti, 0, sumR=1)[:, :, :, 0, 0]
    assert rel(back, backo) < TOL


@pytest.mark.parametrize("stage", [0, 1])
@pytest.mark.parametrize("N,C,shots,S", [((256, 256, 176), 16, 64, 2), ((128, 128, 88), 8, 64, 4),
                                         ((64, 64, 44), 16, 64, 8)])
def test_operators_at_benchmark_sizes(ctx, N, C, shots, S, stage):
    """encode, decode (with We and Mb) and encodedecode (with We) against the
    oracle at the benchmark's line lengths and coil counts, with the coil
    stage as three passes over per-coil volumes (stage 0: expand, weighted /
    gather / scatter dim-2 pass, combine) or as per-tile sample sums and their
    adjoint (stage 1)."""
    import disorder_b200 as db
    from oracle import encoding as oenc
    Ed, Eo, x = _problem(ctx, N, C, shots, S, seed=N[0] + C)
    yo = oenc.encode(x.astype(np.complex128), Eo)
    rng = np.random.default_rng(3)
    we = rng.uniform(0.5, 1.5, yo.shape[0]).astype(np.float32)
    mb = rng.uniform(0.0, 1.0, N[2]).astype(np.float32)
    do = oenc.decode(yo, Eo.__class__(We=we.astype(np.float64), Mb=mb.astype(np.float64)), Eo)
    # encodedecode = decode(We .* encode(x)) without EH.Mb (encodedecode.m:125,133)
    edo = oenc.decode(yo * we.astype(np.float64)[:, None, None], None, Eo)
    ctx.set_tuning("coil_stage", stage)
    try:
        y = db.encode(x, Ed, ctx=ctx)
        d = db.decode(yo.astype(np.complex64), db.Struct(We=we, Mb=mb), Ed, ctx=ctx)
        ed = db.encodedecode(x, Ed, db.Struct(We=we), ctx=ctx)
    finally:
        ctx.set_tuning("coil_stage", 0)
    assert rel(y, yo) < TOL
    assert rel(d, do) < TOL
    assert rel(ed, edo) < TOL


def test_gradient_at_the_coarse_level(ctx):
    """sincRigidTransformGradient at 64x64x44 (the coarsest level, where LM
    runs over all 64 states)."""
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle.grids import generateTransformGrids as ogrids
    from oracle.transform import (precomputeFactorsSincRigidTransform, sincRigidTransform,
                                  sincRigidTransformGradient)
    N = (64, 64, 44)
    rng = np.random.default_rng(44)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    T = synth.motion(6, 5.0, 5.0, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    et, etg = db.precomputeFactorsSincRigidTransform(db.generateTransformGrids(N, N, cent), T, 1, 1)
    _, xB = db.sincRigidTransform(x, et, 1, ctx=ctx)
    G = db.sincRigidTransformGradient(xB, et, etg, ctx=ctx)
    oet, oetg = precomputeFactorsSincRigidTransform(ogrids(N, N, cent, sh=1), T, 1, 1)
    _, oxB = sincRigidTransform(x.astype(np.complex128), oet, 1, keep_intermediates=True)
    oG = sincRigidTransformGradient(oxB, oet, oetg)
    for g in range(6):
        assert rel(G[..., g], oG[g][:, :, :, 0, :]) < TOL, g


def test_lm_at_the_coarse_level(ctx):
    """Two LMsolver iterations at 64x64x44 with 16 coils and 16 motion states
    (the seg_sums reduction and the damped solves at the coarse level)."""
    import disorder_b200 as db
    from oracle import encoding as oenc
    from oracle import solvers as osol
    N = (64, 64, 44)
    Ed, Eo, x = _problem(ctx, N, 16, 16, 16, seed=64)
    y = oenc.encode(x.astype(np.complex128), Eo)
    S = Eo.NMs
    common = dict(Tr=np.zeros_like(Eo.Tr), cT=np.zeros(S, bool), w=np.full(S, 1e-3, np.float32), winit=1e-3,
                  tL=[0.05, 0.02], nF=np.arange(0, 29))
    Edl, Eol = Ed.copy(**common), Eo.copy(**common)
    for it in range(2):
        Edl = db.LMsolver(y.astype(np.complex64), Edl, x, ctx=ctx)
        Eol = osol.LMsolver(y, Eol.copy(Sf=Eo.Sf), x.astype(np.complex128))
        assert np.array_equal(Edl.cT, Eol.cT), it
        assert rel(Edl.Tr, Eol.Tr) < TOL_SOLVER, it
        assert rel(Edl.En, Eol.En) < TOL_SOLVER, it


@pytest.mark.parametrize("tolType,nIt", [("RelativeResidual2Error", 4), ("Energy", 5)])
def test_cg_with_constraint_and_tikhonov(ctx, tolType, nIt):
    """CGsolver with every operator argument set: A.Se (precondition.m:19-23),
    C.Ma (constrain.m:12) and R.Ti (regularize.m:24), from an initial guess."""
    import disorder_b200 as db
    from oracle import encoding as oenc
    from oracle import solvers as osol
    N = (44, 44, 22)
    Ed, Eo, x = _problem(ctx, N, 4, 16, 4, seed=7)
    y = oenc.encode(x.astype(np.complex128), Eo)
    rng = np.random.default_rng(8)
    Se = (1.0 / (np.sum(np.abs(Eo.Sf) ** 2, axis=3) + 1e-9)).astype(np.float32)
    Ma = (rng.uniform(size=N) > 0.2).astype(np.float32)
    Ti = rng.uniform(0.05, 0.5, N).astype(np.float32)
    mbe = (np.arange(N[2]) >= 3).astype(np.float32)
    x0 = (0.5 * x).astype(np.complex64)
    OS = Eo.__class__
    xg, Eng, nng = db.CGsolver(y.astype(np.complex64), Ed, db.Struct(Mbe=mbe), db.Struct(Se=Se),
                               db.Struct(Ma=Ma), db.Struct(Ti=Ti), x0, nIt, tolType, 0.0, ctx=ctx)
    xo, Eno, nno = osol.CGsolver(y, Eo, OS(Mbe=mbe.astype(np.float64)), OS(Se=Se.astype(np.float64)),
                                 OS(Ma=Ma.astype(np.float64)), OS(Ti=Ti.astype(np.float64)),
                                 x0.astype(np.complex128), nIt, tolType, 0.0)
    assert nng == nno
    assert rel(xg, xo) < TOL_SOLVER
    if tolType == "Energy":
        assert rel(Eng, Eno) < TOL_SOLVER
