"""GPU parity of libdisorder (through the C ABI) against the FP64 CPU oracle.

Tolerance: the FP32 path must match the FP64 oracle to 1e-5 relative L2
error on the transform and encoded k-space (the FP32 bar); solver
outputs after several iterations use 1e-4 (iteration amplifies rounding).
"""

import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_SOLVER = 1e-4


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    return db.Context(0)


def _grids(N):
    import disorder_b200 as db
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    return db.generateTransformGrids(N, N, cent, sh=1)


def _ogrids(N):
    from oracle.grids import generateTransformGrids
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    return generateTransformGrids(N, N, cent, sh=1)


def _vol(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _oracle_fwd(x, N, T, di=1, sumR=1, useFull=1):
    from oracle.transform import precomputeFactorsSincRigidTransform, sincRigidTransform
    et, _ = precomputeFactorsSincRigidTransform(_ogrids(N), T.astype(np.float32), di, 0)
    x5 = x.astype(np.complex128)
    if x5.ndim == 4:
        x5 = x5[:, :, :, None, :]
    return sincRigidTransform(x5, et, di, sumR=sumR, useFull=useFull)


def _motion(rng, S, rot=5.0, tr=3.0):
    T = np.zeros((S, 6), np.float32)
    T[:, :3] = rng.uniform(-tr, tr, (S, 3))
    T[:, 3:] = np.radians(rng.uniform(-rot, rot, (S, 3)))
    return T


@pytest.mark.parametrize("di", [1, 0])
def test_precompute_factors(ctx, di):
    """et of precomputeFactorsSincRigidTransform as device arrays, against the
    oracle (rotations beyond 90 degrees for the flip flags)."""
    import disorder_b200 as db
    from oracle.transform import precomputeFactorsSincRigidTransform as opf
    N = (24, 20, 16)
    rng = np.random.default_rng(41)
    T = _motion(rng, 5)
    T[1, 3] = np.radians(120.0)
    T[3, 5] = np.radians(-100.0)
    et, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, di)
    got = et.arrays(ctx)
    ref, _ = opf(_ogrids(N), T, di, 0)
    for m in range(3):
        assert np.array_equal(got["flip"][m], ref.flip[m])
        assert rel(got["e1"][m], np.squeeze(ref.e1[m])) < TOL
        assert rel(got["e2"][m], np.squeeze(ref.e2[m])) < TOL
        assert rel(got["e3"][m], np.squeeze(ref.e3[m])) < TOL


def test_upload_download_round_trip(ctx):
    import ctypes as C
    a = np.random.default_rng(2).standard_normal(1000).astype(np.float32)
    d = C.c_void_p()
    ctx.check(ctx.lib.disorder_upload(ctx.h, a.ctypes.data, a.nbytes, C.byref(d)))
    b = np.zeros_like(a)
    ctx.check(ctx.lib.disorder_download(ctx.h, d, b.ctypes.data, b.nbytes))
    ctx.check(ctx.lib.disorder_free(ctx.h, d))
    assert np.array_equal(a, b)


GRID_SIZES = [(16, 12, 10), (32, 32, 24), (44, 40, 30), (96, 20, 12), (20, 160, 8), (64, 64, 44)]


@pytest.mark.parametrize("N", GRID_SIZES)
def test_forward_transform(ctx, N):
    import disorder_b200 as db
    rng = np.random.default_rng(sum(N))
    x = _vol(rng, N)
    T = _motion(rng, 3)
    et, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, 1)
    y, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    ref = _oracle_fwd(x, N, T)[:, :, :, 0, :]
    assert rel(y, ref) < TOL


@pytest.mark.parametrize("useFull", [0, -1])
def test_forward_partial(ctx, useFull):
    import disorder_b200 as db
    N = (24, 20, 16)
    rng = np.random.default_rng(7)
    x = _vol(rng, N)
    T = _motion(rng, 2)
    et, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, 1)
    y, _ = db.sincRigidTransform(x, et, 1, useFull=useFull, ctx=ctx)
    ref = _oracle_fwd(x, N, T, useFull=useFull)[:, :, :, 0, :]
    assert rel(y, ref) < TOL


@pytest.mark.parametrize("sumR", [1, 0])
def test_inverse_transform(ctx, sumR):
    import disorder_b200 as db
    N = (32, 24, 20)
    rng = np.random.default_rng(11)
    T = _motion(rng, 4)
    u = _vol(rng, N + (4,))
    et, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, 0)
    y, _ = db.sincRigidTransform(u, et, 0, sumR=sumR, ctx=ctx)
    ref = _oracle_fwd(u, N, T, di=0, sumR=sumR)
    ref = ref[:, :, :, 0, 0] if sumR else ref[:, :, :, 0, :]
    assert rel(y, ref) < TOL


def test_flip_branch(ctx):
    import disorder_b200 as db
    N = (16, 16, 12)
    rng = np.random.default_rng(3)
    x = _vol(rng, N)
    T = np.array([[0.5, 0.2, -0.3, 2.2, 0.1, -0.05], [0.0, 0.0, 0.0, 0.05, -1.9, 0.02],
                  [0.1, 0.0, 0.0, 0.02, 0.03, 2.7]], np.float32)
    et, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, 1)
    y, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    ref = _oracle_fwd(x, N, T)[:, :, :, 0, :]
    assert rel(y, ref) < TOL
    eti, _ = db.precomputeFactorsSincRigidTransform(_grids(N), T, 0)
    back, _ = db.sincRigidTransform(y, eti, 0, sumR=0, ctx=ctx)
    refb = _oracle_fwd(ref, N, T, di=0, sumR=0)[:, :, :, 0, :]
    assert rel(back, refb) < TOL


@pytest.mark.parametrize("N", [(16, 12, 10), (32, 28, 22)])
def test_gradient(ctx, N):
    import disorder_b200 as db
    from oracle.transform import (precomputeFactorsSincRigidTransform, sincRigidTransform,
                                  sincRigidTransformGradient)
    rng = np.random.default_rng(5)
    x = _vol(rng, N)
    T = _motion(rng, 3)
    et, etg = db.precomputeFactorsSincRigidTransform(_grids(N), T, 1, 1)
    _, xB = db.sincRigidTransform(x, et, 1, ctx=ctx)
    G = db.sincRigidTransformGradient(xB, et, etg, ctx=ctx)
    oet, oetg = precomputeFactorsSincRigidTransform(_ogrids(N), T, 1, 1)
    _, oxB = sincRigidTransform(x.astype(np.complex128), oet, 1, keep_intermediates=True)
    oG = sincRigidTransformGradient(oxB, oet, oetg)
    for g in range(6):
        assert rel(G[..., g], oG[g][:, :, :, 0, :]) < TOL, g


def _E_pair(ctx, N, C, S, seed, motion=True):
    """(product E, oracle E, scan) on the same inputs."""
    import disorder_b200 as db
    sc, Eo = make_problem(N=N, C=C, S=S, seed=seed, dtype=np.complex128, zero_motion=not motion)
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    Ed = db.Struct(Tr=Eo.Tr, NMs=Eo.NMs, NSe=Eo.NSe, Sf=ctx.upload(sc.S.astype(np.complex64)),
                   grids=db.generateTransformGrids(N, N, cent, sh=1), ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    return Ed, Eo, sc


@pytest.mark.parametrize("N,C,S", [((16, 16, 12), 4, 4), ((32, 32, 20), 3, 16), ((44, 44, 22), 2, 4),
                                   ((24, 24, 10), 2, 9)])
def test_encode_decode_encodedecode(ctx, N, C, S):
    import disorder_b200 as db
    from oracle import encoding as oenc
    Ed, Eo, sc = _E_pair(ctx, N, C, S, seed=21)
    x = sc.x_gt
    y = db.encode(x, Ed, ctx=ctx)
    yo = oenc.encode(x.astype(np.complex128), Eo)
    assert rel(y, yo) < TOL
    rng = np.random.default_rng(2)
    we = rng.uniform(0.5, 1.5, yo.shape[0]).astype(np.float32)
    mb = rng.uniform(0.0, 1.0, N[2]).astype(np.float32)
    EH = db.Struct(We=we, Mb=mb)
    d = db.decode(yo.astype(np.complex64), EH, Ed, ctx=ctx)
    do = oenc.decode(yo, Eo.__class__(We=we.astype(np.float64), Mb=mb.astype(np.float64)), Eo)
    assert rel(d, do) < TOL
    ed = db.encodedecode(x, Ed, db.Struct(We=we), ctx=ctx)
    edo = oenc.encodedecode(x.astype(np.complex128), Eo, Eo.__class__(We=we.astype(np.float64)))
    assert rel(ed, edo) < TOL


def test_no_motion_and_outer_segment(ctx):
    import disorder_b200 as db
    from oracle import encoding as oenc
    N = (16, 16, 8)
    Ed, Eo, sc = _E_pair(ctx, N, 2, 4, seed=5, motion=False)
    y = db.encode(sc.x_gt, Ed, ctx=ctx)
    assert rel(y, oenc.encode(sc.x_gt.astype(np.complex128), Eo)) < TOL
    # move the last shot to the untransformed outer segment (NMs = 3)
    Ed2, Eo2, sc2 = _E_pair(ctx, N, 2, 4, seed=5, motion=True)
    T3 = Eo2.Tr[:3]
    Ed2.Tr, Ed2.NMs = T3, 3
    Eo2 = Eo2.copy(Tr=T3, NMs=3)
    y2 = db.encode(sc2.x_gt, Ed2, ctx=ctx)
    assert rel(y2, oenc.encode(sc2.x_gt.astype(np.complex128), Eo2)) < TOL
    d2 = db.decode(y2, None, Ed2, ctx=ctx)
    assert rel(d2, oenc.decode(y2.astype(np.complex128), None, Eo2)) < TOL


def test_adjointness_on_device(ctx):
    import disorder_b200 as db
    N = (24, 20, 16)
    Ed, Eo, sc = _E_pair(ctx, N, 3, 4, seed=8)
    rng = np.random.default_rng(9)
    x = _vol(rng, N)
    y = db.encode(x, Ed, ctx=ctx)
    v = _vol(rng, y.shape)
    lhs = np.vdot(v.astype(np.complex128), y.astype(np.complex128))
    rhs = np.vdot(db.decode(v, None, Ed, ctx=ctx).astype(np.complex128), x.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_compute_energy(ctx):
    import disorder_b200 as db
    from oracle import encoding as oenc
    N = (16, 16, 12)
    Ed, Eo, sc = _E_pair(ctx, N, 3, 4, seed=12)
    rng = np.random.default_rng(4)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    y = y + 0.01 * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape))
    mbe = (np.arange(N[2]) >= 4).astype(np.float32)
    ti = rng.uniform(0.1, 1.0, N).astype(np.float32)
    En = db.computeEnergy(y.astype(np.complex64), sc.x_gt, Ed, db.Struct(Ti=ti), db.Struct(Mbe=mbe), ctx=ctx)
    Eno = oenc.computeEnergy(y, sc.x_gt.astype(np.complex128), Eo, Eo.__class__(Ti=ti.astype(np.float64)),
                             Eo.__class__(Mbe=mbe.astype(np.float64)))
    assert abs(En[0] - Eno[0]) / Eno[0] < TOL
    assert abs(En[1] - Eno[1]) / Eno[1] < TOL


# (44, 44, 22) reaches the TMA weighted pass, which also emits the forward
# samples that CG's Energy tolerance tracks; (16, 16, 12) the separate gather
# tol 0 with an initial guess starts from one encode and one decode of the
# residual; a positive RelativeResidual2Error tolerance needs b = decode(y)
@pytest.mark.parametrize("tolType,nIt,N,we,tol", [("RelativeResidual2Error", 4, (16, 16, 12), False, 0.0),
                                                 ("RelativeResidual2Error", 4, (44, 44, 22), False, 1e-12),
                                                 ("Energy", 7, (16, 16, 12), False, 0.0),
                                                 ("Energy", 7, (44, 44, 22), False, 0.0),
                                                 ("Energy", 5, (44, 44, 22), True, 0.0)])
def test_cg(ctx, tolType, nIt, N, we, tol):
    import disorder_b200 as db
    from oracle import encoding as oenc
    from oracle import solvers as osol
    Ed, Eo, sc = _E_pair(ctx, N, 4, 4, seed=31)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    Se = (1.0 / (np.sum(np.abs(sc.S) ** 2, axis=3) + 1e-9)).astype(np.float32)
    mbe = (np.arange(N[2]) >= 3).astype(np.float32)
    x0 = 0.5 * sc.x_gt
    # per-sample weights (EH.We, the outlier rejection's soft shot weights)
    wsmp = np.random.default_rng(5).uniform(0.3, 1.0, y.shape[0]).astype(np.float32) if we else None
    EHd = db.Struct(Mbe=mbe, We=wsmp) if we else db.Struct(Mbe=mbe)
    EHo = (Eo.__class__(Mbe=mbe.astype(np.float64), We=wsmp.astype(np.float64)) if we
           else Eo.__class__(Mbe=mbe.astype(np.float64)))
    x, En, nn = db.CGsolver(y.astype(np.complex64), Ed, EHd, db.Struct(Se=Se), None, None, x0, nIt,
                            tolType, tol, ctx=ctx)
    xo, Eno, nno = osol.CGsolver(y, Eo, EHo, Eo.__class__(Se=Se.astype(np.float64)), None, None,
                                 x0.astype(np.complex128), nIt, tolType, tol)
    assert nn == nno
    assert rel(x, xo) < TOL_SOLVER
    if tolType == "Energy":
        assert En.shape == Eno.shape
        assert rel(En, Eno) < TOL_SOLVER


# CG can return its final sample residual (tracked, or encoded once at the
# end); it is compared relative to |y| because it shrinks as CG converges
@pytest.mark.parametrize("tolType,nIt,x_init", [("RelativeResidual2Error", 2, True), ("Energy", 5, True),
                                                ("RelativeResidual2Error", 3, False)])
def test_cg_residual_output(ctx, tolType, nIt, x_init):
    import disorder_b200 as db
    from oracle import encoding as oenc
    N = (44, 44, 22)
    Ed, Eo, sc = _E_pair(ctx, N, 4, 4, seed=31)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    Se = (1.0 / (np.sum(np.abs(sc.S) ** 2, axis=3) + 1e-9)).astype(np.float32)
    mbe = (np.arange(N[2]) >= 3).astype(np.float32)
    r = ctx.empty(y.shape)
    x, _, _ = db.CGsolver(y.astype(np.complex64), Ed, db.Struct(Mbe=mbe), db.Struct(Se=Se), None, None,
                          0.5 * sc.x_gt if x_init else None, nIt, tolType, 0.0, ctx=ctx, residual=r)
    ref = oenc.encode(np.asarray(x).astype(np.complex128), Eo) - y
    rg = r.numpy()
    assert np.linalg.norm(rg - ref) < TOL * np.linalg.norm(y)
    Re = db.api.residualSampleEnergies(r, Ed, db.Struct(Mbe=mbe), ctx=ctx)
    Re2 = db.api.sampleEnergies(y.astype(np.complex64), x, Ed, db.Struct(Mbe=mbe), ctx=ctx)
    assert rel(Re, Re2) < 1e-3


def test_lm_step(ctx):
    import disorder_b200 as db
    from oracle import encoding as oenc
    from oracle import solvers as osol
    N = (24, 24, 16)
    Ed, Eo, sc = _E_pair(ctx, N, 3, 4, seed=17)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    S = Eo.NMs
    common = dict(Tr=np.zeros_like(sc.T_gt), cT=np.zeros(S, bool), w=np.full(S, 1e-3, np.float32), winit=1e-3,
                  tL=[0.05, 0.02], nF=np.arange(3, 13))
    Edl = Ed.copy(**common)
    Eol = Eo.copy(**common)
    for it in range(3):
        Edl = db.LMsolver(y.astype(np.complex64), Edl, sc.x_gt, ctx=ctx)
        # the reference returns E with Sf cropped to nF; solveXT re-sets E.Sf
        # before every call (solveXT.m:498-503), so do the same here
        Eol = osol.LMsolver(y, Eol.copy(Sf=Eo.Sf), sc.x_gt.astype(np.complex128))
        assert np.array_equal(Edl.cT, Eol.cT), it
        assert rel(Edl.Tr, Eol.Tr) < TOL_SOLVER, (it, Edl.Tr, Eol.Tr)
        assert rel(Edl.w, Eol.w) < 1e-6
        assert rel(Edl.En, Eol.En) < TOL_SOLVER
    # the motion estimate moves towards the truth
    assert np.linalg.norm(Edl.Tr - sc.T_gt) < 0.5 * np.linalg.norm(sc.T_gt)
