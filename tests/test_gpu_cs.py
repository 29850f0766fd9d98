"""Compressed-sensing reconstruction on the GPU (disorder_b200.cs,
csrc/shearlet.cu) against the FP64 oracle (oracle/shearlet.py,
oracle/solvers.py::CSsolver): computeShearlet, the shearlet regularizer
(Reconstruction/regularize.m:27-46), both trace estimates
(Reconstruction/traceEstimation.m), the CG with the shearlet term and the
whole CSsolver (Reconstruction/CSsolver.m) with the same trace probes."""

import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu

N = (40, 36, 36)
C, S = 4, 8
TOL = 1e-5
TOL_SOLVER = 1e-4


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


@pytest.fixture(scope="module")
def env():
    import disorder_b200 as db
    from disorder_b200 import cs
    from oracle import shearlet as osh
    ctx = db.Context(0)
    sc, Eo = make_problem(N=N, C=C, S=S, seed=17, dtype=np.complex128)
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    Ed = db.Struct(Tr=Eo.Tr, NMs=Eo.NMs, NSe=Eo.NSe, Sf=ctx.upload(sc.S.astype(np.complex64)),
                   grids=db.generateTransformGrids(N, N, cent, sh=1), ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    return db, cs, osh, ctx, sc, Ed, Eo, cs.ShearletSystem(ctx, N), osh.buildShearlet(list(N), 1, [1])["S"]


def _vol(rng):
    return (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)


def _probes(seed, n=8):
    rng = np.random.default_rng(seed)
    ps = [rng.standard_normal(N).astype(np.float32) for _ in range(n)]
    it = iter(ps)
    return lambda shape: next(it)


def test_coefficients_and_regularizer(env):
    db, cs, osh, ctx, sc, Ed, Eo, sysd, So = env
    rng = np.random.default_rng(1)
    x, u = _vol(rng), _vol(rng)
    We = sysd.coefficients(ctx.upload(x), 1e-2, 1.0)
    Weo = (osh.compute_shearlet(x.astype(np.complex128), So) + 1e-2) ** -1.0
    assert We.shape == N + (50,)
    assert rel(We.numpy(), Weo) < TOL
    Wh = We.numpy().astype(np.float64)
    r = sysd.regularize(ctx.upload(u), We, 0.7)
    ro = osh.regularize_sh(u.astype(np.complex128), So, Wh, 0.7)
    assert rel(r.numpy(), ro) < TOL
    # out = beta out + ... (the CG adds the term to its normal operator)
    base = _vol(rng)
    out = ctx.upload(base)
    sysd.regularize(ctx.upload(u), We, 0.7, out=out, beta=1.0)
    assert rel(out.numpy(), base + ro) < TOL


def test_trace_estimates(env):
    db, cs, osh, ctx, sc, Ed, Eo, sysd, So = env
    rng = np.random.default_rng(2)
    we = rng.uniform(0.5, 1.5, sc.ky.size).astype(np.float32)
    tr, trF = cs.traceEstimation(ctx, N, Ed, db.Struct(We=we), None, None, 1e-2, 4, noise=_probes(3))
    tro, trFo = osh.trace_estimation(np.zeros(N), Eo, Eo.__class__(We=we.astype(np.float64)), None, None, 1e-2, 4,
                                     noise=_probes(3))
    assert len(trF) == len(trFo) and rel(trF, trFo) < TOL
    We = sysd.coefficients(ctx.upload(_vol(rng)), 1e-2, 1.0)
    Rd = db.Struct(Sh=db.Struct(sys=sysd, We=We))
    Ro = Eo.__class__(Sh=Eo.__class__(S=So, We=We.numpy().astype(np.float64)))
    mask = (rng.uniform(size=N) > 0.2).astype(np.float32)
    tr, trF = cs.traceEstimation(ctx, N, None, None, db.Struct(Ma=mask), Rd, 1e-2, 4, noise=_probes(4))
    tro, trFo = osh.trace_estimation(np.zeros(N), None, None, Eo.__class__(Ma=mask.astype(np.float64)), Ro, 1e-2, 4,
                                     noise=_probes(4))
    assert len(trF) == len(trFo) and rel(trF, trFo) < TOL


def test_cg_with_the_shearlet_term(env):
    db, cs, osh, ctx, sc, Ed, Eo, sysd, So = env
    from oracle import encoding as oenc
    from oracle import solvers as osol
    rng = np.random.default_rng(5)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    we = rng.uniform(0.5, 1.5, y.shape[0]).astype(np.float32)
    Ti = np.full(N, 2e-3, np.float32)
    Se = (1.0 / (np.sum(np.abs(sc.S) ** 2, axis=3) + Ti + 0.35)).astype(np.float32)
    x0 = (0.8 * sc.x_gt).astype(np.complex64)
    We = sysd.coefficients(ctx.upload(x0), 1e-2, 1.0)
    Rd = db.Struct(Ti=Ti, Sh=db.Struct(sys=sysd, We=We, la=0.7, p=1.0))
    O = Eo.__class__
    Ro = O(Ti=Ti.astype(np.float64), Sh=O(S=So, We=We.numpy().astype(np.float64), la=0.7, p=1.0))
    x, _, nn = db.CGsolver(y.astype(np.complex64), Ed, db.Struct(We=we), db.Struct(Se=Se), None, Rd, x0, 3, "None",
                           0.0, ctx=ctx)
    xo, _, nno = osol.CGsolver(y, Eo, O(We=we.astype(np.float64)), O(Se=Se.astype(np.float64)), None, Ro,
                               x0.astype(np.complex128), 3, "None", 0.0)
    assert nn == nno == 3
    assert rel(x, xo) < TOL_SOLVER
    # the term changes the solution: without it CG lands elsewhere
    xn, _, _ = db.CGsolver(y.astype(np.complex64), Ed, db.Struct(We=we), db.Struct(Se=Se), None, db.Struct(Ti=Ti),
                           x0, 3, "None", 0.0, ctx=ctx)
    assert rel(xn, xo) > 10 * TOL_SOLVER


def test_cssolver_against_the_oracle(env):
    db, cs, osh, ctx, sc, Ed, Eo, sysd, So = env
    from oracle import encoding as oenc
    from oracle import solvers as osol
    rng = np.random.default_rng(6)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    y = y + 0.02 * np.linalg.norm(y) / np.sqrt(y.size) * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape))
    we = rng.uniform(0.5, 1.5, y.shape[0]).astype(np.float32)
    Ti = np.full(N, 1e-3, np.float32)
    x0 = (0.9 * sc.x_gt).astype(np.complex64)
    O = Eo.__class__
    x, lam = cs.CSsolver(y.astype(np.complex64), Ed, db.Struct(We=we), None, None, db.Struct(Ti=Ti), x0, tol=1e-5,
                         ctx=ctx, noise=_probes(8, 24), system=sysd)
    xo, lamo = osol.CSsolver(y, Eo, O(We=we.astype(np.float64)), None, None, O(Ti=Ti.astype(np.float64)),
                             x0.astype(np.complex128), tol=1e-5, noise=_probes(8, 24))
    print("CSsolver: lambda", lam, "oracle", lamo, "image rel err %.2e" % rel(x.numpy(), xo))
    assert lam[2] == 0 and lamo[2] == 0
    assert rel(lam[:2], lamo[:2]) < TOL_SOLVER
    assert rel(x.numpy(), xo) < TOL_SOLVER
    assert np.all(np.isfinite(x.numpy()))


def test_device_probes(env):
    db, cs, osh, ctx, sc, Ed, Eo, sysd, So = env
    V = int(np.prod(N))
    a, b = ctx.empty(N, np.float32), ctx.empty(N, np.float32)
    for d in (a, b):
        ctx.check(ctx.lib.disorder_trace_probe(ctx.h, V, 1234, None, d.ptr))
    pa, pb = a.numpy(), b.numpy()
    assert np.array_equal(pa, pb)  # a function of (seed, index) only
    assert abs(np.mean(pa.astype(np.float64) ** 2) - 1) < 1e-5  # traceEstimation.m:55
    assert abs(np.mean(pa)) < 0.02 and 0.9 < np.std(pa) < 1.1
    mask = (np.random.default_rng(9).uniform(size=N) > 0.5).astype(np.float32)
    ctx.check(ctx.lib.disorder_trace_probe(ctx.h, V, 1234, ctx.upload(mask).ptr, b.ptr))
    assert np.allclose(b.numpy(), pa * mask, rtol=1e-6, atol=0)
    ctx.check(ctx.lib.disorder_trace_probe(ctx.h, V, 99, None, b.ptr))
    assert not np.allclose(b.numpy(), pa)
    # with device probes the estimates agree with the host-probe ones to their
    # statistical spread
    we = np.ones(sc.ky.size, np.float32)
    t_dev, _ = cs.traceEstimation(ctx, N, Ed, db.Struct(We=we), None, None, 1e-2, 4, rng=np.random.default_rng(1))
    t_host, _ = cs.traceEstimation(ctx, N, Ed, db.Struct(We=we), None, None, 1e-2, 4, noise=_probes(3))
    assert abs(t_dev / t_host - 1) < 0.03


@pytest.mark.parametrize("Nf", [(64, 64, 44), (64, 96, 88), (256, 36, 40), (40, 176, 36), (36, 40, 128)])
def test_register_fft_passes(Nf):
    """Lengths with a fast factorisation take the register-FFT pass kernel:
    64 = 8 x 8, 44 = 4 x 11, 88 = 8 x 11 (shearlet_fb.cu) and 256 = 16 x 16,
    176 = 16 x 11, 128 = 16 x 8 (shearlet_fa.cu, the benchmark's lengths),
    each on the contiguous axis or a strided one; 96, 40 and 36 take the
    generic kernel."""
    import disorder_b200 as db
    from disorder_b200 import cs
    from oracle import shearlet as osh
    ctx = db.Context(0)
    rng = np.random.default_rng(12)
    x = (rng.standard_normal(Nf) + 1j * rng.standard_normal(Nf)).astype(np.complex64)
    u = (rng.standard_normal(Nf) + 1j * rng.standard_normal(Nf)).astype(np.complex64)
    sysd = cs.ShearletSystem(ctx, Nf)
    So = osh.buildShearlet(list(Nf), 1, [1])["S"]
    We = sysd.coefficients(ctx.upload(x), 1e-2, 1.0)
    Weo = (osh.compute_shearlet(x.astype(np.complex128), So) + 1e-2) ** -1.0
    assert rel(We.numpy(), Weo) < TOL
    Wh = We.numpy().astype(np.float64)
    r = sysd.regularize(ctx.upload(u), We, 0.3)
    assert rel(r.numpy(), osh.regularize_sh(u.astype(np.complex128), So, Wh, 0.3)) < TOL
    probe = rng.standard_normal(Nf).astype(np.float32)
    t = sysd.trace(ctx.upload(probe), We)
    pF = np.fft.fftn(probe.astype(np.complex128))
    to = sum(float(np.sum(Wh[..., w] * np.abs(np.fft.ifftn(np.conj(So[..., w]) * pF)) ** 2)) for w in range(So.shape[-1]))
    assert abs(t / to - 1) < TOL
