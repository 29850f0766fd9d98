"""Known-answer tests that pin the CPU oracle (no GPU).

The reference (MATLAB) cannot run here and ships no golden vectors, so the
oracle is pinned by properties the reference algorithm must satisfy exactly.
"""

import numpy as np
import pytest

from conftest import make_problem
from oracle import encoding as enc
from oracle import prep, solvers
from oracle.encoding import Struct
from oracle.grids import generateTransformGrids
from oracle.transform import (precomputeFactorsSincRigidTransform, restrictTransform,
                              sincRigidTransform, sincRigidTransformGradient, wrapToPi,
                              wrapToPiHalf)


def _grids(N):
    cent = [np.ceil((n + 1) / 2.0) for n in N]
    return generateTransformGrids(N, N, cent, sh=1)


def _vol(rng, N):
    return (rng.standard_normal(N) + 1j * rng.standard_normal(N))


def _fwd(x, g, T, **kw):
    et, _ = precomputeFactorsSincRigidTransform(g, np.asarray(T, np.float32), 1, 0)
    return sincRigidTransform(x, et, 1, **kw)


def _inv(x, g, T, sumR=1):
    et, _ = precomputeFactorsSincRigidTransform(g, np.asarray(T, np.float32), 0, 0)
    return sincRigidTransform(x, et, 0, sumR=sumR)


def test_wraps():
    x = np.array([-7.0, -np.pi, -1.0, 0.0, 2.0, np.pi, 4.0, 3 * np.pi])
    w = wrapToPi(x)
    assert np.all(w >= -np.pi) and np.all(w <= np.pi)
    assert w[5] == np.pi and w[7] == pytest.approx(np.pi)
    assert np.allclose(np.exp(1j * w), np.exp(1j * x))
    h = wrapToPiHalf(np.array([0.1, 2.0, -2.0, 3.0]))
    assert np.all(np.abs(h) <= np.pi / 2 + 1e-12)
    T = np.zeros((2, 6), np.float32)
    T[:, 3] = [4.0, -4.0]
    assert np.all(np.abs(restrictTransform(T)[:, 3]) <= np.pi)


def test_identity_at_zero(rng):
    N = (12, 10, 8)
    g = _grids(N)
    x = _vol(rng, N)
    y = _fwd(x, g, np.zeros((1, 6)))
    assert np.max(np.abs(y[..., 0, 0] - x)) < 1e-12


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_integer_translation_is_circshift(rng, axis):
    N = (12, 10, 8)
    g = _grids(N)
    x = _vol(rng, N)
    T = np.zeros((1, 6))
    T[0, axis] = 3
    y = _fwd(x, g, T)[..., 0, 0]
    # the grids are single precision in the reference (generateGrid.m:35), so
    # the phase ramp is exact only to single rounding of 2*pi*q/N
    assert np.max(np.abs(y - np.roll(x, 3, axis=axis))) < 2e-6


@pytest.mark.parametrize("m", [0, 1, 2])
def test_quarter_turn_is_exact_permutation(rng, m):
    # With an even grid centred on an integer voxel the three shears of a
    # 90 degree rotation shift every line by an integer number of voxels.
    N = (8, 8, 8)
    g = _grids(N)
    x = _vol(rng, N)
    T = np.zeros((1, 6), np.float32)
    # single(pi/2) rounds above pi/2, which the reference's wrapToPi sends to
    # the >90 degree flipping branch; take the largest single below pi/2
    T[0, 3 + m] = np.nextafter(np.float32(np.pi / 2), np.float32(0))
    y = _fwd(x, g, T)[..., 0, 0]
    # every output value is one of the input values, exactly (a permutation)
    # (to the single-precision rounding of the reference's grids)
    d = np.abs(y.ravel()[:, None] - x.ravel()[None, :])
    assert np.max(np.min(d, axis=1)) < 1e-5
    assert len(set(np.argmin(d, axis=1))) == x.size
    # and applying it four times gives back the input
    z = x
    for _ in range(4):
        z = _fwd(z, g, T)[..., 0, 0]
    assert np.max(np.abs(z - x)) < 4e-5


def test_unitary_and_adjoint(rng):
    N = (12, 10, 8)
    g = _grids(N)
    x = _vol(rng, N)
    T = np.array([[0.7, -1.3, 0.4, 0.05, -0.08, 0.11], [-0.2, 0.5, 1.1, -0.03, 0.02, 0.07]])
    y = _fwd(x, g, T)
    # T^H T = I per state
    for s in range(2):
        back = _inv(y[..., s:s + 1], g, T[s:s + 1])
        assert np.max(np.abs(back[..., 0, 0] - x)) < 1e-10
    # <T x, v> = <x, T^H v> with the state sum
    v = _vol(rng, N + (1, 2))
    lhs = np.vdot(v, y)
    rhs = np.vdot(_inv(v, g, T)[..., 0, 0], x)
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)


def test_flip_branch_is_consistent(rng):
    # rotations beyond 90 degrees take the flipping branch
    N = (8, 8, 6)
    g = _grids(N)
    x = _vol(rng, N)
    T = np.array([[0.0, 0.0, 0.0, 2.5, 0.0, 0.0]])
    et, _ = precomputeFactorsSincRigidTransform(g, T.astype(np.float32), 1, 0)
    assert et.flip[0][0]
    y = _fwd(x, g, T)
    back = _inv(y, g, T)
    assert np.max(np.abs(back[..., 0, 0] - x)) < 1e-9


def test_gradient_matches_finite_differences(rng):
    N = (10, 8, 6)
    g = _grids(N)
    x = _vol(rng, N)
    T = np.array([[0.4, -0.3, 0.2, 0.06, -0.04, 0.05]])
    et, etg = precomputeFactorsSincRigidTransform(g, T.astype(np.float32), 1, 1)
    _, xB = sincRigidTransform(x, et, 1, keep_intermediates=True)
    G = sincRigidTransformGradient(xB, et, etg)
    for p in range(6):
        h = 1e-3
        Tp, Tm = T.copy(), T.copy()
        Tp[0, p] += h
        Tm[0, p] -= h
        etp, _ = precomputeFactorsSincRigidTransform(g, Tp, 1, 0, cGrid=None)
        etm, _ = precomputeFactorsSincRigidTransform(g, Tm, 1, 0, cGrid=None)
        # the factor routine rounds T to single; use the same rounded step
        hs = (np.float32(Tp[0, p]) - np.float32(Tm[0, p])) / 2
        fd = (sincRigidTransform(x, etp, 1) - sincRigidTransform(x, etm, 1)) / (2 * hs)
        rel = np.linalg.norm(fd - G[p]) / np.linalg.norm(G[p])
        assert rel < 2e-3, (p, rel)


def test_encode_rows_equals_fft():
    sc, E = make_problem(N=(8, 8, 6), C=3, S=4)
    x = sc.x_gt.astype(np.complex128)
    ya = enc.encode(x, E, method="rows")
    yb = enc.encode(x, E, method="fft")
    assert np.max(np.abs(ya - yb)) < 1e-12 * max(1, np.max(np.abs(ya)))
    we = np.random.default_rng(3).uniform(0.5, 1.5, ya.shape[0])
    EH = Struct(We=we)
    da = enc.decode(ya, EH, E, method="rows")
    db = enc.decode(ya, EH, E, method="fft")
    assert np.max(np.abs(da - db)) < 1e-11 * np.max(np.abs(da))
    ea = enc.encodedecode(x, E, EH, method="rows")
    eb = enc.encodedecode(x, E, EH, method="fft")
    assert np.max(np.abs(ea - eb)) < 1e-11 * np.max(np.abs(ea))


def test_encode_decode_adjoint_and_normal():
    sc, E = make_problem(N=(12, 10, 8), C=3, S=4)
    rng = np.random.default_rng(5)
    x = _vol(rng, sc.N)
    y = enc.encode(x, E)
    v = rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)
    we = rng.uniform(0.5, 1.5, y.shape[0])
    EH = Struct(We=we)
    lhs = np.vdot(v * we[:, None, None], y)
    rhs = np.vdot(enc.decode(v, EH, E), x)
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)
    # encodedecode == decode(encode(x)) (CGsolver.m:54-55 use either)
    ed = enc.encodedecode(x, E, EH)
    de = enc.decode(y, EH, E)
    assert np.max(np.abs(ed - de)) < 1e-10 * np.max(np.abs(ed))


def test_outer_segment_is_untransformed():
    sc, E = make_problem(N=(8, 8, 6), C=2, S=4)
    # move two samples of shot 1 into the outer (untransformed) segment
    ky, kz, nEc = sc.ky.copy(), sc.kz.copy(), sc.nEc.copy()
    nEc[1:-1] -= 0
    x = sc.x_gt.astype(np.complex128)
    y = enc.encode(x, E)
    E2 = E.copy(NSe=E.NMs)  # drop the (empty) outer segment
    assert np.allclose(enc.encode(x, E2), y)


def test_cg_monotone_and_converges():
    sc, E = make_problem(N=(8, 8, 6), C=4, S=4)
    y = enc.encode(sc.x_gt.astype(np.complex128), E)
    A = Struct(Se=1.0 / (np.sum(np.abs(E.Sf) ** 2, axis=3) + 1e-9))
    x, En, nn = solvers.CGsolver(y, E, None, A, None, None, None, 40, "Energy", 1e-9)
    assert np.all(np.diff(En.sum(axis=0)) <= 1e-12)
    err = np.linalg.norm(x - sc.x_gt) / np.linalg.norm(sc.x_gt)
    assert err < 1e-3, err
    x1, _, nn1 = solvers.CGsolver(y, E, None, A, None, None, np.zeros(sc.N), 5,
                                  "RelativeResidual2Error", 0)
    assert nn1 == 5


def test_lm_recovers_known_motion():
    sc, E = make_problem(N=(16, 16, 12), C=4, S=4, rot_deg=2.0, trans=1.5)
    x = sc.x_gt.astype(np.complex128)
    y = enc.encode(x, E)  # noise-free, true motion
    S = E.NMs
    Elm = E.copy(Tr=np.zeros_like(sc.T_gt), cT=np.zeros(S, bool), w=np.full(S, 1e-3), winit=1e-3,
                 tL=[1e-6, 1e-6])
    for _ in range(12):
        Elm = solvers.LMsolver(y, Elm, x)
    err = np.abs(Elm.Tr - sc.T_gt)
    assert err[:, :3].max() < 1e-3 and np.degrees(err[:, 3:]).max() < 1e-3, err


def test_lm_energy_never_increases():
    sc, E = make_problem(N=(12, 12, 8), C=3, S=4)
    x = sc.x_gt.astype(np.complex128)
    y = enc.encode(x, E)
    S = E.NMs
    Elm = E.copy(Tr=np.zeros_like(sc.T_gt), cT=np.zeros(S, bool), w=np.full(S, 1e-3), winit=1e-3,
                 tL=[0.05, 0.02], nF=np.arange(2, 8))
    Elm2 = solvers.LMsolver(y, Elm, x)
    assert np.all(Elm2.En <= Elm2.EnPrev + 1e-15)


def test_compress_coils_and_resampling():
    rng = np.random.default_rng(2)
    S = rng.standard_normal((6, 6, 4, 5)) + 1j * rng.standard_normal((6, 6, 4, 5))
    So, _, C, D, U, P = prep.compressCoils(S, [0.9])
    assert np.allclose(P, P.conj().T)
    assert So.shape[3] == C[0] and np.all(np.diff(D) <= 1e-12)
    x = _vol(rng, (8, 6, 4))
    up = prep.resampling(x, (16, 12, 8))
    down = prep.resampling(up, (8, 6, 4))
    assert np.max(np.abs(down - x)) < 1e-12
    resPyr, L, estT, resIso = prep.pyramidPlan([1, 1, 1], 4, 1, (1, 0))
    assert L == 3 and list(resPyr) == [0.25, 0.5, 1.0] and list(estT) == [1, 1, 0]
