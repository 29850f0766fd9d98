"""Shearlet systems (CPU): the device form of the system
(disorder_b200.shearlet: 2-D planes and a product table) against the FP64
oracle's 3-D system (oracle/shearlet.py, Shearlets/buildShearlet.m), the
index tables of Shearlets/getShearletIdxs.m, and properties of the oracle's
shearlet regularizer (Reconstruction/regularize.m:27-46)."""

import numpy as np
import pytest

from disorder_b200 import shearlet as sh
from oracle import shearlet as osh

N = (40, 36, 36)


@pytest.fixture(scope="module")
def systems():
    return osh.buildShearlet(list(N), 1, [1], "kos"), sh.build_planes(N, 1, [1], "kos")


def test_device_planes_give_the_oracle_system(systems):
    o, (planes, table, idxs) = systems
    S = o["S"]
    assert S.shape == N + (50,) and len(table) == 50
    assert np.array_equal(idxs, o["idxs"])
    worst = 0.0
    for w in range(len(table)):
        e = sh.expand(planes, table, N, w)
        worst = max(worst, np.linalg.norm(e - S[..., w]) / np.linalg.norm(S[..., w]))
    assert worst < 1e-6, worst


def test_index_tables():
    # 2-D full system at one scale of shear level 1: 2 cones x 5 shears + lowpass
    i2 = osh.shearlet_idxs(2, [1], 1)
    assert len(i2) == 11 and list(i2[-1]) == [0, 0, 0, 0]
    # 3-D: pyramid 1 all 25 shear pairs, pyramid 2 |sh2| < 2, pyramid 3 both < 2, lowpass
    i3 = osh.shearlet_idxs(3, [1], 0)
    assert len(i3) == 25 + 15 + 9 + 1
    assert len(osh.shearlet_idxs(3, [1], 1)) == 3 * 25 + 1
    assert np.array_equal(sh.shearlet_idxs(3, [1, 2], 0), osh.shearlet_idxs(3, [1, 2], 0))
    # the product table names planes of the 11-plane 2-D systems
    _, table, _ = sh.build_planes((40, 40, 40), 1, [1])
    assert table[:, [1, 3]].max() == 10 and set(table[:, 0]) | set(table[:, 2]) == {0, 1, 2}
    assert list(table[-1]) == [0, 10, 2, 10]


def test_small_grids_are_refused():
    # checkFilterFeasibility.m needs 33 samples per dimension for J = 1, K = [1]
    with pytest.raises(NotImplementedError):
        sh.build_planes((32, 40, 40), 1, [1])
    with pytest.raises(NotImplementedError):
        osh.buildShearlet([40, 40, 32], 1, [1])
    with pytest.raises(NotImplementedError):
        sh.build_planes((40, 40, 40), 1, [1], DFtype="dmaxflat4")


def test_oracle_system_structure(systems):
    o, _ = systems
    S = o["S"]
    # the lowpass passes DC with unit gain; the sum of squares (dual frame
    # weights) is positive everywhere, so every frequency is covered
    assert abs(S[0, 0, 0, -1] - 1) < 1e-12
    assert o["dfw"].min() > 0 and np.all(o["rms"] > 0)


def test_oracle_regularizer_is_hermitian_positive(systems):
    o, _ = systems
    rng = np.random.default_rng(4)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    z = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    We = (osh.compute_shearlet(rng.standard_normal(N), o["S"]) + 1e-2) ** -1.0
    Rx = osh.regularize_sh(x, o["S"], We, 0.8)
    Rz = osh.regularize_sh(z, o["S"], We, 0.8)
    assert abs(np.vdot(z, Rx) - np.conj(np.vdot(x, Rz))) < 1e-9 * abs(np.vdot(x, Rx))
    assert np.vdot(x, Rx).real > 0 and abs(np.vdot(x, Rx).imag) < 1e-9 * np.vdot(x, Rx).real


def test_oracle_trace_estimates_match_the_exact_traces():
    """traceEstimation.m estimates traces with Gaussian probes; both of its
    operators have closed-form traces to check the oracle against:
    - shearlet term: A_w = IDFT diag(conj S_w) DFT is circulant, so every row
      has squared norm mean_k |S_w(k)|^2 and tr = sum_w sum_v We_w(v) mean|S_w|^2;
    - fidelity term: F the unitary 2-D DFT, tr = mean_k W(k) sum_c sum_v |S_c(v)|^2."""
    from oracle.encoding import Struct
    Nt = (36, 36, 36)
    rng = np.random.default_rng(8)
    S = osh.buildShearlet(list(Nt), 1, [1])["S"]
    We = rng.uniform(0.2, 2.0, Nt + (S.shape[-1],))
    exact = float(np.sum(We.reshape(-1, We.shape[-1]).sum(0) * np.mean(np.abs(S.reshape(-1, S.shape[-1])) ** 2, 0)))
    pr = np.random.default_rng(9)
    draw = lambda shape: pr.standard_normal(shape)  # noqa: E731
    tr, trF = osh.trace_estimation(np.zeros(Nt), None, None, None, Struct(Sh=Struct(S=S, We=We)), 2e-3, 4, draw)
    se = np.std(trF, ddof=1) / np.sqrt(len(trF))
    assert abs(tr - exact) < 5 * se + 1e-3 * exact, (tr, exact, se)
    # fidelity term with coil maps and a weight grid over (ky, kz)
    Sf = rng.standard_normal(Nt + (3,)) + 1j * rng.standard_normal(Nt + (3,))
    ky, kz = np.meshgrid(np.arange(Nt[0]), np.arange(Nt[1]), indexing="ij")
    w = rng.uniform(0.0, 1.5, ky.size)
    E = Struct(Sf=Sf, ky=ky.ravel(), kz=kz.ravel())
    exact = float(np.mean(w) * np.sum(np.abs(Sf) ** 2))
    tr, trF = osh.trace_estimation(np.zeros(Nt), E, Struct(We=w), None, None, 2e-3, 4, draw)
    se = np.std(trF, ddof=1) / np.sqrt(len(trF))
    assert abs(tr - exact) < 5 * se + 1e-3 * exact, (tr, exact, se)


def test_oracle_cs_beats_cg_at_scanner_intensities():
    """CSsolver.m's epsil = 0.01 is an absolute intensity: with the unit-norm
    synthetic image scaled to scanner-like values (x 1e6), the shearlet
    reconstruction of a noisy scan improves on plain CG; at unit norm it
    over-smooths."""
    from conftest import make_problem
    from oracle import encoding as oenc
    from oracle import solvers as osol
    Nt = (40, 36, 36)
    sc, Eo = make_problem(N=Nt, C=4, S=8, seed=17, dtype=np.complex128, zero_motion=True)
    O = Eo.__class__
    rng = np.random.default_rng(6)
    y0 = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    y0 = y0 + 0.05 * np.linalg.norm(y0) / np.sqrt(y0.size) * (rng.standard_normal(y0.shape)
                                                                 + 1j * rng.standard_normal(y0.shape))
    Se = 1 / (np.sum(np.abs(sc.S) ** 2, axis=3) + 1e-9)
    errs = {}
    for gain in (1.0, 1e6):
        y = y0 * gain
        x0, _, _ = osol.CGsolver(y, Eo, O(We=np.ones(y.shape[0])), O(Se=Se), None, None, None, 10, "Energy", 1e-3)
        pr = np.random.default_rng(1)
        xc, lam = osol.CSsolver(y, Eo, O(We=np.ones(y.shape[0])), None, None, O(Ti=np.full(Nt, 1e-9)), x0, tol=1e-5,
                                noise=lambda shape: pr.standard_normal(shape))
        g = sc.x_gt * gain
        e = lambda a: float(np.linalg.norm(a.reshape(Nt) - g) / np.linalg.norm(g))  # noqa: E731
        errs[gain] = (e(x0), e(xc))
    assert errs[1e6][1] < 0.9 * errs[1e6][0], errs
    assert errs[1.0][1] > 2 * errs[1.0][0], errs


def test_two_scale_planes_agree():
    """Two scales with shear levels 1 and 2 (the recursion of the lowpass and
    highpass filters, buildWedgeBandpassAndLowpassFilters.m:47-53, and two
    wedge sets) give the same 2-D planes from the device-form builder and the
    oracle."""
    Nt = (80, 76, 74)
    K = [1, 2]
    o_planes = osh.shearlet_planes(list(Nt), K)
    d_planes, table, idxs = sh.build_planes(Nt, 2, K)
    assert len(idxs) == len(osh.shearlet_idxs(3, K, 0)) and table.shape == (len(idxs), 4)
    for P, Q in zip(d_planes, o_planes):
        assert P.shape == Q.shape
        assert np.linalg.norm(P - Q) / np.linalg.norm(Q) < 1e-6


def test_integer_shears_are_circular_row_shifts():
    """Methods/shearing.m shears by a DFT phase ramp (shifting.m's array
    branch); with integer shifts that is exactly a circular shift of each row,
    which the device-form builder uses."""
    rng = np.random.default_rng(13)
    for shape in ((9, 17), (10, 16), (33, 65)):
        v = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        for k in (-2, -1, 1, 2):
            a = sh._shear_rows(v, k)
            b = osh.shearing_21(v, k)
            assert np.allclose(a, b, rtol=0, atol=1e-12 * np.abs(v).max()), (shape, k)


def test_centred_crop_and_pad_agree():
    """resampling.m with fo = 2 (centred zero pad or crop) in both builders."""
    rng = np.random.default_rng(14)
    for src, dst in (((1, 9), (40, 36)), ((33, 4), (40, 36)), ((9, 9), (36, 41)), ((41, 40), (36, 33))):
        v = rng.standard_normal(src)
        assert np.array_equal(sh._centre(v, dst), osh.resampling_space(v, dst))
