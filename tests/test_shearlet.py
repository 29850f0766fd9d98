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
