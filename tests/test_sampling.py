"""DISORDER sample orders (disorder_b200.sampling) against the oracle's
loop-by-loop restatement of Acquisition/samplingDISORDER.m and
electrostaticRepulsionDISORDER.m (oracle/sampling.py): identical points,
shot maps and echo maps for every segment and sample order, on a
rectangular and an elliptical shutter, with the same random draws; and the
properties the method is built on (every tile inside the shutter gives each
shot one point, zig-zag echoes)."""

import numpy as np
import pytest

from disorder_b200 import sampling as ps
from oracle import sampling as osm

ORDERS = [(seg, so) for seg in ("Checkered", "RandomCheckered", "Random", "Sequential")
          for so in ("AlternatingZigZag", "ZigZag")]


@pytest.mark.parametrize("U", [(4, 4), (3, 5), (8, 8), (2, 6)])
def test_electrostatic_order_matches_oracle(U):
    a = ps.electrostatic_order(U)
    assert np.array_equal(a, osm.electrostatic_order(U))
    assert sorted(a.tolist()) == list(range(U[0] * U[1]))
    assert a[0] == (U[0] + 1) // 2 - 1 + U[0] * ((U[1] + 1) // 2 - 1)  # the tile's centre first


@pytest.mark.parametrize("seg,so", ORDERS)
@pytest.mark.parametrize("K,shutter", [((16, 16), "rectangular"), ((24, 20), "elliptical")])
def test_sample_orders_match_oracle(K, shutter, seg, so):
    pts = ps.cartesian_points(K, shutter)
    args = (pts, (4, 4), seg, so, None)
    try:
        ref = osm.samplingDISORDER(*args, rng=np.random.default_rng(7))
    except ValueError:
        with pytest.raises(ValueError):
            ps.samplingDISORDER(*args, rng=np.random.default_rng(7))
        return
    out = ps.samplingDISORDER(*args, rng=np.random.default_rng(7))
    assert np.array_equal(out[0], ref[0])
    assert out[1] == ref[1] and list(out[2]) == list(ref[2])
    assert np.array_equal(out[4], ref[4]) and np.array_equal(out[5], ref[5])
    # a reordering of the input points
    assert sorted(map(tuple, out[0].tolist())) == sorted(map(tuple, pts.tolist()))


def test_random_checkered_tiles_give_each_shot_one_point():
    K, U = (32, 24), (4, 4)
    pts = ps.cartesian_points(K)
    k, NP, Kr, kGrid, Shot, Echo = ps.samplingDISORDER(pts, U, "RandomCheckered", "AlternatingZigZag",
                                                       rng=np.random.default_rng(1))
    S = U[0] * U[1]
    assert NP == pts.shape[0] and Shot.min() == 1 and Shot.max() == S
    # tiles start where (k - ceil(U/2)) mod U == 0 on the centred grid
    o = [int(np.nonzero(np.mod(kGrid[d] - (U[d] + 1) // 2, U[d]) == 0)[0][0]) for d in range(2)]
    for a in range(o[0], K[0] - U[0] + 1, U[0]):
        for b in range(o[1], K[1] - U[1] + 1, U[1]):
            assert sorted(Shot[a:a + U[0], b:b + U[1]].ravel().tolist()) == list(range(1, S + 1))
    # each shot: NP / S echoes numbered 1..NP/S
    for s in range(1, S + 1):
        assert sorted(Echo[Shot == s].tolist()) == list(range(1, NP // S + 1))
    # consecutive shots walk their points in opposite directions (alternating zig-zag)
    first = k[: NP // S]
    second = k[NP // S: 2 * NP // S]
    assert first[0, 0] <= first[-1, 0] and second[0, 0] >= second[-1, 0]


def test_shot_map_feeds_the_reconstruction_sampling():
    from disorder_b200 import synth
    K, U = (16, 16), (4, 4)
    _, _, _, _, Shot, _ = ps.samplingDISORDER(ps.cartesian_points(K), U, "RandomCheckered",
                                              rng=np.random.default_rng(3))
    H = ps.shot_map(Shot)
    assert H[0, 0] == Shot[K[0] // 2, K[1] // 2]  # DC first
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, 16)
    assert np.all(np.diff(nEc)[:16] == 16) and len(ky) == K[0] * K[1]


def test_bad_arguments():
    pts = ps.cartesian_points((8, 8))
    with pytest.raises(ValueError):
        ps.samplingDISORDER(pts, (4, 4), "Spiral")
    with pytest.raises(ValueError):
        ps.samplingDISORDER(pts[:-1], (4, 4), "Checkered", "ZigZag")


def test_electrostatic_order_rejects_bad_sizes():
    import ctypes as C
    from disorder_b200 import _lib
    out = np.zeros(4, np.int32)
    p = out.ctypes.data_as(C.POINTER(C.c_int32))
    lib = _lib.load()
    assert lib.disorder_electrostatic_order(0, 4, p) == 1  # DISORDER_BAD_ARG
    assert lib.disorder_electrostatic_order(2, 2, None) == 1
    assert lib.disorder_electrostatic_order(2, 2, p) == 0 and sorted(out.tolist()) == [0, 1, 2, 3]
