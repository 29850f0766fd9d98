"""DISORDER sample orders: the acquisition-side trajectory generator
(Acquisition/samplingDISORDER.m) whose shot map the aligned reconstruction
consumes.

``samplingDISORDER(k, U, SegmentOrder, SampleOrder, K, rng)`` reorders a set
of phase-encode points k (NP x 2, integer coordinates of the spectral grid)
into S = U1 U2 shots, as samplingDISORDER.m:29-198 does:
- the spectral grid is cut into U1 x U2 tiles (:46-58); tiles whose four
  corners are sampled lie inside the shutter (:61-76), and their points go
  tile by tile, each tile's S positions in column-major order (:90-93);
- the remaining (boundary) points follow by angle (:95-101);
- within each run of S points, position p goes to segment Srand(p): the
  electrostatic order of the tile for 'Checkered' (disorder_electrostatic_order),
  a random permutation per run for 'RandomCheckered', and a random
  permutation of all points for 'Random' (:104-110);
- each shot's points are sorted by tile row, tile column (mirrored on even
  tile rows) and position, zig-zag, and reversed on even shots for
  'AlternatingZigZag' (:113-145); 'Sequential' runs the checkered path with
  1 x 1 tiles on the transposed grid (:38,160-182).
It returns the reordered points (shots one after another), NP, K, the
spectral grid, and the 1-based shot and echo number of every grid point
(:184-198). ``shot_map`` turns the shot numbers into the DC-first map H of
the reconstruction driver. Random permutations come from a numpy Generator,
drawn in the order the reference draws its randperm.
"""

import ctypes as C

import numpy as np

from . import _lib


def electrostatic_order(U):
    """0-based column-major order of a U[0] x U[1] tile's positions
    (Acquisition/electrostaticRepulsionDISORDER.m; native, disorder_electrostatic_order)."""
    n1, n2 = int(U[0]), int(U[1])
    out = np.zeros(n1 * n2, np.int32)
    st = _lib.load().disorder_electrostatic_order(n1, n2, out.ctypes.data_as(C.POINTER(C.c_int32)))
    if st:
        raise _lib.DisorderError(st, "electrostatic order of a %d x %d tile" % (n1, n2))
    return out.astype(np.int64)


def spectral_grid(K):
    """Methods/generateGrid.m:27-40 with nor = K, cent = ceil((K+1)/2): the
    integer coordinates (1:K) - ceil((K+1)/2) per dimension."""
    return [np.arange(1, int(K[d]) + 1) - (int(K[d]) + 2) // 2 for d in range(2)]


def _wrap_to_pi_single(x):
    """Mapping Toolbox wrapToPi on single values (only |x| > pi changes)."""
    x = np.asarray(x, np.float32).copy()
    q = (x < -np.pi) | (np.pi < x)
    if np.any(q):
        pi = np.float32(np.pi)
        t = (x[q] + pi).astype(np.float32)
        pos = t > 0
        t = np.mod(t, np.float32(2 * np.pi)).astype(np.float32)
        t[(t == 0) & pos] = np.float32(2 * np.pi)
        x[q] = (t - pi).astype(np.float32)
    return x


def samplingDISORDER(k, U=None, SegmentOrder="RandomCheckered", SampleOrder="AlternatingZigZag", K=None,
                     rng=None):
    k = np.array(k, np.int64)
    if k.ndim != 2 or k.shape[1] != 2:
        raise ValueError("k must be NP x 2")
    NP = k.shape[0]
    if U is None:
        U = [int(round(np.sqrt(NP)))] * 2
    U = [int(U[0]), int(U[1])]
    if K is None:
        K = list(k.max(axis=0) - k.min(axis=0) + 1)
    K = [int(K[0]), int(K[1])]
    if SegmentOrder not in ("Sequential", "Checkered", "RandomCheckered", "Random"):
        raise ValueError("unknown segment order %r" % SegmentOrder)
    if SampleOrder not in ("ZigZag", "AlternatingZigZag"):
        raise ValueError("unknown sample order %r" % SampleOrder)
    if rng is None and (SegmentOrder in ("RandomCheckered", "Random") or
                        (SegmentOrder == "Sequential" and SampleOrder == "ZigZag")):
        rng = np.random.default_rng()
    Uor, SegOr = list(U), SegmentOrder
    if SegmentOrder == "Sequential":
        SegmentOrder, U = "Checkered", [1, 1]
        k = k[:, ::-1].copy()
        K = K[::-1]
    S = U[0] * U[1]
    if not (SampleOrder == "AlternatingZigZag" or NP % S == 0):
        raise ValueError("Number of profiles (%d) not a multiple of number of shots (%d)" % (NP, S))
    kGrid = spectral_grid(K)

    # tiles: starts st[d] (with one tile before the first), ends st + U - 1
    st = []
    for d in range(2):
        g = kGrid[d]
        s = g[np.mod(g - (U[d] + 1) // 2, U[d]) == 0]
        st.append(np.concatenate([[s[0] - (s[1] - s[0])], s]))
    UperK = [len(st[0]), len(st[1])]
    # tiles inside the shutter: all four corners sampled
    mk = k.min(axis=0) - 1
    samp = np.zeros(K, bool)
    samp[k[:, 0] - mk[0] - 1, k[:, 1] - mk[1] - 1] = True
    a0, b0 = np.meshgrid(st[0], st[1], indexing="ij")
    a1, b1 = a0 + U[0] - 1, b0 + U[1] - 1
    inside = (a0 >= kGrid[0][0]) & (a1 <= kGrid[0][-1]) & (b0 >= kGrid[1][0]) & (b1 <= kGrid[1][-1])

    def at(a, b):
        i, j = a - mk[0] - 1, b - mk[1] - 1
        ok = (i >= 0) & (i < K[0]) & (j >= 0) & (j < K[1])
        out = np.zeros(a.shape, bool)
        out[ok] = samp[i[ok], j[ok]]
        return out

    inside &= at(a0, b0) & at(a1, b0) & at(a0, b1) & at(a1, b1)
    # each point's tile (tiles are contiguous from st[d][0] in steps of U[d])
    tm = (k[:, 0] - st[0][0]) // U[0]
    tn = (k[:, 1] - st[1][0]) // U[1]
    assigned = inside[tm, tn]
    acc_m, acc_n = np.nonzero(inside.T)[::-1]  # column-major order of the tiles
    i = np.arange(S)
    kk = np.empty((NP, 2), np.int64)
    nin = len(acc_m) * S
    kk[:nin, 0] = (st[0][acc_m][:, None] + i % U[0]).ravel()
    kk[:nin, 1] = (st[1][acc_n][:, None] + i // U[0]).ravel()
    # boundary points by angle (single precision, as the reference)
    out = k[~assigned].astype(np.float32)
    ang = _wrap_to_pi_single(-np.arctan2(out[:, 1], out[:, 0]).astype(np.float32))
    rad = np.sqrt(np.sum(out * out, axis=1, dtype=np.float32)).astype(np.float32)
    order = np.argsort((ang + np.float32(1e-5) * rad).astype(np.float32), kind="stable")
    kk[nin:] = out[order].astype(np.int64)
    if nin + out.shape[0] != NP:
        raise ValueError("the tiles inside the shutter hold points that are not sampled")
    # segments within each run of S points
    Srand = electrostatic_order(U)
    for e in range(0, S * (NP // S), S):
        if SegmentOrder == "RandomCheckered":
            Srand = rng.permutation(S)
        blk = kk[e:e + S].copy()
        kk[e + Srand] = blk
    if SegmentOrder == "Random":
        kk = kk[rng.permutation(NP)]
    # echo order within each shot: tile row, tile column (mirrored on even
    # tile rows, 1-based), position; reversed on even shots
    bm = (kk[:, 0] - st[0][0]) // U[0] + 1
    bn = (kk[:, 1] - st[1][0]) // U[1] + 1
    even = (bm % 2) == 0
    bn = np.where(even, UperK[1] + 1 - bn, bn)
    k2 = np.where(even, -kk[:, 1], kk[:, 1]).astype(np.float64)
    for s in range(S):
        vS = np.arange(s, NP, S)
        or2 = 1e6 * bn[vS].astype(np.float64)
        if SegOr == "Sequential" and SampleOrder == "ZigZag":
            or2 = or2[rng.permutation(len(or2))]
        key = 1e9 * bm[vS].astype(np.float64) + or2 + 1e3 * kk[vS, 0].astype(np.float64) + k2[vS]
        o = np.argsort(key, kind="stable")
        if (s + 1) % 2 == 0 and SampleOrder == "AlternatingZigZag":
            o = o[::-1]
        if SegmentOrder != "Random":
            kk[vS] = kk[vS[o]]
            bm[vS], bn[vS], k2[vS] = bm[vS[o]], bn[vS[o]], k2[vS[o]]
    k = np.concatenate([kk[np.arange(s, NP, S)] for s in range(S)], axis=0)
    if SegOr == "Sequential":
        k = k[:, ::-1].copy()
        K = K[::-1]
        kGrid = spectral_grid(K)
        U = Uor
        S = U[0] * U[1]
        if SampleOrder == "ZigZag":
            if NP % S:  # NE = NP/S indexes the shots' runs (samplingDISORDER.m:166-167)
                raise ValueError("Number of profiles (%d) not a multiple of number of shots (%d)" % (NP, S))
            NE = NP // S
            for s in range(S):
                v = np.arange(s * NE, (s + 1) * NE)
                or2 = np.where(np.mod(k[v, 0], 2) == 0, -k[v, 1], k[v, 1]).astype(np.float64)
                o = np.argsort(1e3 * k[v, 0].astype(np.float64) + or2, kind="stable")
                k[v] = k[v[o]]
    S = Uor[0] * Uor[1]
    Echo = np.zeros(K, np.int64)
    Shot = np.zeros(K, np.int64)
    counts = [len(range(s, NP, S)) for s in range(S)]
    shot = np.repeat(np.arange(1, S + 1), counts)
    echo = np.concatenate([np.arange(1, c + 1) for c in counts])
    Echo[k[:, 0] - kGrid[0][0], k[:, 1] - kGrid[1][0]] = echo
    Shot[k[:, 0] - kGrid[0][0], k[:, 1] - kGrid[1][0]] = shot
    return k, NP, K, kGrid, Shot, Echo


def cartesian_points(K, shutter="rectangular"):
    """The phase-encode points of a K[0] x K[1] spectral grid (centred
    integer coordinates), all of them or those inside the inscribed ellipse."""
    g = spectral_grid(K)
    a, b = np.meshgrid(g[0], g[1], indexing="ij")
    pts = np.stack([a.ravel(order="F"), b.ravel(order="F")], axis=1)
    if shutter == "elliptical":
        r = (pts[:, 0] / (K[0] / 2.0)) ** 2 + (pts[:, 1] / (K[1] / 2.0)) ** 2
        pts = pts[r <= 1.0]
    return pts


def shot_map(Shot):
    """The DC-first (ifftshifted) 1-based shot map H of the reconstruction
    driver from samplingDISORDER's centred shot numbers (0: not sampled)."""
    return np.fft.ifftshift(np.asarray(Shot, np.int32))
