"""DISORDER sample orders (oracle).

TEST INFRASTRUCTURE ONLY. Restates, loop by loop,
  Acquisition/samplingDISORDER.m:29-198 (tiles of the spectral grid,
    tiles inside the shutter, angular traversal of the boundary samples,
    checkered / random-checkered / random segment orders, zig-zag and
    alternating zig-zag echo orders, shot and echo maps),
  Acquisition/electrostaticRepulsionDISORDER.m:9-52 (greedy order of a
    tile's positions by minimum wrapped electric repulsion),
  Methods/generateGrid.m:27-40 for the spectral grid (nor = N, cent =
    ceil((N+1)/2): integer coordinates) and the Mapping Toolbox wrapToPi in
    single precision (the boundary samples' angles are single,
    samplingDISORDER.m:84-86).

MATLAB's randperm is not reproducible here: every random permutation is
drawn from a numpy Generator in the order the reference draws them, so the
product and this restatement agree for the same seed. Indices are 0-based
internally, shot and echo numbers 1-based as in the reference.
"""

import numpy as np


def electrostatic_order(N):
    """electrostaticRepulsionDISORDER.m:9-52: the order (0-based, column-major
    positions of an N[0] x N[1] grid) in which a greedy walk places points,
    each new one where the summed inverse squared distance to the points
    already placed (nearest of the 9 periodic images) is least; the first
    strictly smaller value by more than 1e-9 in scan order wins."""
    N1, N2 = int(N[0]), int(N[1])
    P = N1 * N2
    ind = [0] * P
    poi = []
    free = [True] * P
    c0 = (int(np.ceil(N1 / 2.0)) - 1) + N1 * (int(np.ceil(N2 / 2.0)) - 1)  # sub2ind(N, ceil(N/2))
    ind[0] = c0
    poi.append((c0 % N1 + 1, c0 // N1 + 1))
    free[c0] = False
    sh1, sh2 = (-N1, 0, N1), (-N2, 0, N2)
    for n in range(1, P):
        best, bi = np.inf, -1
        for m in range(P):
            if not free[m]:
                continue
            c1, c2 = m % N1 + 1, m // N1 + 1
            w = 0.0
            for (p1, p2) in poi:
                dmin = np.inf
                for a in sh2:
                    for b in sh1:
                        d = float((c1 - (p1 + b)) ** 2 + (c2 - (p2 + a)) ** 2)
                        if d < dmin:
                            dmin = d
                w += 1.0 / dmin
            if w < best - 1e-9:
                best, bi = w, m
        ind[n] = bi
        poi.append((bi % N1 + 1, bi // N1 + 1))
        free[bi] = False
    return np.array(ind, np.int64)


def _grid(K):
    """generateGrid(K, 0, K, ceil((K+1)/2), 0): (1:K) - ceil((K+1)/2)."""
    return [np.arange(1, int(K[d]) + 1) - int(np.ceil((int(K[d]) + 1) / 2.0)) for d in range(2)]


def _wrap_to_pi_single(x):
    x = np.array(x, np.float32)
    pi = np.float32(np.pi)
    for i in range(x.size):
        v = x.flat[i]
        if v < -np.pi or np.pi < v:
            t = np.float32(v + pi)
            pos = t > 0
            t = np.float32(np.mod(t, np.float32(2 * np.pi)))
            if t == 0 and pos:
                t = np.float32(2 * np.pi)
            x.flat[i] = np.float32(t - pi)
    return x


def samplingDISORDER(k, U=None, SegmentOrder="RandomCheckered", SampleOrder="AlternatingZigZag", K=None,
                     rng=None):
    """Returns (k reordered (NP, 2), NP, K, kGrid, ShotNumber (K), EchoNumber (K))."""
    k = np.array(k, np.int64)
    NP = k.shape[0]
    if U is None:
        U = [int(round(np.sqrt(NP)))] * 2
    U = [int(U[0]), int(U[1])]
    if K is None:
        K = list(k.max(axis=0) - k.min(axis=0) + 1)
    K = [int(K[0]), int(K[1])]
    Uor, SegOr = list(U), SegmentOrder
    if SegmentOrder == "Sequential":
        SegmentOrder, U = "Checkered", [1, 1]
        k = k[:, ::-1].copy()
        K = K[::-1]
    S = U[0] * U[1]
    if not (SampleOrder == "AlternatingZigZag" or NP % S == 0):
        raise ValueError("Number of profiles (%d) not a multiple of number of shots (%d)" % (NP, S))
    kGrid = _grid(K)
    if SegmentOrder in ("Random", "RandomCheckered", "Checkered"):
        # tiles: starts and ends per dimension (samplingDISORDER.m:46-58)
        Ul, UperK = [], []
        for d in range(2):
            g = kGrid[d]
            st = [int(v) for v in g if (v - int(np.ceil(U[d] / 2.0))) % U[d] == 0]
            st = [st[0] - (st[1] - st[0])] + st
            Ul.append([(s, s + U[d] - 1) for s in st])
            UperK.append(len(st))
        # tiles with all four corners sampled (:61-76)
        mk = k.min(axis=0) - 1
        sampled = set((int(a - mk[0]), int(b - mk[1])) for a, b in k)
        inside = np.zeros(UperK, bool)
        for m in range(UperK[0]):
            for n in range(UperK[1]):
                (a0, a1), (b0, b1) = Ul[0][m], Ul[1][n]
                if a0 >= kGrid[0][0] and a1 <= kGrid[0][-1] and b0 >= kGrid[1][0] and b1 <= kGrid[1][-1]:
                    corners = [(a0, b0), (a1, b0), (a0, b1), (a1, b1)]
                    inside[m, n] = sum((c[0] - mk[0], c[1] - mk[1]) in sampled for c in corners) == 4
        # accepted tiles in column-major order, their profiles (:79-86)
        acc = [(m, n) for n in range(UperK[1]) for m in range(UperK[0]) if inside[m, n]]
        assigned = np.zeros(NP, bool)
        for (m, n) in acc:
            (a0, a1), (b0, b1) = Ul[0][m], Ul[1][n]
            for p in range(NP):
                if a0 <= k[p, 0] <= a1 and b0 <= k[p, 1] <= b1:
                    assigned[p] = True
        kk = np.zeros((NP, 2), np.int64)
        cont = 0
        for (m, n) in acc:  # each tile's S positions, column-major (:90-93)
            for i in range(S):
                kk[cont + i] = (i % U[0] + Ul[0][m][0], i // U[0] + Ul[1][n][0])
            cont += S
        # boundary samples by angle (:95-101)
        out = k[~assigned].astype(np.float32)
        ang = _wrap_to_pi_single(-np.arctan2(out[:, 1], out[:, 0]).astype(np.float32))
        rad = np.sqrt(np.sum(out * out, axis=1, dtype=np.float32)).astype(np.float32)
        key = (ang + np.float32(1e-5) * rad).astype(np.float32)
        order = np.argsort(key, kind="stable")
        kk[cont:cont + out.shape[0]] = out[order].astype(np.int64)
        # segment order within each block of S (:104-110)
        Srand = electrostatic_order(U)
        for e in range(0, S * (NP // S), S):
            if SegmentOrder == "RandomCheckered":
                Srand = rng.permutation(S)
            blk = kk[e:e + S].copy()
            for i in range(S):
                kk[e + Srand[i]] = blk[i]
        if SegmentOrder == "Random":
            kk = kk[rng.permutation(NP)]
        # echo order within each shot (:113-145)
        for s in range(S):
            vS = np.arange(s, NP, S)
            kke = kk[vS].astype(np.float64)
            blk = np.zeros((len(vS), 2))
            for l in range(len(vS)):
                ent = False
                for m in range(UperK[0]):
                    if Ul[0][m][0] <= kke[l, 0] <= Ul[0][m][1]:
                        for n in range(UperK[1]):
                            if Ul[1][n][0] <= kke[l, 1] <= Ul[1][n][1]:
                                blk[l] = (m + 1, n + 1)
                                if (m + 1) % 2 == 0:
                                    kke[l, 1] = -kke[l, 1]
                                    blk[l, 1] = UperK[1] - n
                                    ent = True
                                    break
                        if ent:
                            break
            if not np.any(blk):
                raise ValueError("Sample not assigned to a block")
            or2 = 1e6 * blk[:, 1]
            if SegOr == "Sequential" and SampleOrder == "ZigZag":
                or2 = or2[rng.permutation(len(or2))]
            key = 1e9 * blk[:, 0] + or2 + 1e3 * kke[:, 0] + kke[:, 1]
            o = np.argsort(key, kind="stable")
            if (s + 1) % 2 == 0 and SampleOrder == "AlternatingZigZag":
                o = o[::-1]
            if SegmentOrder != "Random":
                kk[vS] = kk[vS[o]]
        # shots one after another (:147-153)
        k = np.concatenate([kk[np.arange(s, NP, S)] for s in range(S)], axis=0)
    if SegOr == "Sequential":
        k = k[:, ::-1].copy()
        K = K[::-1]
        kGrid = _grid(K)
        U = Uor
        S = U[0] * U[1]
    if SegOr == "Sequential" and SampleOrder == "ZigZag":
        if NP % S:  # NE = NP/S indexes the shots' runs (samplingDISORDER.m:166-167)
            raise ValueError("Number of profiles (%d) not a multiple of number of shots (%d)" % (NP, S))
        NE = NP // S
        for s in range(S):
            v = np.arange(s * NE, (s + 1) * NE)
            kke = k[v].astype(np.float64)
            or2 = kke[:, 1].copy()
            even = np.mod(kke[:, 0], 2) == 0
            or2[even] = -or2[even]
            o = np.argsort(1e3 * kke[:, 0] + or2, kind="stable")
            k[v] = k[v[o]]
    S = Uor[0] * Uor[1]
    Echo = np.zeros(K, np.int64)
    Shot = np.zeros(K, np.int64)
    cont = 0
    for s in range(S):
        for e in range(len(range(s, NP, S))):
            i, j = k[cont, 0] - kGrid[0][0], k[cont, 1] - kGrid[1][0]
            Echo[i, j] = e + 1
            Shot[i, j] = s + 1
            cont += 1
    return k, NP, K, kGrid, Shot, Echo
