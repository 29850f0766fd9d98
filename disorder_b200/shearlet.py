"""Shearlet systems for the compressed-sensing reconstruction (host side).

Builds the digital shearlet system of Shearlets/buildShearlet.m (ShearLab 3D,
Kutyniok et al., ACM TOMS 42(1), 2016) for a 3-D grid as the device keeps it:
the 2-D shearlets of the three dimension pairs (buildShearlet.m:103-109) and
the table that names, for each 3-D shearlet, the two 2-D planes whose product
it is (buildShearlet.m:136-146). The 3-D filters themselves (50 complex
volumes at J = 1) are never formed; the kernels evaluate the products where
they need them (csrc/shearlet.cu).

Supported: 3-D grids, complex = 0, the filters CSsolver uses ('kos' or 'ko'
directional filter, 'maxflat2' scaling filter) and checkFilterFeasibility's
first configuration (every dimension at least 33 for J = 1, K = [1]). The
pieces follow:
- getShearletIdxs.m:29-74 (index tables);
- buildDirectionalFilter.m:34-47,149 and buildQuadratureMirrorFilter.m;
- checkFilterFeasibility.m:16-38;
- buildWedgeBandpassAndLowpassFilters.m:34-119, with Methods/shearing.m's
  integer shears done as exact circular row shifts (the DFT phase ramp of
  shifting.m:38-47 shifts by exactly that many samples).
The construction runs once per reconstruction grid, in float64, and the
planes are rounded to complex64 for the device.
"""

import math

import numpy as np

# the 2-D systems' dimension pairs (0-based); the plane of pair q is indexed
# (n[PAIRS[q][0]], n[PAIRS[q][1]]), first index fastest
PAIRS = ((0, 1), (0, 2), (2, 1))

# maximally flat 9-tap lowpass (buildQuadratureMirrorFilter.m, 'maxflat', P = 2)
MAXFLAT2 = np.array([.0104933261758410, -.0263483047033631, -.0517766952966370, .276348304703363,
                     .582566738241592, .276348304703363, -.0517766952966369, -.0263483047033631,
                     .0104933261758408])


def _alternate(n):
    """(-1)^(i - floor(n/2)) for i = 0..n-1 (mirrorModulation.m, c = 0)."""
    return 1.0 - 2.0 * ((np.arange(n) - n // 2) & 1)


def _zero_stuff(v, ups, axis):
    """Methods/upsampling.m (odd = 1) along one axis."""
    shp = list(v.shape)
    shp[axis] = ups * shp[axis] - (ups - 1)
    out = np.zeros(shp, dtype=v.dtype)
    idx = [slice(None)] * v.ndim
    idx[axis] = slice(None, None, ups)
    out[tuple(idx)] = v
    return out


def _centre(v, shape):
    """Methods/resampling.m with fo = 2: centred zero pad / crop to shape."""
    for ax, n in enumerate(shape):
        m = v.shape[ax]
        if m == n:
            continue
        lo, hi = min(m, n), max(m, n)
        start = math.ceil((hi + 1) / 2) - math.ceil((lo - 1) / 2) - 1
        idx = [slice(None)] * v.ndim
        idx[ax] = slice(start, start + lo)
        if m < n:
            shp = list(v.shape)
            shp[ax] = n
            out = np.zeros(shp, dtype=v.dtype)
            out[tuple(idx)] = v
            v = out
        else:
            v = v[tuple(idx)]
    return v


def _f2(v):
    """DFT of a centred 2-D filter, frequency 0 first (ifftshift, then fft)."""
    return np.fft.fft2(np.fft.ifftshift(v))


def _if2(v):
    return np.fft.fftshift(np.fft.ifft2(v))


def _shear_rows(v, k):
    """Methods/shearing.m with dims [2 1]: row i moves by -k (i - floor(N1/2))
    samples along dim 2, circularly."""
    if k == 0:
        return v
    out = np.empty_like(v)
    c = v.shape[0] // 2
    for i in range(v.shape[0]):
        out[i] = np.roll(v[i], -k * (i - c))
    return out


def directional_filter(name="kos"):
    """The 3 x 4 diamond filter of buildDirectionalFilter.m:34-47 (Kovacevic's
    orthogonal filter, 'ko', or its smooth variant, 'kos'), scaled to sum
    sqrt(2), halved by sqrt(2) and mirror-modulated along dim 2 (:149)."""
    if name == "kos":
        a0 = a1 = -math.sqrt(3)
        a2 = 2 + math.sqrt(3)
    elif name == "ko":
        a0, a1, a2 = 2.0, 0.5, 1.0
    else:
        raise NotImplementedError("directional filter %r is not built (use 'kos' or 'ko')" % name)
    h = np.array([[0.0, -a1, -a0 * a1, 0.0],
                  [-a2, -a0 * a2, -a0, 1.0],
                  [0.0, a0 * a1 * a2, -a1 * a2, 0.0]])
    h *= math.sqrt(2) / h.sum()
    return (h / math.sqrt(2)) * _alternate(4)[None, :]


def scaling_filter(name="maxflat2"):
    if name != "maxflat2":
        raise NotImplementedError("scaling filter %r is not built (use 'maxflat2')" % name)
    return MAXFLAT2 / MAXFLAT2.sum()


def feasible(Nab, K, DF, SF):
    """checkFilterFeasibility.m:16-38, first configuration: True when the
    requested filters fit a plane of size Nab."""
    L = SF.size
    l1 = L
    for _ in range(len(K) - 1):
        l1 = L + 2 * (l1 - 1)
    l2 = L
    for _ in range(max(K)):
        l2 = L + 2 * (l2 - 1)
    l2 += (DF.shape[0] - 1) * 2 ** (max(K) + 1)
    return all(n >= l1 and n >= l2 and n >= DF.shape[1] for n in Nab)


def _filters_2d(Nab, K, DF, SF):
    """buildWedgeBandpassAndLowpassFilters.m:34-119 for one plane orientation:
    (wedges {k: (Na, Nb, 2^(k+1)+1)}, bandpass (Na, Nb, J), lowpass)."""
    Na, Nb = Nab
    J, Kmax = len(K), max(K) + 1
    WF = SF * _alternate(SF.size)
    DF = DF / np.abs(DF).sum()
    lp1, hp = [None] * J, [None] * J
    lp1[-1], hp[-1] = SF, WF
    for j in range(J - 2, -1, -1):
        lp1[j] = np.convolve(SF, _zero_stuff(lp1[j + 1], 2, 0))
        hp[j] = np.convolve(SF, _zero_stuff(hp[j + 1], 2, 0))
    lp2 = [None] * Kmax
    lp2[-1] = SF
    for k in range(Kmax - 2, -1, -1):
        lp2[k] = np.convolve(SF, _zero_stuff(lp2[k + 1], 2, 0))
    bp = np.stack([_f2(_centre(hp[j][None, :], Nab)) for j in range(J)], axis=2)
    wedges = {}
    for k in sorted(set(K)):
        s = 2 ** k
        dfu = _zero_stuff(DF, 2 ** (k + 1), 0)
        col = lp2[Kmax - k - 1]
        cv = np.stack([np.convolve(dfu[:, j], col) for j in range(dfu.shape[1])], axis=1)
        wu = _zero_stuff(_centre(cv, Nab), s, 1)
        aux = _centre(lp2[Kmax - max(k - 1, 0) - 1][None, :], wu.shape)
        if k >= 1:
            wu = _if2(_f2(wu) * _f2(aux))
            faux = _f2(aux[:, ::-1])
        w = np.zeros((Na, Nb, 2 * s + 1), dtype=np.complex128)
        for l in range(-s, s + 1):
            t = _shear_rows(wu, l)
            if k >= 1:
                t = _if2(_f2(t) * faux)
            w[:, :, s - l] = _f2(s * t[:, 0:s * Nb:s])
        wedges[k] = w
    lp = _f2(_centre(np.outer(lp1[0], lp1[0]), Nab))
    return wedges, bp, lp


def shearlet_idxs(nd, K, full):
    """getShearletIdxs.m:29-74 (complex = 0): 1-based rows, lowpass last."""
    rows = []
    if nd == 2:
        for cone in (1, 2):
            for sc in range(1, len(K) + 1):
                s = 2 ** K[sc - 1]
                rows += [[cone, sc, 1, h] for h in range(-s, s + 1) if full or cone == 1 or abs(h) < s]
        rows.append([0, 0, 0, 0])
    else:
        for pyr in (1, 2, 3):
            for sc in range(1, len(K) + 1):
                s = 2 ** K[sc - 1]
                for h1 in range(-s, s + 1):
                    for h2 in range(-s, s + 1):
                        if full or pyr == 1 or (pyr == 2 and abs(h2) < s) or (abs(h1) < s and abs(h2) < s):
                            rows.append([pyr, sc, 1, h1, h2])
        rows.append([0, 0, 0, 0, 0])
    return np.array(rows, dtype=np.int64)


def _plane_index(K, cone, scale, shearing):
    """buildShearlet.m:155-158 (complex = 0, half = 1), 0-based."""
    K = np.asarray(K)
    ind = int(np.sum(2 ** (K + 1) + 1)) * (cone - 1) + 2 ** int(K[scale - 1]) + 1 + shearing
    if scale > 1:
        ind += int(np.sum(2 ** (K[:scale - 1] + 1) + 1))
    return ind - 1


def build_planes(N, J=1, K=None, DFtype="kos", QMFtype="maxflat2", full=0):
    """The device form of buildShearlet(N, J, [], K, DFtype, QMFtype, full):
    (planes, table, idxs). planes[q]: (Na, Nb, NS2) complex64 Fortran arrays
    (the 2-D system of pair q, full = 1); table: (NW, 4) int32 rows (pair A,
    plane A, pair B, plane B); idxs: the 3-D index table (NW x 5)."""
    if K is None:
        K = [int(math.ceil(j / 2)) for j in range(1, J + 1)]
    K = [int(k) for k in K]
    if len(K) != J:
        raise ValueError("K must have J entries")
    N = [int(n) for n in N]
    if len(N) != 3:
        raise ValueError("shearlet systems are built for 3-D grids")
    DF, SF = directional_filter(DFtype), scaling_filter(QMFtype)
    idx2 = shearlet_idxs(2, K, 1)
    planes = []
    for a, b in PAIRS:
        Nab = (N[a], N[b])
        if not feasible(Nab, K, DF, SF):
            raise NotImplementedError("shearlet system (J=%d, K=%s) not available for a %d x %d plane with the "
                                      "%s/%s filters" % (J, K, Nab[0], Nab[1], DFtype, QMFtype))
        f0 = _filters_2d(Nab, K, DF, SF)
        f1 = _filters_2d(Nab[::-1], K, DF, SF)
        P = np.zeros((Nab[0], Nab[1], len(idx2)), dtype=np.complex128)
        for s, (cone, sc, _, h) in enumerate(idx2):
            if cone == 0:
                P[:, :, s] = f0[2]
            else:
                k = K[sc - 1]
                if cone == 1:
                    P[:, :, s] = f0[0][k][:, :, 2 ** k - h] * np.conj(f0[1][:, :, sc - 1])
                else:
                    P[:, :, s] = (f1[0][k][:, :, 2 ** k + h] * np.conj(f1[1][:, :, sc - 1])).T
        planes.append(np.asfortranarray(P.astype(np.complex64)))
    idx3 = shearlet_idxs(3, K, full)
    lp = len(idx2) - 1
    table = np.zeros((len(idx3), 4), dtype=np.int32)
    for w, (pyr, sc, _, h1, h2) in enumerate(idx3):
        if pyr == 0:
            table[w] = (0, lp, 2, lp)
        elif pyr == 1:
            table[w] = (0, _plane_index(K, 1, sc, h1), 2, _plane_index(K, 1, sc, h2))
        elif pyr == 2:
            table[w] = (1, _plane_index(K, 1, sc, h1), 2, _plane_index(K, 2, sc, h2))
        else:
            table[w] = (0, _plane_index(K, 2, sc, h1), 1, _plane_index(K, 2, sc, h2))
    return planes, table, idx3


def expand(planes, table, N, w):
    """The 3-D shearlet w as an (N1, N2, N3) complex64 array (host; for
    inspection and tests, the device never forms it)."""
    out = np.ones(N, dtype=np.complex64)
    for h in range(2):
        q, k = int(table[w, 2 * h]), int(table[w, 2 * h + 1])
        a, b = PAIRS[q]
        shape = [1, 1, 1]
        shape[a], shape[b] = N[a], N[b]
        P = planes[q][:, :, k]
        out = out * (P if a < b else P.T).reshape(shape)
    return out
