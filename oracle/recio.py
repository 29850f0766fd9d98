"""Acquisition structure of Reconstruction/solveXT.m (oracle).

TEST INFRASTRUCTURE ONLY. Restates solveXT.m:74-142 loop by loop (the
profile -> shot / sweep assignment and the timeIndex fill), Methods/fct.m
(the orthonormal DCT-II by Makhoul's reordering and one FFT), and the data
steps of solveXT.m:39-72 (Methods/computeROI.m, extractROI.m, the 'tukey'
filter of buildFilter.m and resSub.m), in float64.
"""

import math

import numpy as np


def fct(x):
    """Methods/fct.m along dim 1: reorder [1:2:n, flip(2:2:n)], FFT, weight by
    2 exp(-i pi k / 2n) / sqrt(2n) with the first weight / sqrt(2), real part."""
    x = np.asarray(x, np.float64)
    n = x.shape[0]
    ind = list(range(0, n, 2)) + list(range(1, n, 2))[::-1]
    v = np.fft.fft(x[ind], axis=0)
    ww = 2 * np.exp(-1j * np.pi * np.arange(n) / (2 * n)) / np.sqrt(2 * n)
    ww[0] = ww[0] / np.sqrt(2)
    return np.real(ww.reshape((n,) + (1,) * (x.ndim - 1)) * v)


def acquisition_structure(z2, z3, kRange2, kRange3, TFEfactor, ZReconLength=1, NY=None, NRepeats=1,
                          groupSweeps=1):
    """solveXT.m:74-142 (same arguments and outputs as the product's)."""
    z2 = list(np.asarray(z2).ravel())
    z3 = list(np.asarray(z3).ravel())
    NEchos = max(TFEfactor, ZReconLength)
    NProfs = len(z2)
    if NProfs <= 1 or NProfs != len(z3):
        raise ValueError("separable trajectories")
    kTraj = [[float(z3[n]), float(z2[n])] for n in range(NProfs)]  # perm(1:2) = [3 2]
    if NEchos == 1:
        NEchos = NProfs
    NShots = NProfs / NEchos
    if NShots != math.floor(NShots):
        raise ValueError("interrupted scan")
    NShots = int(NShots)
    if NShots < NRepeats:
        NShots = NRepeats
        NProfs = NShots * NEchos
        kTraj = kTraj * NRepeats
        NEchos = NProfs // NShots
    kRange = [list(kRange3), list(kRange2)]
    kShift = [math.floor((kRange[n][1] - kRange[n][0] + 1) / 2) + 1 for n in range(2)]
    kSize = [kRange[n][1] - kRange[n][0] + 1 for n in range(2)]
    kIndex = [[int(kTraj[n][m] + kShift[m]) for m in range(2)] for n in range(NProfs)]
    steady = False
    if NShots % NRepeats == 0:
        steady = (NShots // NRepeats) == 1
    if steady:
        kT = np.abs(fct(np.array(kTraj)))
        half = NProfs // 2
        iAs = []
        for m in range(2):  # MATLAB max: first index of the maximum
            best, ib = -1.0, 0
            for i in range(half):
                if kT[i, m] > best:
                    best, ib = kT[i, m], i
            iAs.append(ib + 1)
        iM = min(iAs)
        if iM <= 1:
            raise ValueError("no sweep period")
        NSamples = NProfs / (iM - 1)
        NSweeps = int(round(NProfs / (NSamples * groupSweeps)))
        if NSweeps < 1:
            raise ValueError("no sweeps")
    else:
        NSweeps = NShots
    sweepSample = [math.ceil(NSweeps * ((n + 1 - 0.5) / NProfs)) for n in range(NProfs)]
    NY = [int(v) for v in (NY if NY is not None else kSize)]
    timeIndex = np.zeros((NY[0], NY[1], NRepeats), np.int64)
    for n in range(NProfs):
        i1, i2 = kIndex[n][0] - 1, kIndex[n][1] - 1
        if not (0 <= i1 < NY[0] and 0 <= i2 < NY[1]):
            raise ValueError("profile outside the grid")
        for s in range(NRepeats):
            if timeIndex[i1, i2, s] == 0:
                timeIndex[i1, i2, s] = n + 1
                break
    timeIndex = np.fft.ifftshift(timeIndex, axes=(0, 1))
    H = np.zeros((NY[0], NY[1]), np.int64)
    for i in range(NY[0]):
        for j in range(NY[1]):
            t = timeIndex[i, j, 0]
            if t:
                H[i, j] = sweepSample[t - 1]
    return {"NEchos": NEchos, "NShots": NShots, "NProfs": NProfs, "NSweeps": NSweeps, "steady_state": steady,
            "kTraj": np.array(kTraj), "kShift": np.array(kShift, float), "kSize": np.array(kSize, float),
            "kIndex": np.array(kIndex), "sweepSample": np.array(sweepSample), "timeIndex": timeIndex, "H": H}


def computeROI(x, ext=0, sy=None, ev=None, fu=0):
    """Methods/computeROI.m:20-57, the while loops as written."""
    a = (np.abs(np.asarray(x)) > 1e-6).astype(np.float64)
    ND = a.ndim if fu else min(a.ndim, 3)
    sy = [0] * ND if sy is None else list(sy)
    ev = [0] * ND if ev is None else list(ev)
    ROI = np.zeros((ND, 6))
    for n in range(ND):
        ROI[n, 0], ROI[n, 1], ROI[n, 2] = 1, a.shape[n], a.shape[n]
    step = [1, -1]
    for l in range(2):
        for n in range(ND):
            while not np.any(np.take(a, int(ROI[n, l]) - 1, axis=n)):
                ROI[n, l] += step[l]
    ROI[:, 0] = np.maximum(ROI[:, 0] - ext, 1)
    ROI[:, 1] = np.minimum(ROI[:, 1] + ext, ROI[:, 2])
    ROI[:, 3] = ROI[:, 1] - ROI[:, 0] + 1
    ROI[:, 4] = ROI[:, 0] - 1
    ROI[:, 5] = ROI[:, 2] - ROI[:, 1]
    for n in range(ND):
        if sy[n]:
            indSm = 1 if ROI[n, 4] <= ROI[n, 5] else 2
            for col in (3 - indSm, 4):
                ROI[n, col - 1] += ROI[n, 5] - ROI[n, 4]
            ROI[n, 5] = ROI[n, 4]
        if ev[n] and ROI[n, 3] % 2 != 0:
            ROI[n, 3] -= 1
            ROI[n, 0] += 1
            ROI[n, 4] += 1
    return ROI.astype(np.int64)


def extractROI(x, ROI, ext=1, dims=None):
    """Methods/extractROI.m:14-28."""
    x = np.asarray(x)
    ND = min(ROI.shape[0], x.ndim)
    dims = list(range(1, ND + 1)) if dims is None else ([dims] if np.isscalar(dims) else list(dims))
    idx = [np.arange(x.shape[d]) for d in range(x.ndim)]
    for d in dims:
        idx[d - 1] = np.arange(int(ROI[d - 1, 0]) - 1, int(ROI[d - 1, 1]))
    if ext:
        return x[np.ix_(*idx)]
    shape = list(x.shape)
    for d in dims:
        shape[d - 1] = int(ROI[d - 1, 2])
    y = np.zeros(shape, dtype=x.dtype)
    y[np.ix_(*idx)] = x
    return y


def buildFilter_tukey(N, sp, gibbsRing):
    """Methods/buildFilter.m:93-101 ('tukey') with the 1-D 'tukeyIso' windows
    of :69-92, element by element."""
    ND = len(N)
    sp = list(np.broadcast_to(np.asarray(sp, np.float64), (ND,)))
    g = list(np.atleast_1d(np.asarray(gibbsRing, np.float64)))
    g = g + [g[-1]] * (ND - len(g))
    x = np.ones(N)
    for m in range(ND):
        cent = math.ceil((N[m] + 1) / 2)
        w = np.ones(N[m])
        alpha = 1 - g[m]
        for i in range(N[m]):
            kk = abs((2 * np.pi / sp[m]) / N[m] * ((i + 1) - cent))
            if g[m] != 0 and kk >= np.pi * alpha:
                w[i] = 0.5 * (1 + math.cos(math.pi * ((kk - math.pi * alpha) / ((1 - alpha) * math.pi))))
            if kk >= np.pi:
                w[i] = 0
        shape = [1] * ND
        shape[m] = N[m]
        x = x * w.reshape(shape)
    return np.fft.fftshift(x)


def resSub(x, first=5):
    """Methods/resSub.m:15-30 with orDim = first:ndims(x)."""
    x = np.asarray(x)
    if x.ndim < first:
        return x
    N = list(x.shape[:first - 1]) + [int(np.prod(x.shape[first - 1:]))]
    return x.reshape(N, order="F")


def prepare_rec(y, S, M, voxSiz, apod=(0.1, 0.0, 0.0)):
    """solveXT.m:39-72, the data steps in order."""
    ROI = computeROI(M, 0, [0, 0, 0], [1, 0, 0])
    y, S, M = (extractROI(a, ROI, 1, 1) for a in (y, S, M))
    perm = lambda a: np.transpose(a, [2, 1, 0] + list(range(3, np.ndim(a))))  # noqa: E731
    y, S, M = perm(y), perm(S), perm(M)
    voxSiz = [voxSiz[2], voxSiz[1], voxSiz[0]]
    ap = [apod[2], apod[1], apod[0]]
    NY = y.shape
    w = np.fft.ifftshift(buildFilter_tukey(list(NY[:3]), [10, 10, 1], ap))
    y = y * w.reshape(tuple(NY[:3]) + (1,) * (y.ndim - 3))
    y = resSub(y, 5)
    return {"y": y, "S": S, "M": M, "ROI": ROI, "voxSiz": tuple(voxSiz)}
