"""Acquisition structure of Reconstruction/solveXT.m (oracle).

TEST INFRASTRUCTURE ONLY. Restates solveXT.m:74-142 loop by loop (the
profile -> shot / sweep assignment and the timeIndex fill) and Methods/fct.m
(the orthonormal DCT-II by Makhoul's reordering and one FFT), in float64.
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
