"""Scanner acquisition order -> the reconstruction's motion states.

``acquisition_structure`` is the ACQUISITION STRUCTURE block of
Reconstruction/solveXT.m:74-142. The scanner lists, in acquisition order,
the phase-encode coordinates of every profile (``rec.Assign.z{2}``,
``rec.Assign.z{3}``). The reconstruction needs the shots (or, for
steady-state sequences, sweeps) they fall into, and which profile sampled
each point of the phase-encode grid (``timeIndex``), to build its per-state
sample lists (``E.mSt``, solveXT.m:349-350). The result's ``H`` is that
state map at full resolution, DC first: the shot map
``recon.aligned_reconstruction`` takes.

Conventions follow solveXT.m: the phase encodes are permuted to the first
dimensions with perm(1:3) = [3 2 1] (:51), so grid dimension 1 is the
scanner's dimension 3 and grid dimension 2 its dimension 2 (:80, :99).

Not restated here (the rest of solveXT.m's ingestion of the ``rec``
structure): the readout ROI (computeROI / extractROI, :40-47), the Tukey
apodization (buildFilter, :70) and reading ``rec`` files, which writeRaw.m
saves as MATLAB v7.3 (HDF5) files.
"""

import math

import numpy as np


class AcquisitionError(ValueError):
    """A scan the aligned reconstruction does not process (solveXT.m sets
    rec.Fail and returns: separable trajectories, interrupted scans)."""


def _dct_ortho(x):
    """Orthonormal DCT-II along axis 0 (Methods/fct.m)."""
    from scipy.fft import dct
    return dct(np.asarray(x, np.float64), type=2, norm="ortho", axis=0)


def acquisition_structure(z2, z3, kRange2, kRange3, TFEfactor, ZReconLength=1, NY=None, NRepeats=1,
                          groupSweeps=1):
    """solveXT.m:74-142.

    z2, z3: per-profile phase-encode coordinates rec.Assign.z{2}, z{3}, in
    acquisition order (integers centred on the k-space origin);
    kRange2, kRange3: rec.Enc.kRange{2}, {3} as (min, max);
    TFEfactor, ZReconLength: rec.Par.Labels fields (echoes per shot);
    NY: the grid size (N1, N2) after the permutation (default the k-space
    extent); NRepeats: averages along dimension 5 of the data;
    groupSweeps: parXT.groupSweeps (steady-state sequences only).

    Returns a dict with NEchos, NShots, NProfs, NSweeps, steady_state,
    kTraj (NProfs x 2, grid order), kShift, kSize, kIndex (1-based grid
    indices), sweepSample (1-based sweep of each profile), timeIndex
    (N1 x N2 x NRepeats, 1-based profile per grid point and repeat, 0 when
    unsampled, ifftshifted along dims 1-2) and H (the state of repeat 1 per
    grid point, DC first, 0 unsampled)."""
    z2 = np.asarray(z2).ravel()
    z3 = np.asarray(z3).ravel()
    NEchos = max(int(TFEfactor), int(ZReconLength))  # :75
    NProfs = z2.size
    if NProfs <= 1 or NProfs != z3.size:  # :77
        raise AcquisitionError("separable y-z trajectories: the aligned reconstruction is not performed")
    kTraj = np.stack([z3, z2], axis=1).astype(np.float64)  # :79-80, perm = [3 2 1]
    if NEchos == 1:
        NEchos = NProfs
    NShots = NProfs / NEchos
    if NShots != int(NShots):  # :83
        raise AcquisitionError("number of shots %.2f: probably an interrupted scan" % NShots)
    NShots = int(NShots)
    NRepeats = int(NRepeats)
    if NShots < NRepeats:  # :85-90
        NShots = NRepeats
        NProfs = NShots * NEchos
        kTraj = np.tile(kTraj, (NRepeats, 1))
        NEchos = NProfs // NShots
    kRange = np.array([kRange3, kRange2], dtype=np.float64)  # :98-99
    kShift = np.floor((kRange[:, 1] - kRange[:, 0] + 1) / 2) + 1  # :100
    kSize = kRange[:, 1] - kRange[:, 0] + 1  # :101
    kIndex = (kTraj + kShift[None, :]).astype(np.int64)  # :102
    steady = NShots % NRepeats == 0 and NShots // NRepeats == 1  # :109-112
    if steady:  # :115-123
        kT = np.abs(_dct_ortho(kTraj))
        iM = int(np.min(np.argmax(kT[:NProfs // 2], axis=0))) + 1
        if iM <= 1:
            raise AcquisitionError("steady-state sequence with no sweep period in its trajectory")
        NSamples = NProfs / (iM - 1)
        NSweeps = int(round(NProfs / (NSamples * groupSweeps)))
        if NSweeps < 1:
            raise AcquisitionError("steady-state sequence: no sweeps with groupSweeps=%g" % groupSweeps)
    else:
        NSweeps = NShots
    sweepSample = np.ceil(NSweeps * ((np.arange(1, NProfs + 1) - 0.5) / NProfs)).astype(np.int64)  # :129
    NY = tuple(int(v) for v in (NY if NY is not None else kSize))
    k1, k2 = kIndex[:, 0] - 1, kIndex[:, 1] - 1
    if np.any(k1 < 0) or np.any(k2 < 0) or np.any(k1 >= NY[0]) or np.any(k2 >= NY[1]):
        raise AcquisitionError("profiles outside the %d x %d phase-encode grid" % NY)
    # :132-141: profile n goes to the first repeat slice whose grid point is
    # still empty; profiles beyond NRepeats visits of a point are dropped
    lin = k1 + NY[0] * k2
    order = np.argsort(lin, kind="stable")
    sl = np.empty(NProfs, np.int64)
    _, first, counts = np.unique(lin[order], return_index=True, return_counts=True)
    sl[order] = np.arange(NProfs) - np.repeat(first, counts)
    keep = sl < NRepeats
    timeIndex = np.zeros(NY + (NRepeats,), np.int64)
    timeIndex[k1[keep], k2[keep], sl[keep]] = np.arange(1, NProfs + 1)[keep]
    timeIndex = np.fft.ifftshift(timeIndex, axes=(0, 1))  # :142
    t0 = timeIndex[:, :, 0]
    H = np.zeros(NY, np.int64)
    H[t0 > 0] = sweepSample[t0[t0 > 0] - 1]  # stateSample = sweepSample (:130), E.mSt (:349-350)
    return {"NEchos": NEchos, "NShots": NShots, "NProfs": NProfs, "NSweeps": NSweeps, "steady_state": bool(steady),
            "kTraj": kTraj, "kShift": kShift, "kSize": kSize, "kIndex": kIndex, "sweepSample": sweepSample,
            "timeIndex": timeIndex, "H": H}


def profile_order(Shot, Echo, N, shots=None):
    """The scanner-side view of a DISORDER trajectory: the phase-encode
    coordinates (z2, z3) of every profile in acquisition order (shot by shot,
    echo by echo) from samplingDISORDER's shot and echo maps (N1 x N2 grids
    over the scanner's dims 3 and 2, centred), for acquisition_structure."""
    Shot = np.asarray(Shot)
    Echo = np.asarray(Echo)
    N = tuple(int(v) for v in N)
    sel = Shot > 0
    c = [np.arange(n) - n // 2 for n in N]
    k1 = np.broadcast_to(c[0][:, None], N)[sel]
    k2 = np.broadcast_to(c[1][None, :], N)[sel]
    order = np.lexsort((Echo[sel], Shot[sel]))
    return k2[order], k1[order]  # z{2} is grid dim 2, z{3} grid dim 1
