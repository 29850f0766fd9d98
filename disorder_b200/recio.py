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

``prepare_rec`` is the data steps before it (solveXT.m:39-72): the readout
ROI (computeROI / extractROI), the permutation of the phase encodes to the
front, the Tukey apodization (buildFilter 'tukey') and the averages folded
into dimension 5 (resSub). Not restated: reading ``rec`` files, which
writeRaw.m saves as MATLAB v7.3 (HDF5) files.
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


# ---------------------------------------------------------------- data preparation
def compute_roi(x, ext=0, sy=None, ev=None, fu=0):
    """Methods/computeROI.m:20-57: the bounding box of |x| > 1e-6 per
    dimension (the first 3 unless fu), widened by ext, optionally made
    symmetric (sy) or of even extent (ev). Rows [first last N extent before
    after], 1-based like the reference."""
    a = np.abs(np.asarray(x)) > 1e-6
    ND = a.ndim if fu else min(a.ndim, 3)
    sy = np.zeros(ND) if sy is None else np.asarray(sy)
    ev = np.zeros(ND) if ev is None else np.asarray(ev)
    if not a.any():
        raise ValueError("computeROI: the array has no element above 1e-6")
    ROI = np.zeros((ND, 6), np.int64)
    for n in range(ND):
        other = tuple(d for d in range(a.ndim) if d != n)
        hit = np.flatnonzero(a.any(axis=other))
        ROI[n, :3] = (hit[0] + 1, hit[-1] + 1, a.shape[n])
    ROI[:, 0] = np.maximum(ROI[:, 0] - ext, 1)
    ROI[:, 1] = np.minimum(ROI[:, 1] + ext, ROI[:, 2])
    ROI[:, 3] = ROI[:, 1] - ROI[:, 0] + 1
    ROI[:, 4] = ROI[:, 0] - 1
    ROI[:, 5] = ROI[:, 2] - ROI[:, 1]
    for n in range(ND):
        if sy[n]:
            d = ROI[n, 5] - ROI[n, 4]
            ROI[n, [1 if ROI[n, 4] <= ROI[n, 5] else 0, 3]] += d  # the side with the smaller margin
            ROI[n, 5] = ROI[n, 4]
        if ev[n] and ROI[n, 3] % 2:
            ROI[n, 3] -= 1
            ROI[n, [0, 4]] += 1
    return ROI


def extract_roi(x, ROI, ext=1, dims=None):
    """Methods/extractROI.m:14-28: crop x to ROI rows first:last along dims
    (ext = 1), or place x there in zeros of the full size (ext = 0)."""
    x = np.asarray(x)
    ND = min(ROI.shape[0], x.ndim)
    dims = list(range(1, ND + 1)) if dims is None else ([dims] if np.isscalar(dims) else list(dims))
    sl = [slice(None)] * x.ndim
    for d in dims:
        sl[d - 1] = slice(int(ROI[d - 1, 0]) - 1, int(ROI[d - 1, 1]))
    if ext:
        return x[tuple(sl)]
    shape = list(x.shape)
    for d in dims:
        shape[d - 1] = int(ROI[d - 1, 2])
    y = np.zeros(shape, dtype=x.dtype)
    y[tuple(sl)] = x
    return y


def tukey_filter(N, sp, gibbsRing):
    """Methods/buildFilter.m:93-101 ('tukey', c = 0): the product over dims
    of 1-D Tukey windows of the radial k of each dim,
    k = 2 pi |n - ceil((N+1)/2)| / (sp N) (generateGrid with nor 2 i pi / sp,
    :29), 1 below pi (1 - g), a raised cosine up to pi, 0 beyond
    (tukeyIso, :86-92); then fftshift."""
    N = [int(n) for n in N]
    ND = len(N)
    sp = np.broadcast_to(np.asarray(sp, np.float64), (ND,))
    g = list(np.atleast_1d(np.asarray(gibbsRing, np.float64)))
    g = g + [g[-1]] * (ND - len(g))
    x = np.ones(N)
    for m in range(ND):
        n = np.arange(1, N[m] + 1)
        kk = np.abs(2 * np.pi / sp[m] / N[m] * (n - math.ceil((N[m] + 1) / 2)))
        w = np.ones(N[m])
        alpha = 1 - g[m]
        if g[m] != 0:
            taper = kk >= np.pi * alpha
            w[taper] = 0.5 * (1 + np.cos(np.pi * ((kk[taper] - np.pi * alpha) / ((1 - alpha) * np.pi))))
        w[kk >= np.pi] = 0
        shape = [1] * ND
        shape[m] = N[m]
        x = x * w.reshape(shape)
    return np.fft.fftshift(x)


def merge_averages(y, first=5):
    """Methods/resSub.m:15-30 with orDim = first:ndims: the dimensions from
    `first` (1-based) on folded into one."""
    y = np.asarray(y)
    if y.ndim < first:
        return y
    return y.reshape(y.shape[:first - 1] + (int(np.prod(y.shape[first - 1:])),), order="F")


def prepare_rec(y, S, M, voxSiz, apod=(0.1, 0.0, 0.0)):
    """The data steps of solveXT.m:39-72 in their order: the readout ROI of
    the mask with even extent (computeROI(rec.M,[],[0 0 0],[1 0 0]), :40),
    y, S and M cropped to it along dim 1 (extractROI(.,ROI,1,1), :45-47),
    the phase encodes permuted to the front (perm(1:3) = [3 2 1], :50-57),
    the Tukey apodization of y (buildFilter(NY(1:3),'tukey',[10 10 1],gpu,
    apod) ifftshifted, :70) and the averages folded into dim 5 (resSub,
    :71). Returns a dict with y, S, M, ROI, voxSiz and NY (the size of y
    with the averages as dim 5)."""
    M = np.asarray(M)
    ROI = compute_roi(M, 0, [0, 0, 0], [1, 0, 0])
    y = extract_roi(y, ROI, 1, 1)
    S = extract_roi(S, ROI, 1, 1)
    M = extract_roi(M, ROI, 1, 1)
    perm = lambda a: np.transpose(a, (2, 1, 0) + tuple(range(3, np.ndim(a))))  # noqa: E731
    y, S, M = perm(y), perm(S), perm(M)
    voxSiz = tuple(np.asarray(voxSiz, np.float64)[[2, 1, 0]])
    ap = np.asarray(apod, np.float64)[[2, 1, 0]]
    NY = y.shape
    w = np.fft.ifftshift(tukey_filter(NY[:3], [10, 10, 1], ap)).astype(np.float32 if y.dtype == np.complex64
                                                                     else np.float64)
    y = y * w.reshape(NY[:3] + (1,) * (y.ndim - 3))
    y = merge_averages(y, 5)
    NYo = tuple(y.shape) + (1,) * (5 - y.ndim)
    return {"y": y, "S": S, "M": M, "ROI": ROI, "voxSiz": voxSiz, "NY": NYo}
