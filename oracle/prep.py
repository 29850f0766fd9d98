"""Data preparation around the hot path (oracle; test infrastructure).

Restates Methods/compressCoils.m:76-118 (useFold=0 branch),
Methods/pyramidPlan.m:19-33, Methods/resampling.m:16-95 (no mirroring,
complex input) and Methods/buildHarmonicSampling.m:25-50.
"""

import numpy as np

from .grids import fftGPU, ifftGPU


def compressCoils(S, perc, y=None, reg=1e-9):
    """Methods/compressCoils.m:76-118 (the branch taken when the coil and data
    grids agree). S: (N1,N2,N3,C). y: samples with coils on the last axis.

    P = sum_voxels S~ S^H with S~ = S/(sum_c |S|^2 + reg) (:78-88); [U,D] =
    svd(P) (:93); C(n) = first count whose cumulative singular value share
    reaches perc(n) (or perc(n) itself when >= 1) (:107-110); A = U(:,1:C)^H;
    S <- A S, y <- A y along the coil dim (:115-118). P is Hermitian positive
    semi-definite, so its SVD is its eigendecomposition.
    Returns (S, y, C, D, U, P).
    """
    perc = np.atleast_1d(np.asarray(perc, float))
    nrm = np.sum(np.abs(S) ** 2, axis=3, keepdims=True)
    Saux = S / (nrm + reg)
    Sf = S.reshape(-1, S.shape[3])
    P = Saux.reshape(-1, S.shape[3]).T @ np.conj(Sf)  # P(c,c') = sum Saux_c conj(S_c')
    U, D, _ = np.linalg.svd(P)
    D = np.abs(D)
    C = np.zeros(len(perc), int)
    cs = np.cumsum(D) / np.sum(D)
    for n, pc in enumerate(perc):
        C[n] = int(np.argmax(cs >= pc)) + 1 if pc < 1 else int(pc)
    A = np.conj(U[:, :C.max()]).T
    So = np.tensordot(S, A, axes=([3], [1]))
    yo = None
    if y is not None:
        yo = np.moveaxis(np.tensordot(A, np.moveaxis(y, -1, 0), axes=([1], [0])), 0, -1)
    return So, yo, C, D, U, P


def pyramidPlan(voxSiz, resolMax=4, NWend=1, accel=(1, 0)):
    """Methods/pyramidPlan.m:19-33. Returns (resPyr, L, estT, resIso)."""
    voxSiz = np.asarray(voxSiz, float)
    Lr = int(np.round(np.log2(max(resolMax / voxSiz.min(), 1)))) + 1
    resPyr = 1.0 / np.flip(2.0 ** np.arange(Lr))
    L = Lr + int(np.round(np.log2(NWend)))
    resPyr = np.concatenate([resPyr, np.ones(L - Lr)])
    estT = np.ones(L, int)
    estT[max(L - accel[0], 0):L] = 0
    resIso = np.sqrt(2) * (np.prod(voxSiz) ** (1 / 3)) / resPyr
    L = max(L - accel[1], 1)
    return resPyr[:L], L, estT[:L], resIso[:L]


def resampling(x, Nres, fo=0):
    """Methods/resampling.m:16-95 for complex arrays, mirror=0: per changed
    dim, (fo=0) DFT/Nor, fftshift, centred crop/zero-pad to Nres, ifftshift,
    (fo=0) inverse DFT*Nres. fo=1: input/output already in (DC-first) k-space;
    fo=2: already shifted k-space."""
    Nres = list(Nres)
    for m, nr in enumerate(Nres):
        no = x.shape[m]
        if no == nr:
            continue
        Nmin, Nmax = min(no, nr), max(no, nr)
        zeroF = int(np.ceil((Nmax + 1) / 2))
        orig = zeroF - int(np.ceil((Nmin - 1) / 2))
        fina = zeroF + int(np.floor((Nmin - 1) / 2))
        if fo == 0:
            x = fftGPU(x, m) / no
        if fo != 2:
            x = np.fft.fftshift(x, axes=m)
        sl = [slice(None)] * x.ndim
        sl[m] = slice(orig - 1, fina)
        if no < nr:
            shp = list(x.shape)
            shp[m] = nr
            xr = np.zeros(shp, dtype=x.dtype)
            xr[tuple(sl)] = x
            x = xr
        else:
            x = x[tuple(sl)]
        if fo != 2:
            x = np.fft.ifftshift(x, axes=m)
        if fo == 0:
            x = ifftGPU(x, m) * nr
    return x


def buildHarmonicSampling(state_map, NStates):
    """Methods/buildHarmonicSampling.m:25-50 for the index part: state_map is
    the (NY1, NY2, NRep) array H of 1-based motion states (0 = no state). For
    s = 1..NStates+1 the samples are the column-major linear indices where
    H == mod(s, NStates+1) (:37). Returns 0-based per-sample (ky, kz, rep),
    the linear indices iSt (to pick y rows), segment offsets nSt and the
    0-based segment of each sample mSt."""
    H = np.asarray(state_map)
    NH = H.shape + (1,) * (3 - H.ndim)
    Hf = H.reshape(-1, order="F")
    idx_all, seg_all = [], []
    for s in range(1, NStates + 2):
        ind = np.flatnonzero(Hf == (s % (NStates + 1)))
        idx_all.append(ind)
        seg_all.append(np.full(len(ind), s - 1))
    iSt = np.concatenate(idx_all)
    mSt = np.concatenate(seg_all)
    ky, kz, rep = np.unravel_index(iSt, NH, order="F")
    nSa = np.array([len(i) for i in idx_all])
    nSt = np.concatenate([[0], np.cumsum(nSa)])
    return ky.astype(np.int32), kz.astype(np.int32), rep.astype(np.int32), iSt, nSt, mSt
