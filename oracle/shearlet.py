"""Shearlet system, shearlet regularizer and trace estimation (oracle).

TEST INFRASTRUCTURE ONLY. Restates in float64 (the reference builds in
single precision):
- Shearlets/buildShearlet.m:81-158, 3-D systems with complex=0;
- Shearlets/getShearletIdxs.m:1-74 (without the name/value filters);
- Shearlets/buildDirectionalFilter.m:25-47,149 ('ko' and 'kos');
- Shearlets/buildQuadratureMirrorFilter.m ('maxflat2');
- Shearlets/checkFilterFeasibility.m:1-38 (configuration 1 only);
- Shearlets/buildWedgeBandpassAndLowpassFilters.m:1-129 (complex=0);
- Methods/mirrorModulation.m, Methods/upsampling.m, Methods/shearing.m and
  Methods/resampling.m with fo=2 (centred crop / zero pad, no DFT);
- the shearlet branch of Reconstruction/regularize.m:27-46, computeShearlet
  of Reconstruction/CSsolver.m:91-101 and Reconstruction/traceEstimation.m.

Parity of this file against the reference is unpinned: the reference is
MATLAB, which is not available here, and it ships no shearlet outputs. The
tests check the system's structure (filter count, index table, the
ShearLab partition properties) and the device path against it.
"""

import math

import numpy as np

from .grids import fftGPU, ifftGPU

EPS = np.finfo(np.float64).eps


# ---------------------------------------------------------------- Methods helpers
def _msize(x):
    """MATLAB size(): at least two dimensions."""
    s = list(np.shape(x))
    return s + [1] * (2 - len(s)) if len(s) < 2 else s


def _as2d(v):
    """A MATLAB row vector (1 x L) from a 1-D array."""
    v = np.asarray(v)
    return v.reshape(1, -1) if v.ndim == 1 else v


def mirror_modulation(x, dirs=None):
    """Methods/mirrorModulation.m:13-24 (c = 0): multiply by (-1)^n along the
    given dims (1-based), n the index relative to floor(N/2)+1."""
    x = np.array(_as2d(x), dtype=np.float64)
    N = _msize(x)
    dirs = range(1, len(N) + 1) if dirs is None else dirs
    for d in ([dirs] if np.isscalar(dirs) else dirs):
        m = d - 1
        n = np.arange(1, N[m] + 1) - (N[m] // 2 + 1)
        shape = [1] * x.ndim
        shape[m] = N[m]
        x = x * np.where(n % 2 == 0, 1.0, -1.0).reshape(shape)
    return x


def upsampling(x, dims, ups=2, odd=1):
    """Methods/upsampling.m:14-25: insert ups-1 zeros between samples along
    each dim (1-based); the new length is ups*N-(ups-1)*odd."""
    x = np.asarray(x)
    for d in ([dims] if np.isscalar(dims) else dims):
        m = d - 1
        shp = list(x.shape)
        shp[m] = ups * shp[m] - (ups - 1) * odd
        out = np.zeros(shp, dtype=x.dtype)
        sl = [slice(None)] * x.ndim
        sl[m] = slice(0, None, ups)
        out[tuple(sl)] = x
        x = out
    return x


def resampling_space(x, Nres):
    """Methods/resampling.m with fo=2: per dim whose size changes, keep (crop)
    or place (zero pad) the centred range orig:fina, zeroF = ceil((Nmax+1)/2),
    orig = zeroF - ceil((Nmin-1)/2), fina = zeroF + floor((Nmin-1)/2)."""
    x = np.asarray(x)
    Nres = list(Nres)
    for m in range(len(Nres)):
        Nor = x.shape[m]
        if Nor == Nres[m]:
            continue
        Nmin, Nmax = min(Nor, Nres[m]), max(Nor, Nres[m])
        zeroF = math.ceil((Nmax + 1) / 2)
        orig = zeroF - math.ceil((Nmin - 1) / 2)
        fina = zeroF + (Nmin - 1) // 2
        sl = [slice(None)] * x.ndim
        sl[m] = slice(orig - 1, fina)
        if Nor < Nres[m]:
            shp = list(x.shape)
            shp[m] = Nres[m]
            out = np.zeros(shp, dtype=x.dtype)
            out[tuple(sl)] = x
            x = out
        else:
            x = x[tuple(sl)]
    return x


def shearing_21(x, k):
    """Methods/shearing.m:13-19 with dims = [2 1]: row n1 of x is shifted
    along dim 2 by -k*(n1 - floor(N1/2) - 1), through the DFT phase ramp of
    Methods/shifting.m:38-47 (the shift is an array, so the DFT branch)."""
    if k == 0:
        return x
    N1, N2 = x.shape
    h = -k * (np.arange(1, N1 + 1) - (N1 // 2 + 1)).astype(np.float64)
    kg = (2 * np.pi / N2) * (np.arange(1, N2 + 1) - math.ceil((N2 + 1) / 2))
    kg = np.fft.ifftshift(kg)
    ph = np.exp(-1j * h[:, None] * kg[None, :])
    return ifftGPU(fftGPU(x, 1) * ph, 1)


def _conv2_col(a, col):
    """conv2(a, col) for a column vector col: full 2-D convolution."""
    out = np.zeros((a.shape[0] + len(col) - 1, a.shape[1]), dtype=np.result_type(a, col))
    for j in range(a.shape[1]):
        out[:, j] = np.convolve(a[:, j], col)
    return out


def _fft2d(x):
    """buildWedgeBandpassAndLowpassFilters.m:121-123: ifftshift then DFT, dims 1, 2."""
    for m in (0, 1):
        x = fftGPU(np.fft.ifftshift(x, axes=m), m)
    return x


def _ifft2d(x):
    """buildWedgeBandpassAndLowpassFilters.m:125-127: inverse DFT then fftshift."""
    for m in (0, 1):
        x = np.fft.fftshift(ifftGPU(x, m), axes=m)
    return x


# ---------------------------------------------------------------- filters
def directional_filter(DFtype="kos"):
    """Shearlets/buildDirectionalFilter.m:34-47 (di = 1) and :149 (modu = 1):
    Kovacevic's orthogonal 3 x 4 diamond filter ('ko', or its smooth version
    'kos'), normalised to sum sqrt(2), then mirror-modulated along dim 2 at
    1/sqrt(2)."""
    if DFtype == "ko":
        a0, a1, a2 = 2.0, 0.5, 1.0
    elif DFtype == "kos":
        a0, a1, a2 = -math.sqrt(3), -math.sqrt(3), 2 + math.sqrt(3)
    else:
        raise NotImplementedError("directional filter %s" % DFtype)
    h0 = np.array([[0, -a1, -a0 * a1, 0],
                   [-a2, -a0 * a2, -a0, 1],
                   [0, a0 * a1 * a2, -a1 * a2, 0]], dtype=np.float64)
    h0 = h0 * (math.sqrt(2) / h0.sum())
    return mirror_modulation(h0 / math.sqrt(2), 2)


# maximally flat 9-tap lowpass of buildQuadratureMirrorFilter.m (maxflat, P = 2)
_MAXFLAT2 = (.0104933261758410, -.0263483047033631, -.0517766952966370, .276348304703363, .582566738241592,
             .276348304703363, -.0517766952966369, -.0263483047033631, .0104933261758408)


def qmf_filter(QMFtype="maxflat2"):
    """Shearlets/buildQuadratureMirrorFilter.m: the 1-D scaling filter,
    normalised to unit sum (:60)."""
    if QMFtype != "maxflat2":
        raise NotImplementedError("quadrature mirror filter %s" % QMFtype)
    f = np.array(_MAXFLAT2, dtype=np.float64)
    return _as2d(f / f.sum())


def check_filter_feasibility(N, K, DF, SF):
    """Shearlets/checkFilterFeasibility.m:16-38 for configuration 1 (the
    requested filters). Returns (DF, SF, WF, SF2)."""
    WF = mirror_modulation(SF)
    SF2 = SF
    L = SF.size
    lcheck1 = L
    for _ in range(len(K) - 1):
        lcheck1 = L + 2 * (lcheck1 - 1)
    lcheck2 = L
    for _ in range(max(K)):
        lcheck2 = L + 2 * (lcheck2 - 1)
    lcheck2 = lcheck2 + (DF.shape[0] - 1) * 2 ** (max(K) + 1)
    if any(lcheck1 > n for n in N) or any(lcheck2 > n for n in N) or any(DF.shape[1] > n for n in N):
        raise NotImplementedError("shearlet system not available for size %s with the requested filters "
                                  "(needs every dimension >= %d)" % (list(N), max(lcheck1, lcheck2)))
    return DF, SF, WF, SF2


def wedge_bandpass_lowpass(N, K, DF, SF1, WF, SF2):
    """Shearlets/buildWedgeBandpassAndLowpassFilters.m:34-119 (complex = 0).
    Returns (WD, BP, LP): WD[k] the (N1, N2, 2^(k+1)+1) wedge filters of
    shear level k (dict), BP (N1, N2, J) the bandpass filters, LP the lowpass,
    all in the frequency domain with frequency 0 first."""
    N = list(N)
    J = len(K)
    Kmax = max(K) + 1
    DF = DF / np.abs(DF).sum()
    FHP = [None] * J
    FLP1 = [None] * J
    FLP2 = [None] * Kmax
    FHP[J - 1] = _as2d(WF)
    FLP1[J - 1] = _as2d(SF1)
    FLP2[Kmax - 1] = _as2d(SF2)
    for j in range(J - 2, -1, -1):  # :47-50
        FLP1[j] = _as2d(np.convolve(FLP1[J - 1].ravel(), upsampling(FLP1[j + 1], 2).ravel()))
        FHP[j] = _as2d(np.convolve(FLP1[J - 1].ravel(), upsampling(FHP[j + 1], 2).ravel()))
    for k in range(Kmax - 2, -1, -1):  # :51-53
        FLP2[k] = _as2d(np.convolve(FLP2[Kmax - 1].ravel(), upsampling(FLP2[k + 1], 2).ravel()))
    BP = np.zeros(N + [J], dtype=np.complex128)
    for j in range(J):  # :56-57
        BP[:, :, j] = _fft2d(resampling_space(FHP[j], N).astype(np.complex128))
    WD = {}
    for k in sorted(set(K)):  # :72-116
        WD[k] = np.zeros(N + [2 ** (k + 1) + 1], dtype=np.complex128)
        DFups = upsampling(DF, 1, 2 ** (k + 1))
        col = FLP2[Kmax - k - 1].ravel()
        WDups = upsampling(resampling_space(_conv2_col(DFups, col), N), 2, 2 ** k).astype(np.complex128)
        FLPaux = resampling_space(FLP2[Kmax - max(k - 1, 0) - 1], WDups.shape).astype(np.complex128)
        if k >= 1:
            WDups = _ifft2d(_fft2d(WDups) * _fft2d(FLPaux))
        FLPauxfl = np.flip(FLPaux, 1)
        for l in range(-2 ** k, 2 ** k + 1):
            sh = shearing_21(WDups, l)
            if k >= 1:
                sh = _ifft2d(_fft2d(sh) * _fft2d(FLPauxfl))
            sh = (2 ** k) * sh[:, 0:(2 ** k) * N[1]:2 ** k]
            WD[k][:, :, 2 ** k - l] = _fft2d(sh)
    LP = _fft2d(resampling_space(FLP1[0].T @ FLP1[0], N).astype(np.complex128))  # :119
    return WD, BP, LP


# ---------------------------------------------------------------- the system
def shearlet_idxs(ND, K, full=0):
    """Shearlets/getShearletIdxs.m:29-74 (complex = 0, every scale, shearing,
    cone and pyramid): rows [cone scale half shearing] (2-D) or [pyramid
    scale half shearing1 shearing2] (3-D), 1-based, the lowpass row last."""
    rows = []
    if ND == 2:
        for cone in (1, 2):
            for scale in range(1, len(K) + 1):
                s = 2 ** K[scale - 1]
                for sh in range(-s, s + 1):
                    if full or cone == 1 or abs(sh) < s:
                        rows.append([cone, scale, 1, sh])
        rows.append([0, 0, 0, 0])
    elif ND == 3:
        for pyr in (1, 2, 3):
            for scale in range(1, len(K) + 1):
                s = 2 ** K[scale - 1]
                for sh1 in range(-s, s + 1):
                    for sh2 in range(-s, s + 1):
                        if full or pyr == 1 or (pyr == 2 and abs(sh2) < s) or (abs(sh1) < s and abs(sh2) < s):
                            rows.append([pyr, scale, 1, sh1, sh2])
        rows.append([0, 0, 0, 0, 0])
    else:
        raise ValueError("ND must be 2 or 3")
    return np.array(rows, dtype=np.int64)


def _ind_from_idxs(K, cone, scale, half, shearing):
    """buildShearlet.m:155-158 (complex = 0), 1-based."""
    K = np.asarray(K)
    ind = int(np.sum(2 ** (K + 1) + 1)) * (cone - 1) + 2 ** int(K[scale - 1]) + half + shearing
    if scale > 1:
        ind += int(np.sum(2 ** (K[:scale - 1] + 1) + 1))
    return ind


def _normalization(S, nd):
    """buildShearlet.m:148-153: rms per shearlet and the dual frame weights."""
    A = np.abs(S) ** 2
    rms = np.sqrt(A.reshape(-1, A.shape[-1]).sum(0) / np.prod(S.shape[:nd]))
    return rms, A.sum(-1)


# the 2-D systems' dimension pairs (buildShearlet.m:90-91), 0-based
PAIRS = ((0, 1), (0, 2), (2, 1))


def shearlet_planes(N, K, DFtype="kos", QMFtype="maxflat2"):
    """buildShearlet.m:99-109: the 2-D shearlet systems (full = 1) of the three
    dimension pairs, as a list of (Na, Nb, NS2) arrays (Na = N[pair[0]])."""
    idxs2 = shearlet_idxs(2, K, 1)
    DF = directional_filter(DFtype)
    SF = qmf_filter(QMFtype)
    out = []
    for pair in PAIRS:
        Nc = [N[pair[0]], N[pair[1]]]
        DFc, SF1, WF, SF2 = check_filter_feasibility(Nc, K, DF, SF)
        F = []
        Ncur = list(Nc)
        for _ in range(2):  # :115-122
            F.append(wedge_bandpass_lowpass(Ncur, K, DFc, SF1, WF, SF2))
            Ncur = Ncur[1:] + Ncur[:1]
        S = np.zeros(Nc + [len(idxs2)], dtype=np.complex128)
        for s, (cone, scale, half, sh) in enumerate(idxs2):  # :124-134
            if cone == 0:
                S[:, :, s] = F[0][2]
            elif cone == 1:
                kk = K[scale - 1]
                S[:, :, s] = F[0][0][kk][:, :, -sh + 2 ** kk] * np.conj(F[0][1][:, :, scale - 1])
            else:
                kk = K[scale - 1]
                S[:, :, s] = (F[1][0][kk][:, :, sh + 2 ** kk] * np.conj(F[1][1][:, :, scale - 1])).T
        out.append(S)
    return out


def _place(S2, pair, N):
    """buildShearlet.m:107-108: the pair's 2-D filters as a broadcastable
    (N1|1, N2|1, N3|1, NS2) array."""
    shape = [1, 1, 1, S2.shape[2]]
    a, b = pair
    shape[a] = N[a]
    shape[b] = N[b]
    if a < b:
        return S2.reshape(shape)
    return np.transpose(S2, (1, 0, 2)).reshape(shape)


def buildShearlet(N, J=1, K=None, DFtype="kos", QMFtype="maxflat2", full=0):
    """Shearlets/buildShearlet.m:81-113 for 3-D N. Returns a dict with S
    (N1, N2, N3, NW) complex, idxs (NW x 5), dfw and rms."""
    if K is None:
        K = [int(math.ceil(j / 2)) for j in range(1, J + 1)]
    K = [int(k) for k in K]
    N = [int(n) for n in N]
    if len(N) != 3:
        raise NotImplementedError("only 3-D shearlet systems are restated")
    planes = [_place(S2, pair, N) for S2, pair in zip(shearlet_planes(N, K, DFtype, QMFtype), PAIRS)]
    idxs = shearlet_idxs(3, K, full)
    S = np.zeros(N + [len(idxs)], dtype=np.complex128)
    P1, P2, P3 = planes
    for s, (pyr, scale, half, sh1, sh2) in enumerate(idxs):  # :136-146
        if pyr == 0:
            v = P1[..., -1] * P3[..., -1]
        elif pyr == 1:
            v = P1[..., _ind_from_idxs(K, 1, scale, half, sh1) - 1] * P3[..., _ind_from_idxs(K, 1, scale, half, sh2) - 1]
        elif pyr == 2:
            v = P2[..., _ind_from_idxs(K, 1, scale, half, sh1) - 1] * P3[..., _ind_from_idxs(K, 2, scale, half, sh2) - 1]
        else:
            v = P1[..., _ind_from_idxs(K, 2, scale, half, sh1) - 1] * P2[..., _ind_from_idxs(K, 2, scale, half, sh2) - 1]
        S[..., s] = v
    rms, dfw = _normalization(S, 3)
    return {"S": S, "K": K, "full": full, "idxs": idxs, "dfw": dfw, "rms": rms}


# ---------------------------------------------------------------- shearlet operators
def _fft3(x):
    for m in range(3):
        x = fftGPU(x, m)
    return x


def _ifft3(x):
    for m in range(3):
        x = ifftGPU(x, m)
    return x


def compute_shearlet(x, S):
    """Reconstruction/CSsolver.m:91-101: |IDFT(conj(S_w) .* DFT(x))| for every
    shearlet w, as an (N1, N2, N3, NW) real array."""
    xF = _fft3(np.asarray(x, np.complex128))
    return np.stack([np.abs(_ifft3(np.conj(S[..., w]) * xF)) for w in range(S.shape[-1])], axis=-1)


def regularize_sh(x, S, We, la, p=1.0):
    """Reconstruction/regularize.m:27-46: (la p / 2) IDFT(sum_w S_w .* DFT(We_w
    .* IDFT(conj(S_w) .* DFT(x))))."""
    xF = _fft3(np.asarray(x, np.complex128))
    acc = np.zeros_like(xF)
    for w in range(S.shape[-1]):
        t = _ifft3(np.conj(S[..., w]) * xF) * We[..., w]
        acc += S[..., w] * _fft3(t)
    return (la * p / 2) * _ifft3(acc)


def _we_grid(E, EH):
    """traceEstimation.m:42-49: the per-sample weights EH.We on the (ky, kz)
    grid. Grid points that no sample hits get weight 0 (the reference leaves
    the entries that iSt does not overwrite as they were, which matters only
    when the samples do not cover the grid)."""
    W = np.zeros((E.Sf.shape[0], E.Sf.shape[1]))
    np.add.at(W, (np.asarray(E.ky), np.asarray(E.kz)), np.asarray(EH.We, np.float64))
    return W


def trace_estimation(x, E=None, EH=None, C=None, R=None, tol=1e-2, BlSz=1, noise=None):
    """Reconstruction/traceEstimation.m:1-113 (no SENSE folding, no resampling).
    noise(shape) draws the real Gaussian probes (plugNoise(x, 1)); rounds of
    BlSz probes run until the standard error of the mean is below tol of
    the mean (at least 2 probes). Returns (tr, trF)."""
    NX = tuple(np.shape(x)[:3])
    N = int(np.prod(NX))
    W = _we_grid(E, EH) if (E is not None and EH is not None and EH.has("We")) else None
    trF = []
    while True:
        tr_round = []
        for _ in range(BlSz):
            v = np.asarray(noise(NX), np.float64)
            v = v / np.sqrt(np.sum(v * v) / N)  # :55
            if C is not None and C.has("Ma"):
                v = v * C.Ma
            tc = 0.0
            if E is not None:  # :61-84
                xs = v[..., None] * np.asarray(E.Sf, np.complex128)
                if W is not None:
                    for m in (0, 1):
                        xs = fftGPU(xs, m) / np.sqrt(xs.shape[m])
                    tc += float(np.sum(W[:, :, None, None] * np.abs(xs) ** 2))
                else:
                    tc += float(np.sum(np.abs(xs) ** 2))
            if R is not None and R.has("Sh"):  # :85-102
                S, We = R.Sh.S, R.Sh.We
                xF = _fft3(v.astype(np.complex128))
                for w in range(S.shape[-1]):
                    t = _ifft3(np.conj(S[..., w]) * xF)
                    tc += float(np.sum(We[..., w] * np.abs(t) ** 2))
            tr_round.append(tc)
        trF.extend(tr_round)
        n = len(trF)
        mea = float(np.mean(trF))
        std = float(np.std(trF, ddof=1)) / np.sqrt(n) if n > 1 else np.inf
        if n >= 2 and std / (mea + EPS) < tol:  # :106-112
            return mea, np.array(trF)
