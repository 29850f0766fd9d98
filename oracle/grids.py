"""Grids, DFT matrices and DFT-along-an-axis helpers (oracle; test infrastructure).

Restates Methods/generateGrid.m, Methods/generateTransformGrids.m,
Methods/build1DFTM.m, Methods/buildStandardDFTM.m, Methods/fftGPU.m and
Methods/ifftGPU.m.
"""

import numpy as np

try:  # multithreaded FFTs for the timed CPU baseline; same arithmetic as numpy
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

# Number of FFT worker threads (1 keeps tests deterministic and light).
WORKERS = 1

# per = [1 3 2; 2 1 3] in 0-based form (generateTransformGrids.m:55-56)
PER = np.array([[0, 2, 1], [1, 0, 2]])


def _fft(x, axis):
    if _sfft is not None:
        return _sfft.fft(x, axis=axis, workers=WORKERS)
    return np.fft.fft(x, axis=axis)


def _ifft(x, axis):
    if _sfft is not None:
        return _sfft.ifft(x, axis=axis, workers=WORKERS)
    return np.fft.ifft(x, axis=axis)


def fftGPU(x, m):
    """DFT along axis m with the unnormalised DFT matrix F = dftmtx(N).

    Methods/fftGPU.m:27-45 applies F (build1DFTM(N,0), build1DFTM.m:21) along
    dim m by reshape+GEMM; F_jk = exp(-2*pi*i*j*k/N) with DC first, which is
    exactly the standard forward DFT.
    """
    return _fft(x, m)


def ifftGPU(x, m):
    """Inverse DFT along axis m with FH = conj(F)/N (Methods/ifftGPU.m:23-48,
    build1DFTM.m:30-31,52)."""
    return _ifft(x, m)


def along(v, axis, ndim=5):
    """Reshape a 1-D vector so that it lies along ``axis`` of an ndim array
    (the permute in generateGrid.m:37-38)."""
    shape = [1] * ndim
    shape[axis] = -1
    return np.reshape(v, shape)


def generateGrid(N, nor=1.0, cent=None, shift=0):
    """Methods/generateGrid.m:27-40. Returns (pGrid list of 1-D float32, cent).

    pGrid{m} = single((nor(m)/N(m))*((1:N(m))-cent(m))); the value is formed in
    double precision and then rounded to single, as in the reference.
    """
    N = [int(n) for n in N]
    nd = len(N)
    if cent is None:
        cent = [(n + 1) / 2.0 for n in N]
    cent = [c - shift for c in np.broadcast_to(np.asarray(cent, float), (nd,))]
    nor = np.broadcast_to(np.asarray(nor, float), (nd,))
    grids_ = []
    for m in range(nd):
        g = (nor[m] / N[m]) * (np.arange(1, N[m] + 1, dtype=np.float64) - cent[m])
        grids_.append(g.astype(np.float32))
    return grids_, cent


class TransformGrids:
    """Output of generateTransformGrids (Methods/generateTransformGrids.m:23-67).

    rGrid[m], kGrid[m]: 1-D float32 vectors along axis m (kGrid ifftshifted when
    sh=1, :50-52). rk(n, m) returns rkGrid{n}{m} = rGrid{per(3-n,m)} .*
    kGrid{per(n,m)} as a 5-D float32 array (:57-62). cGrid is the grid centre.
    """

    def __init__(self, rGrid, kGrid, cGrid, sh):
        self.rGrid = rGrid
        self.kGrid = kGrid
        self.cGrid = cGrid
        self.sh = sh

    @property
    def N(self):
        return [len(k) for k in self.kGrid]

    def rk(self, n, m, ndim=5):
        """rkGrid{n}{m} for n in {1,2} (1-based like the reference), m 0-based."""
        ra = PER[2 - n, m]  # per(3-n, m)
        ka = PER[n - 1, m]  # per(n, m)
        return (along(self.rGrid[ra], ra, ndim) * along(self.kGrid[ka], ka, ndim)).astype(np.float32)


def generateTransformGrids(N, Nres=None, cent=None, sh=0):
    """Methods/generateTransformGrids.m:23-67 (no slabs, no prods).

    N is the full-resolution size; Nres the grid size at this level (defaults
    to N). rGrid is in full-resolution voxel units and kGrid in radians per
    full-resolution voxel (:48-49).
    """
    N = list(N) + [1] * (3 - len(N))
    N = [int(n) for n in N[:3]]
    if Nres is None:
        Nres = [int(round(n)) for n in N]
    Nres = [int(n) for n in Nres]
    if cent is None:
        cent = [n / 2.0 + 1 for n in Nres]
    rGrid, cGrid = generateGrid(Nres, nor=N, cent=cent)
    kc = [np.ceil((n + 1) / 2.0) for n in Nres]
    kGrid, _ = generateGrid(Nres, nor=[2 * np.pi * Nres[m] / N[m] for m in range(3)], cent=kc)
    if sh:
        kGrid = [np.fft.ifftshift(k) for k in kGrid]
    return TransformGrids(rGrid, kGrid, cGrid, sh)


def build1DFTM(N, fn=0):
    """Methods/build1DFTM.m:21-31,52 (re=0): F = single(dftmtx(N)); F/sqrt(N)
    when fn; FH = conj(F) (divided by N when fn == 0). dftmtx(N)_jk =
    exp(-2*pi*i*j*k/N) is restated from its definition (0-based j, k)."""
    j = np.arange(N)
    F = np.exp(-2j * np.pi * np.outer(j, j) / N)
    if fn:
        F = F / np.sqrt(N)
    FH = np.conj(F)
    if not fn:
        FH = FH / N
    return F, FH
