"""Compressed-sensing reconstruction with a shearlet regularizer
(Reconstruction/CSsolver.m:1-103) on the device.

The shearlet system is built on the host as 2-D planes
(disorder_b200.shearlet) and held by the library (disorder_shearlet_create);
computeShearlet, the regularizer term and the trace estimates run as device
passes (csrc/shearlet.cu), and the inner CG is the library's CG with the
shearlet term in its normal operator (disorder_cg_solve_shearlet).

Differences from the reference, all on paths this module does not take:
- input and output grids are the same (CSsolver.m:41-48,74 resample from
  E.NXAcq to EH.NXRec; a different output grid raises);
- checkFilterFeasibility's fallback filter configurations 2-7 are not built
  (grids below 33 voxels along a dimension raise);
- the trace estimate's weight grid is zero where no sample falls
  (traceEstimation.m:42-49 keeps whatever EH.We held there).
"""

import ctypes as C

import numpy as np

from . import shearlet as _sh
from ._lib import DisorderError
from .api import DeviceArray, Struct, CGsolver, _dev, default_context

EPS = np.finfo(np.float64).eps


class ShearletSystem:
    """A shearlet system of a 3-D grid on the device (disorder_shearlet):
    buildShearlet(N, J, 0, K, DFtype) of Shearlets/buildShearlet.m."""

    def __init__(self, ctx, N, J=1, K=None, DFtype="kos", QMFtype="maxflat2", full=0):
        self.ctx = ctx
        self.N = tuple(int(n) for n in N)
        planes, table, idxs = _sh.build_planes(self.N, J, K, DFtype, QMFtype, full)
        self.idxs = idxs
        self.table = table
        self.n_filters = len(table)
        self.h = None
        h = C.c_void_p()
        Nc = (C.c_int32 * 3)(*self.N)
        tab = np.ascontiguousarray(table.ravel(), dtype=np.int32)
        ctx.check(ctx.lib.disorder_shearlet_create(
            ctx.h, Nc, planes[0].shape[2], planes[0].ctypes.data, planes[1].ctypes.data, planes[2].ctypes.data,
            self.n_filters, tab.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(h)))
        self.h = h
        ctx.adopt(self)

    @property
    def V(self):
        return int(np.prod(self.N))

    def close(self):
        if self.h is not None and self.ctx.h is not None:
            self.ctx.lib.disorder_shearlet_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def coefficients(self, x, eps=1e-2, p=1.0, out=None):
        """R.Sh.We of CSsolver.m:58-59,78-80: (|IDFT(conj(S_w) .* DFT(x))| +
        eps)^(p-2) for every shearlet, a device (N1, N2, N3, NW) float32 array."""
        xd, _ = _dev(self.ctx, x, np.complex64)
        out = out or self.ctx.empty(self.N + (self.n_filters,), np.float32)
        self.ctx.check(self.ctx.lib.disorder_shearlet_coefficients(self.ctx.h, self.h, xd.ptr, float(eps),
                                                                   float(p - 2), out.ptr))
        return out

    def regularize(self, x, We, la, p=1.0, out=None, beta=0.0):
        """The shearlet term of Reconstruction/regularize.m:27-46 (device)."""
        xd, _ = _dev(self.ctx, x, np.complex64)
        out = out or self.ctx.empty(self.N, np.complex64)
        self.ctx.check(self.ctx.lib.disorder_shearlet_regularize(self.ctx.h, self.h, xd.ptr, We.ptr,
                                                                 float(la * p / 2), float(beta), out.ptr))
        return out

    def trace(self, probe, We):
        """traceEstimation.m:85-102 for one real probe (device float32 V)."""
        tr = C.c_double()
        self.ctx.check(self.ctx.lib.disorder_shearlet_trace(self.ctx.h, self.h, probe.ptr, We.ptr, C.byref(tr)))
        return float(tr.value)


def _host(a):
    return a.numpy() if isinstance(a, DeviceArray) else np.asarray(a)


def _weight_grid(E, EH):
    """EH.We (per sample) on the (ky, kz) grid (traceEstimation.m:42-49)."""
    N1, N2 = E.Sf.shape[0], E.Sf.shape[1]
    W = np.zeros((N1, N2), np.float64)
    np.add.at(W, (_host(E.ky).ravel(), _host(E.kz).ravel()), _host(EH.We).astype(np.float64).ravel())
    return W.astype(np.float32)


class _DeviceProbes:
    """Probes drawn on the device (disorder_trace_probe), seeded from rng."""

    def __init__(self, rng):
        self.rng = rng if rng is not None else np.random.default_rng()


def _noise_source(noise, rng):
    """noise(shape) -> host float32 probes (given), else device probes."""
    return noise if noise is not None else _DeviceProbes(rng)


def traceEstimation(ctx, NX, E=None, EH=None, Cs=None, R=None, tol=1e-2, BlSz=1, noise=None, rng=None):
    """Reconstruction/traceEstimation.m:1-113 (no SENSE folding): Hutchinson
    estimates of the fidelity term (E.Sf with EH.We on the k-space grid) and
    the shearlet term (R.Sh), BlSz real Gaussian probes per round until the
    standard error is below tol of the mean. noise(shape) or rng draws the
    probes (the device draws them from rng's seeds when noise is None).
    Returns (tr, trF)."""
    NX = tuple(int(n) for n in NX[:3])
    V = int(np.prod(NX))
    draw = noise if noise is not None else _noise_source(None, rng)
    Ma = Mad = None
    if Cs is not None and Cs.has("Ma"):
        Ma = _host(Cs.Ma).reshape(NX, order="F").astype(np.float64)
        Mad = ctx.upload(Ma.astype(np.float32), np.float32)
    pd = ctx.empty(NX, np.float32)
    Wd = Sd = None
    nC = 0
    if E is not None:
        Sd, _ = _dev(ctx, E.Sf, np.complex64)
        nC = Sd.shape[3] if len(Sd.shape) > 3 else 1
        # without EH.We the reference sums |S .* x|^2 without a DFT, which the
        # unit-weight grid gives through the unitary DFT (Parseval)
        W = _weight_grid(E, EH) if (EH is not None and EH.has("We")) else np.ones(NX[:2], np.float32)
        Wd = ctx.upload(W, np.float32)
    Nc = (C.c_int32 * 3)(*NX)
    trF = []
    while True:
        for _ in range(BlSz):
            if isinstance(draw, _DeviceProbes):  # traceEstimation.m:54-59 on the device
                seed = int(draw.rng.integers(1, 2 ** 63))
                ctx.check(ctx.lib.disorder_trace_probe(ctx.h, V, seed, Mad.ptr if Mad is not None else None, pd.ptr))
            else:
                v = np.asarray(draw(NX), np.float64)
                v = v / np.sqrt(np.sum(v * v) / V)  # traceEstimation.m:55
                if Ma is not None:
                    v = v * Ma
                h = np.asfortranarray(v.astype(np.float32))
                ctx.check(ctx.lib.disorder_memcpy_h2d(ctx.h, pd.ptr, h.ctypes.data, h.nbytes))
            tc = 0.0
            if E is not None:
                t = C.c_double()
                ctx.check(ctx.lib.disorder_fidelity_trace(ctx.h, Nc, pd.ptr, Sd.ptr, nC, Wd.ptr, C.byref(t)))
                tc += t.value
            if R is not None and R.has("Sh"):
                tc += R.Sh.sys.trace(pd, R.Sh.We)
            trF.append(tc)
        n = len(trF)
        mea = float(np.mean(trF))
        std = float(np.std(trF, ddof=1)) / np.sqrt(n) if n > 1 else np.inf
        if n >= 2 and std / (mea + EPS) < tol:
            return mea, np.array(trF)


def CSsolver(y, E, EH, A=None, Cs=None, R=None, x=None, nIt=300, tolType="Energy", tol=1e-5, deb=0, nOu=2,
             ctx=None, noise=None, rng=None, system=None):
    """Reconstruction/CSsolver.m:1-103: the shearlet-regularised CG
    reconstruction, with lambda from trace estimates. R.Ti (R.Ti.la) is
    required when Cs carries no mask (CSsolver.m:47,72). system: a prebuilt
    ShearletSystem of x's grid (built here otherwise). Returns (x, lambda),
    x on the device."""
    ctx = ctx or default_context()
    R = R or Struct()
    y, _ = _dev(ctx, y, np.complex64)  # device samples: the CG calls below then work on device arrays
    if x is None:  # :33-38
        EH0 = EH.copy(We=np.ones(_host(EH.We).size, np.float32)) if (EH is not None and EH.has("We")) else EH
        if EH0 is not None and EH0.has("Mbe"):
            EH0 = EH0.copy(Mbe=np.ones(_host(EH0.Mbe).size, np.float32))
        x, _, _ = CGsolver(y, E, EH0, A, Cs, R, None, nIt, tolType, tol, ctx=ctx)
    if EH is not None and EH.has("Mbe"):  # :33
        EH = EH.copy(Mbe=np.ones(_host(EH.Mbe).size, np.float32))
    if isinstance(x, DeviceArray):  # the caller's array stays as it was
        xd = ctx.empty(x.shape, np.complex64)
        ctx.check(ctx.lib.disorder_memcpy_d2d(ctx.h, xd.ptr, x.ptr, x.nbytes))
    else:
        xd, _ = _dev(ctx, x, np.complex64)
    NN = tuple(xd.shape[:3])
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    if tuple(Sd.shape[:3]) != NN:
        raise DisorderError(1, "CSsolver: reconstruction grid %s differs from the encoding grid %s (resampled "
                               "reconstructions are not supported)" % (NN, tuple(Sd.shape[:3])))
    if Cs is not None and Cs.has("Ma"):  # :46
        Cs = Cs.copy(Ma=(_host(Cs.Ma) > 0.5).astype(np.float32))
    elif not R.has("Ti"):
        raise DisorderError(1, "CSsolver: R.Ti is required when C has no mask (CSsolver.m:47)")
    epsil, p = 1e-2, 1.0  # :51-53
    sys_ = system or ShearletSystem(ctx, NN, 1, [1], "kos")
    if sys_.N != NN:
        raise DisorderError(1, "CSsolver: shearlet system of %s for a %s grid" % (sys_.N, NN))
    if deb >= 1:
        print("Size shearlets: %s %d" % (" ".join(str(n) for n in NN), sys_.n_filters))
    We = sys_.coefficients(xd, epsil, p)  # :57-59
    Sh = Struct(sys=sys_, We=We, la=0.0, p=p)
    draw = _noise_source(noise, rng)
    trFid, _ = traceEstimation(ctx, NN, E, EH, Cs, None, 1e-2, 4, noise=draw)  # :63
    trReg, _ = traceEstimation(ctx, NN, None, None, Cs, Struct(Sh=Sh), 1e-2, 4, noise=draw)  # :64
    la = (2 / p) * trFid / (trReg + EPS)  # :65
    lam = np.zeros(nOu + 1)
    lam[0] = la
    # A.Se = (sum_c |S_c|^2 (+ R.Ti.la) + la p / 2)^-1  (:71-74)
    nC = Sd.shape[3] if len(Sd.shape) > 3 else 1
    w0 = ctx.empty(NN, np.float32)  # 1 / sum_c |S_c|^2 on the device
    ctx.check(ctx.lib.disorder_precondition_weights(ctx.h, Sd.ptr, nC, int(np.prod(NN)), 0.0, w0.ptr))
    with np.errstate(divide="ignore"):
        S2 = 1.0 / w0.numpy().astype(np.float64)
    w0.close()
    if Cs is None or not Cs.has("Ma"):
        S2 = S2 + _host(R.Ti).reshape(NN, order="F")
    for n in range(1, nOu + 1):  # :69-88
        Se = ctx.upload((1.0 / (S2 + la * p / 2)).astype(np.float32), np.float32)
        Rn = R.copy(Sh=Sh.copy(la=la))
        xd, _, _ = CGsolver(y, E, EH, Struct(Se=Se), Cs, Rn, xd, 3, "None", tol, ctx=ctx)
        if n != nOu:
            sys_.coefficients(xd, epsil, p, out=We)
            trReg, _ = traceEstimation(ctx, NN, None, None, Cs, Struct(Sh=Sh), 1e-2, 4, noise=draw)
            la = (2 / p) * trFid / (trReg + EPS)
            lam[n] = la
            if deb >= 1:
                print("It %d. Lambda: %.6g" % (n, la))
    return xd, lam
