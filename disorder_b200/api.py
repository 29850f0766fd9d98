"""Host-side mirror of the reference's MATLAB call surface for the hot path.

The functions keep the reference's names, argument order and structure
fields so that a call site reads like the MATLAB one:

    y  = encode(x, E)                          Reconstruction/encode.m:1
    x  = decode(y, EH, E)                      Reconstruction/decode.m:1
    x  = encodedecode(x, E, EH)                Reconstruction/encodedecode.m:1
    En = computeEnergy(y, x, E, R, EH)         Reconstruction/computeEnergy.m:1
    x, En, nn = CGsolver(y, E, EH, A, C, R, x, nIt, tolType, tol)
                                               Reconstruction/CGsolver.m:1
    E  = LMsolver(y, E, x, C)                  Reconstruction/LMsolver.m:1
    et = precomputeFactorsSincRigidTransform(grids, T, di, cg)
    x, xB = sincRigidTransform(x, et, di, sumR, useFull)
    G  = sincRigidTransformGradient(xB, et)    Methods/sincRigidTransformGradient.m:1

All computation runs in libdisorder.so on the GPU through the C ABI; there is
no CPU path. Arrays are numpy arrays (copied to the device for the call, the
result copied back) or DeviceArray objects (kept resident). Arrays use the
reference's MATLAB dimension order with column-major memory: volumes
(N1,N2,N3), coils (N1,N2,N3,C), samples (Ns,N3,C), motion (S,6).
"""

import ctypes as C
import weakref

import numpy as np

from . import _lib
from ._lib import DisorderError

# E/EH fields this implementation supports (the hot-path fields); anything
# else set on a structure is rejected with disorder:UNSUPPORTED_FIELD, like a
# MATLAB error at the gateway.
E_FIELDS = {"Tr", "NMs", "NSe", "Sf", "grids", "ky", "kz", "nEc", "mSt", "vA", "w", "cT", "winit", "tL", "nF",
            "En", "EnPrev", "Je", "bS", "dS", "oS", "Uf", "UAf", "kG", "rkG", "Fof", "Fob", "rG", "iSt", "nSt",
            "plan_cache"}
EH_FIELDS = {"We", "Mb", "Mbe", "Ub", "UAb"}
UNSUPPORTED = {"Af", "Ti", "Gf", "Xf", "Ff", "NXAcq", "ZSl", "Sp", "Bf", "Gh", "Ef", "Es", "Fms", "Bm", "Dc", "Tf",
               "Zf", "Fd", "Pf", "Ps"}


# ---------------------------------------------------------------- device plumbing
class Context:
    """One CUDA device and stream (disorder_ctx)."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.disorder_ctx_create(device, C.byref(h))
        if st:
            raise DisorderError(st, "cannot create a context on CUDA device %d" % device)
        self.h = h
        self.device = device
        # plans, device arrays and networks of this context: they are released
        # before the context itself, whatever order the garbage collector
        # finalises a cycle that holds them in
        self._children = weakref.WeakSet()

    def check(self, st):
        if st:
            raise DisorderError(st, self.lib.disorder_last_error(self.h).decode())

    def adopt(self, obj):
        """Register an object with a close() that must run before the context goes."""
        self._children.add(obj)

    def close(self):
        if getattr(self, "h", None):
            for ch in list(getattr(self, "_children", ())):
                try:
                    ch.close()
                except Exception:
                    pass
            self.lib.disorder_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        self.check(self.lib.disorder_synchronize(self.h))

    PRECISIONS = {"fp32": 0, "bf16x3": 1, "tf32x3": 2}

    TUNING = {"tma": 0, "coil_stage": 1}

    def set_tuning(self, key, value):
        """A kernel choice of this context (disorder_ctx_set_tuning): 'tma'
        (1: TMA tile copies, 0: cp.async pipelines), 'coil_stage' (0: three
        passes, 1: sample sums)."""
        self.check(self.lib.disorder_ctx_set_tuning(self.h, self.TUNING.get(key, key), int(value)))

    def set_precision(self, mode):
        """Arithmetic of the tensor-core contractions (disorder_ctx_set_precision):
        'fp32' (CUDA cores), 'bf16x3' or 'tf32x3' (tcgen05, split operands)."""
        self.check(self.lib.disorder_ctx_set_precision(self.h, self.PRECISIONS[mode] if isinstance(mode, str)
                                                       else int(mode)))
        self.precision = mode

    @property
    def launches(self):
        return int(self.lib.disorder_kernel_launches(self.h))

    @property
    def stream(self):
        return self.lib.disorder_ctx_get_stream(self.h)

    def event(self, slot):
        self.check(self.lib.disorder_event_record(self.h, slot))

    def elapsed_ms(self, a, b):
        ms = C.c_float()
        self.check(self.lib.disorder_event_elapsed(self.h, a, b, C.byref(ms)))
        return float(ms.value)

    def empty(self, shape, dtype=np.complex64):
        return DeviceArray(self, shape, dtype)

    def upload(self, a, dtype=None):
        a = np.asarray(a)
        if dtype is not None:
            a = a.astype(dtype, copy=False)
        a = np.asfortranarray(a)
        d = DeviceArray(self, a.shape, a.dtype)
        if a.nbytes:
            self.check(self.lib.disorder_memcpy_h2d(self.h, d.ptr, a.ctypes.data, a.nbytes))
        return d


class DeviceArray:
    """Device memory holding a column-major array (the resident form of a
    MATLAB array behind a MEX handle)."""

    def __init__(self, ctx, shape, dtype):
        self.ctx = ctx
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = C.c_void_p()
        ctx.check(ctx.lib.disorder_malloc(ctx.h, max(self.nbytes, 1), C.byref(p)))
        self.ptr = p.value
        ctx.adopt(self)

    def numpy(self):
        out = np.empty(self.shape, dtype=self.dtype, order="F")
        if self.nbytes:
            self.ctx.check(self.ctx.lib.disorder_memcpy_d2h(self.ctx.h, out.ctypes.data, self.ptr, self.nbytes))
        return out

    def free(self):
        if self.ptr is not None and self.ctx.h is not None:
            self.ctx.lib.disorder_free(self.ctx.h, self.ptr)
        self.ptr = None

    def close(self):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def view(self, offset_elems, shape):
        """A non-owning view starting offset_elems elements in."""
        v = DeviceArray.__new__(DeviceArray)
        v.ctx, v.dtype, v.shape = self.ctx, self.dtype, tuple(shape)
        v.nbytes = int(np.prod(v.shape)) * v.dtype.itemsize
        v.ptr = self.ptr + offset_elems * self.dtype.itemsize
        v._owner = self
        v.free = lambda: None
        return v


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _dev(ctx, a, dtype):
    """(DeviceArray, was_host) for a numpy or device argument (None -> (None, False))."""
    if a is None:
        return None, False
    if isinstance(a, DeviceArray):
        if a.dtype != np.dtype(dtype):
            raise DisorderError(1, "expected %s device data, got %s" % (np.dtype(dtype), a.dtype))
        return a, False
    return ctx.upload(np.asarray(a), dtype), True


def _fptr(a):
    if a is None:
        return None
    a = np.ascontiguousarray(np.asfortranarray(a, dtype=np.float32).ravel(order="F"))
    return a, a.ctypes.data_as(_lib.FP)


# ---------------------------------------------------------------- grids
class Grids:
    """generateTransformGrids output (Methods/generateTransformGrids.m:23-67):
    rGrid[m], kGrid[m] float32 vectors (kGrid ifftshifted, sh=1), cGrid."""

    def __init__(self, rGrid, kGrid, cGrid):
        self.rGrid = [np.asarray(r, np.float32) for r in rGrid]
        self.kGrid = [np.asarray(k, np.float32) for k in kGrid]
        self.cGrid = [float(c) for c in cGrid]

    @property
    def N(self):
        return tuple(len(k) for k in self.kGrid)


def generateTransformGrids(N, Nres=None, cent=None, sh=1):
    """Methods/generateTransformGrids.m:23-67 (via generateGrid.m:27-40): rGrid
    in full-resolution voxels, kGrid in radians per full-resolution voxel,
    both rounded to single precision as in the reference."""
    N = [int(n) for n in (list(N) + [1, 1])[:3]]
    Nres = N if Nres is None else [int(n) for n in Nres]
    cent = [n / 2.0 + 1 for n in Nres] if cent is None else list(cent)
    r, k = [], []
    for m in range(3):
        idx = np.arange(1, Nres[m] + 1, dtype=np.float64)
        r.append(((N[m] / Nres[m]) * (idx - cent[m])).astype(np.float32))
        kk = ((2 * np.pi * Nres[m] / N[m]) / Nres[m] * (idx - np.ceil((Nres[m] + 1) / 2.0))).astype(np.float32)
        k.append(np.fft.ifftshift(kk) if sh else kk)
    return Grids(r, k, cent)


# ---------------------------------------------------------------- plans / structures
class Plan:
    """A disorder_plan: grids plus the segment sample lists of an E structure."""

    def __init__(self, ctx, grids, ky, kz, nEc, n_mot):
        self.ctx = ctx
        self.grids = grids
        self.N = grids.N
        self._keep = []
        gd = _lib.GridDesc()
        for m in range(3):
            gd.N[m] = self.N[m]
            r = np.ascontiguousarray(grids.rGrid[m], np.float32)
            k = np.ascontiguousarray(grids.kGrid[m], np.float32)
            self._keep += [r, k]
            gd.rG[m] = r.ctypes.data_as(_lib.FP)
            gd.kG[m] = k.ctypes.data_as(_lib.FP)
            gd.cent[m] = grids.cGrid[m]
        off = np.ascontiguousarray(nEc, np.int64)
        ky = np.ascontiguousarray(ky, np.int32)
        kz = np.ascontiguousarray(kz, np.int32)
        self._keep += [off, ky, kz]
        sd = _lib.SamplingDesc()
        sd.n_seg = len(off) - 1
        sd.n_mot = int(n_mot)
        sd.seg_offsets = off.ctypes.data_as(C.POINTER(C.c_int64))
        sd.ky = ky.ctypes.data_as(C.POINTER(C.c_int32))
        sd.kz = kz.ctypes.data_as(C.POINTER(C.c_int32))
        h = C.c_void_p()
        ctx.check(ctx.lib.disorder_plan_create(ctx.h, C.byref(gd), C.byref(sd), C.byref(h)))
        self.h = h
        self.n_seg = sd.n_seg
        self.n_mot = sd.n_mot
        self.n_samples = int(off[-1])
        self.nEc = off.copy()
        ctx.adopt(self)

    def close(self):
        # a plan goes before its context (disorder_plan_destroy uses the
        # context's stream); once the context is gone there is nothing to free
        if getattr(self, "h", None) is not None and self.ctx.h is not None:
            self.ctx.lib.disorder_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Struct:
    """A MATLAB-struct-like bag of fields (E, EH, A, C, R)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def has(self, name):
        return getattr(self, name, None) is not None

    def copy(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return Struct(**d)


def _check_fields(S, allowed, what):
    if S is None:
        return
    for k, v in S.__dict__.items():
        if v is None:
            continue
        if k in UNSUPPORTED or k not in allowed:
            raise DisorderError(2, "%s.%s is not supported by the B200 hot path" % (what, k))


def _plan(E, ctx):
    _check_fields(E, E_FIELDS, "E")
    key = (id(ctx), id(E.ky), id(E.kz), id(E.nEc), int(E.NMs), tuple(E.grids.N))
    pc = getattr(E, "plan_cache", None)
    if pc is not None and pc[0] == key:
        return pc[1]
    p = Plan(ctx, E.grids, E.ky, E.kz, E.nEc, E.NMs)
    E.plan_cache = (key, p)
    return p


def _T(E):
    if not E.has("Tr"):
        return None
    T = np.asarray(E.Tr, np.float32)
    if not np.any(T != 0):
        return None  # the reference's any(E.Tr(:)~=0) branch (encode.m:61)
    return _fptr(T)


def _out(d, host):
    return d.numpy() if host else d


# ---------------------------------------------------------------- operators
def encode(x, E, ctx=None):
    """Reconstruction/encode.m:1-147 (hot fields): samples (Ns, N3, C)."""
    ctx = ctx or default_context()
    p = _plan(E, ctx)
    xd, host = _dev(ctx, x, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    y = ctx.empty((p.n_samples, p.N[2], Cn))
    T = _T(E)
    ctx.check(ctx.lib.disorder_encode(ctx.h, p.h, xd.ptr, Sd.ptr, Cn, T[1] if T else None, y.ptr))
    return _out(y, host)


def decode(y, EH, E, ctx=None):
    """Reconstruction/decode.m:1-160 (hot fields): volume (N1, N2, N3)."""
    ctx = ctx or default_context()
    _check_fields(EH, EH_FIELDS, "EH")
    p = _plan(E, ctx)
    yd, host = _dev(ctx, y, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    We, _ = _dev(ctx, EH.We if (EH is not None and EH.has("We") and len(EH.We)) else None, np.float32)
    Mb, _ = _dev(ctx, EH.Mb if (EH is not None and EH.has("Mb")) else None, np.float32)
    x = ctx.empty(p.N)
    T = _T(E)
    ctx.check(ctx.lib.disorder_decode(ctx.h, p.h, yd.ptr, Sd.ptr, Cn, T[1] if T else None,
                                      We.ptr if We else None, Mb.ptr if Mb else None, x.ptr))
    return _out(x, host)


def encodedecode(x, E, EH=None, ctx=None):
    """Reconstruction/encodedecode.m:1-250 (hot fields): E^H W E x."""
    ctx = ctx or default_context()
    _check_fields(EH, EH_FIELDS, "EH")
    p = _plan(E, ctx)
    xd, host = _dev(ctx, x, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    We, _ = _dev(ctx, EH.We if (EH is not None and EH.has("We") and len(EH.We)) else None, np.float32)
    out = ctx.empty(p.N)
    T = _T(E)
    ctx.check(ctx.lib.disorder_encodedecode(ctx.h, p.h, xd.ptr, Sd.ptr, Cn, T[1] if T else None,
                                            We.ptr if We else None, out.ptr))
    return _out(out, host)


def computeEnergy(y, x, E, R=None, EH=None, ctx=None):
    """Reconstruction/computeEnergy.m:34-80 (no=2): [fidelity, regularisation]."""
    ctx = ctx or default_context()
    _check_fields(EH, EH_FIELDS, "EH")
    p = _plan(E, ctx)
    yd, _ = _dev(ctx, y, np.complex64)
    xd, _ = _dev(ctx, x, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    Mb, _ = _dev(ctx, EH.Mb if (EH is not None and EH.has("Mb")) else None, np.float32)
    Mbe, _ = _dev(ctx, EH.Mbe if (EH is not None and EH.has("Mbe")) else None, np.float32)
    Ti, _ = _dev(ctx, R.Ti if (R is not None and R.has("Ti")) else None, np.float32)
    En = (C.c_double * 2)()
    T = _T(E)
    ctx.check(ctx.lib.disorder_compute_energy(ctx.h, p.h, yd.ptr, xd.ptr, Sd.ptr, Cn, T[1] if T else None,
                                              Mb.ptr if Mb else None, Mbe.ptr if Mbe else None,
                                              Ti.ptr if Ti else None, En))
    return np.array([En[0], En[1]])


def sampleEnergies(y, x, E, EH=None, ctx=None):
    """Reconstruction/computeEnergy.m:34-80 with avdi=1 (solveXT.m:443): per
    sample, the sum over readout rows (weighted by EH.Mb and EH.Mbe) and
    coils of |encode(x) - y|^2. Returns (n_samples,) float64."""
    ctx = ctx or default_context()
    p = _plan(E, ctx)
    yd, _ = _dev(ctx, y, np.complex64)
    xd, _ = _dev(ctx, x, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    ws = [getattr(EH, f) for f in ("Mb", "Mbe") if EH is not None and EH.has(f)]
    if len(ws) == 2:  # sqrt(Mb) and sqrt(Mbe) both weight the residual (computeEnergy.m:36-37)
        ws = [np.prod([w.numpy() if isinstance(w, DeviceArray) else np.asarray(w) for w in ws], axis=0)]
    Mbe, _ = _dev(ctx, ws[0] if ws else None, np.float32)
    En = np.zeros(max(p.n_samples, 1))
    T = _T(E)
    ctx.check(ctx.lib.disorder_sample_energies(ctx.h, p.h, yd.ptr, Sd.ptr, Cn, xd.ptr, T[1] if T else None,
                                               Mbe.ptr if Mbe else None, En.ctypes.data_as(_lib.DP)))
    return En[:p.n_samples]


def residualSampleEnergies(r, E, EH=None, ctx=None):
    """sampleEnergies for a residual r = encode(x) - y already on the device
    (for example CGsolver's residual output). Returns (n_samples,) float64."""
    ctx = ctx or default_context()
    p = _plan(E, ctx)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    ws = [getattr(EH, f) for f in ("Mb", "Mbe") if EH is not None and EH.has(f)]
    if len(ws) == 2:
        ws = [np.prod([w.numpy() if isinstance(w, DeviceArray) else np.asarray(w) for w in ws], axis=0)]
    Mbe, _ = _dev(ctx, ws[0] if ws else None, np.float32)
    En = np.zeros(max(p.n_samples, 1))
    ctx.check(ctx.lib.disorder_residual_energies(ctx.h, p.h, r.ptr, Cn, Mbe.ptr if Mbe else None,
                                                 En.ctypes.data_as(_lib.DP)))
    return En[:p.n_samples]


TOLTYPES = {"RelativeResidual2Error": 1, "Energy": 6, "None": 7}


def CGsolver(y, E, EH, A=None, Cs=None, R=None, x=None, nIt=300, tolType="Energy", tol=1e-5, ctx=None,
             residual=None):
    """Reconstruction/CGsolver.m:1-119 with E.Je=1. Returns (x, En, nn).
    residual: optional device array (Ns, N3, C) that receives the final
    sample residual encode(x) - y (disorder_cg_solve_residual)."""
    ctx = ctx or default_context()
    _check_fields(EH, EH_FIELDS, "EH")
    if tolType not in TOLTYPES:
        raise DisorderError(1, "The %s stopping criterion is not implemented for CG solver" % tolType)
    p = _plan(E, ctx)
    yd, host = _dev(ctx, y, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    g = lambda S, f: getattr(S, f) if (S is not None and S.has(f)) else None  # noqa: E731
    We, _ = _dev(ctx, g(EH, "We") if g(EH, "We") is not None and len(EH.We) else None, np.float32)
    Mb, _ = _dev(ctx, g(EH, "Mb"), np.float32)
    Mbe, _ = _dev(ctx, g(EH, "Mbe"), np.float32)
    Se, _ = _dev(ctx, g(A, "Se"), np.float32)
    Ma, _ = _dev(ctx, g(Cs, "Ma"), np.float32)
    Ti, _ = _dev(ctx, g(R, "Ti"), np.float32)
    if x is None:
        xd, x_init = ctx.empty(p.N), 0
    elif isinstance(x, DeviceArray):
        xd, x_init = x, 1
    else:
        xd, x_init = ctx.upload(x, np.complex64), 1
    ncol = (nIt + 1) // 2 + 1
    En = (C.c_double * (2 * ncol))()
    n_en, nn = C.c_int32(), C.c_int32()
    T = _T(E)
    ptr = lambda d: d.ptr if d is not None else None  # noqa: E731
    args = (ctx.h, p.h, yd.ptr, Sd.ptr, Cn, T[1] if T else None, ptr(We), ptr(Mb), ptr(Mbe), ptr(Se), ptr(Ma),
            ptr(Ti), xd.ptr, x_init, int(nIt), TOLTYPES[tolType], float(tol), En, C.byref(n_en), C.byref(nn))
    if R is not None and R.has("Sh"):
        # the shearlet term (Reconstruction/regularize.m:27-46): R.Sh holds the
        # system (disorder_b200.cs.ShearletSystem), We, la and p
        if residual is not None:
            raise DisorderError(1, "CG with R.Sh does not return the sample residual")
        sh = R.Sh
        ctx.check(ctx.lib.disorder_cg_solve_shearlet(*args[:12], sh.sys.h, sh.We.ptr, float(sh.la * sh.p / 2),
                                                     *args[12:]))
    elif residual is not None:
        ctx.check(ctx.lib.disorder_cg_solve_residual(*args, residual.ptr))
    else:
        ctx.check(ctx.lib.disorder_cg_solve(*args))
    Enm = np.array(En[:2 * n_en.value]).reshape(2, -1, order="F") if n_en.value else np.zeros((2, 0))
    return (_out(xd, host), Enm, nn.value)


def LMsolver(y, E, x, Cs=None, ctx=None):
    """Reconstruction/LMsolver.m:1-226 (E.Fs branch): one Levenberg-Marquardt
    step of the per-state motion. Returns an updated copy of E (Tr, cT, w, En)."""
    ctx = ctx or default_context()
    if Cs is not None and any(v is not None for v in Cs.__dict__.values()):
        raise DisorderError(2, "C (motion constraints) is not supported by the B200 hot path")
    p = _plan(E, ctx)
    yd, _ = _dev(ctx, y, np.complex64)
    xd, _ = _dev(ctx, x, np.complex64)
    Sd, _ = _dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    S = p.n_mot
    T = np.asfortranarray(np.asarray(E.Tr, np.float32).copy())
    w = np.ascontiguousarray(np.asarray(E.w, np.float32).copy())
    cT = np.ascontiguousarray(np.asarray(E.cT, bool).astype(np.uint8))
    tL = np.ascontiguousarray(np.asarray(E.tL, np.float32))
    lo, hi = 0, 0
    if E.has("nF"):
        nF = np.asarray(E.nF)
        lo, hi = int(nF[0]), int(nF[-1]) + 1
        if not np.array_equal(nF, np.arange(lo, hi)):
            raise DisorderError(1, "E.nF must be a contiguous readout range")
    En = (C.c_double * S)()
    EnPrev = (C.c_double * S)()
    Tf = np.asfortranarray(T)
    ctx.check(ctx.lib.disorder_lm_step(ctx.h, p.h, yd.ptr, Sd.ptr, Cn, xd.ptr, Tf.ctypes.data_as(_lib.FP),
                                       w.ctypes.data_as(_lib.FP), cT.ctypes.data_as(C.POINTER(C.c_uint8)),
                                       float(E.winit), tL.ctypes.data_as(_lib.FP), lo, hi, En, EnPrev))
    En = np.array(En[:])
    EnPrev = np.array(EnPrev[:])
    Enmin = np.minimum(EnPrev, En)
    est = ~np.asarray(E.cT, bool)
    if E.has("En"):
        Eo = np.asarray(E.En, float).copy()
        Eo[est] = Enmin[est]
    else:
        Eo = Enmin
    return E.copy(Tr=np.array(Tf), w=w, cT=cT.astype(bool), En=Eo, EnPrev=EnPrev)


# ---------------------------------------------------------------- transform
class Factors:
    """precomputeFactorsSincRigidTransform output: the transform factors are
    formed on the device inside each transform call from (grids, T, di)."""

    def __init__(self, grids, T, di, cg):
        self.grids, self.T, self.di, self.cg = grids, np.asarray(T, np.float32), di, cg

    def arrays(self, ctx=None):
        """The factors as the reference holds them (disorder_precompute_factors):
        {'e1': [N[m] x S], 'e2': [N[a] x N[b] x S], 'e3': [...], 'flip': (3, S)}
        with (a, b) = (0, 1), (0, 2), (1, 2) for m = 0, 1, 2."""
        ctx = ctx or default_context()
        p = _transform_plan(ctx, self.grids)
        N = tuple(int(n) for n in p.N)
        S = int(self.T.shape[0])
        pairs = [(0, 1), (0, 2), (1, 2)]
        n2 = sum(N[a] * N[b] for a, b in pairs) * S
        e1 = ctx.empty((sum(N) * S,))
        e2 = ctx.empty((n2,))
        e3 = ctx.empty((n2,))
        flip = np.zeros(3 * S, np.uint8)
        Tf = np.asfortranarray(self.T)
        ctx.check(ctx.lib.disorder_precompute_factors(ctx.h, p.h, Tf.ctypes.data_as(_lib.FP), S, int(self.di), e1.ptr,
                                                      e2.ptr, e3.ptr, flip.ctypes.data_as(C.POINTER(C.c_uint8))))
        h1, h2, h3 = e1.numpy(), e2.numpy(), e3.numpy()
        out = {"e1": [], "e2": [], "e3": [], "flip": flip.reshape(3, S).astype(bool)}
        o = 0
        for m in range(3):
            out["e1"].append(h1[o:o + N[m] * S].reshape((N[m], S), order="F"))
            o += N[m] * S
        o = 0
        for a, b in pairs:
            n = N[a] * N[b] * S
            out["e2"].append(h2[o:o + n].reshape((N[a], N[b], S), order="F"))
            out["e3"].append(h3[o:o + n].reshape((N[a], N[b], S), order="F"))
            o += n
        return out


def precomputeFactorsSincRigidTransform(grids, T, di=1, cg=0):
    """Methods/precomputeFactorsSincRigidTransform.m:1 with gr=1, sh=1.
    Returns (et, etg) like the reference (etg is the same handle when cg)."""
    et = Factors(grids, T, di, cg)
    return et, (et if cg else None)


def _transform_plan(ctx, grids):
    S1 = np.zeros(1, np.int64)
    return Plan(ctx, grids, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int64), 0)


class Intermediates:
    """xB of sincRigidTransform: what the gradient needs (the input volume)."""

    def __init__(self, x):
        self.x = x


def sincRigidTransform(x, et, di=None, sumR=1, useFull=1, ctx=None):
    """Methods/sincRigidTransform.m:1-116. x: (N1,N2,N3) or (N1,N2,N3,S).
    Returns (x, xB)."""
    ctx = ctx or default_context()
    di = et.di if di is None else di
    p = _transform_plan(ctx, et.grids)
    S = et.T.shape[0]
    xd, host = _dev(ctx, x, np.complex64)
    xs = xd.shape[3] if len(xd.shape) > 3 else 1
    out_shape = p.N + (S,) if (di == 1 or not sumR) else p.N
    out = ctx.empty(out_shape)
    T = _fptr(et.T)
    ctx.check(ctx.lib.disorder_sinc_rigid_transform(ctx.h, p.h, xd.ptr, xs, T[1], S, int(di), int(sumR),
                                                    int(useFull), out.ptr))
    return _out(out, host), Intermediates(x)


def sincRigidTransformGradient(xB, et, etg=None, ctx=None):
    """Methods/sincRigidTransformGradient.m:1-150: derivatives (N1,N2,N3,S,6)."""
    ctx = ctx or default_context()
    p = _transform_plan(ctx, et.grids)
    S = et.T.shape[0]
    xd, host = _dev(ctx, xB.x, np.complex64)
    G = ctx.empty(p.N + (S, 6))
    T = _fptr(et.T)
    ctx.check(ctx.lib.disorder_sinc_rigid_transform_gradient(ctx.h, p.h, xd.ptr, T[1], S, G.ptr, None))
    return _out(G, host)


# ---------------------------------------------------------------- data preparation
def resampling(x, Nres, n_vols=None, ctx=None):
    """Methods/resampling.m:45-94 for image-space complex data (fo=0): Fourier
    crop/zero-pad of each volume to Nres. x: (N1,N2,N3) or (N1,N2,N3,K)."""
    ctx = ctx or default_context()
    xd, host = _dev(ctx, x, np.complex64)
    shp = tuple(xd.shape[:3]) + (1,) * (3 - len(xd.shape[:3]))
    K = int(np.prod(xd.shape[3:])) if len(xd.shape) > 3 else 1
    Nres = tuple(int(n) for n in Nres)
    out = ctx.empty(Nres + tuple(xd.shape[3:]))
    nin = (C.c_int32 * 3)(*shp)
    nout = (C.c_int32 * 3)(*Nres)
    ctx.check(ctx.lib.disorder_resample(ctx.h, xd.ptr, nin, K, nout, out.ptr))
    return _out(out, host)


def compressCoils(S, perc, y=None, C_max=0, ctx=None):
    """Methods/compressCoils.m:76-118: returns (S, y, C, D, U)."""
    ctx = ctx or default_context()
    Sd, host = _dev(ctx, S, np.complex64)
    Cin = Sd.shape[-1]
    V = int(np.prod(Sd.shape[:-1]))
    yd, _ = _dev(ctx, y, np.complex64)
    So = ctx.empty(Sd.shape)
    yo = ctx.empty(yd.shape) if yd is not None else None
    Cout = C.c_int32()
    D = (C.c_double * Cin)()
    U = (C.c_double * (2 * Cin * Cin))()
    ny = int(np.prod(yd.shape[:-1])) if yd is not None else 0
    ctx.check(ctx.lib.disorder_compress_coils(ctx.h, Sd.ptr, Cin, V, yd.ptr if yd else None, ny, float(perc),
                                              int(C_max), So.ptr, yo.ptr if yo else None, C.byref(Cout), D, U))
    c = Cout.value
    Sv = So.view(0, tuple(Sd.shape[:-1]) + (c,))
    yv = yo.view(0, tuple(yd.shape[:-1]) + (c,)) if yo is not None else None
    Um = np.array(U[:]).reshape(-1, 2)
    Um = (Um[:, 0] + 1j * Um[:, 1]).reshape(Cin, Cin, order="F")
    if host:
        Sv = Sv.numpy()
        yv = yv.numpy() if yv is not None else None
    return Sv, yv, c, np.array(D[:]), Um


def precondition_weights(Sf, reg=1e-9, ctx=None):
    """A.Se = 1 ./ (sum_c |S_c|^2 + reg) (Reconstruction/solveXT.m:231-233)."""
    ctx = ctx or default_context()
    Sd, host = _dev(ctx, Sf, np.complex64)
    V = int(np.prod(Sd.shape[:3]))
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    out = ctx.empty(Sd.shape[:3], np.float32)
    ctx.check(ctx.lib.disorder_precondition_weights(ctx.h, Sd.ptr, Cn, V, float(reg), out.ptr))
    return _out(out, host)


def gather_samples(y, idx, scale, ctx=None):
    """Rows idx of a (Ns, N3, C) sample array times scale (a pyramid-level crop)."""
    ctx = ctx or default_context()
    yd, host = _dev(ctx, y, np.complex64)
    idx_d = ctx.upload(np.asarray(idx, np.int32))
    rows = int(np.prod(yd.shape[1:]))
    out = ctx.empty((len(idx),) + tuple(yd.shape[1:]))
    ctx.check(ctx.lib.disorder_gather_samples(ctx.h, yd.ptr, yd.shape[0], rows, idx_d.ptr, len(idx), float(scale),
                                              out.ptr))
    return _out(out, host)
