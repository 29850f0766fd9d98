"""CGsolver and LMsolver (oracle).

TEST INFRASTRUCTURE ONLY. Restates Reconstruction/CGsolver.m:26-109,
Reconstruction/stopCondition.m:10-21, Reconstruction/precondition.m:19-23
(A.Se), Reconstruction/constrain.m:12 (C.Ma), Reconstruction/regularize.m:24,27-46
(Tikhonov R.Ti and the shearlet term R.Sh), Reconstruction/CSsolver.m:1-103 and Reconstruction/LMsolver.m:15-226 (the E.Fs branch, motion
states along dim 5, one block of states).
"""

import itertools

import numpy as np

from . import encoding as enc
from .shearlet import buildShearlet, compute_shearlet, regularize_sh, trace_estimation
from .transform import (precomputeFactorsSincRigidTransform, restrictTransform,
                        sincRigidTransform, sincRigidTransformGradient)

EPS = np.finfo(np.float64).eps


def stopCondition(tolType):
    """Reconstruction/stopCondition.m:10-21 (CG solver)."""
    table = {"NormwiseBackward2Error": 0, "RelativeResidual2Error": 1, "DataUpdate2Error": 2,
             "RelativeResidualIError": 3, "DataUpdateIError": 4, "Convergent2Variables": 5,
             "Energy": 6, "None": 7}
    t = table.get(tolType, -1)
    if t in (-1, 5):
        raise ValueError("The %s stopping criterion is not implemented for CG solver" % tolType)
    return t


def precondition(x, A):
    """Reconstruction/precondition.m:19-23 (A.Se only)."""
    if A is None or not A.has("Se"):
        return x
    return x * A.Se


def constrain(x, C):
    """Reconstruction/constrain.m:12 (C.Ma only)."""
    if C is None or not C.has("Ma"):
        return x
    return x * C.Ma


def regularize(x, R):
    """Reconstruction/regularize.m:24 (Tikhonov, R.Ti = R.Ti.la) and :27-46
    (shearlet, R.Sh with fields S, We, la, p)."""
    out = np.zeros_like(x)
    if R is not None and R.has("Ti"):
        out = out + R.Ti * x
    if R is not None and R.has("Sh"):
        sh = R.Sh
        x3 = x.reshape(x.shape[:3])
        out = out + regularize_sh(x3, sh.S, sh.We, sh.la, sh.p).astype(out.dtype).reshape(out.shape)
    return out


def CGsolver(y, E, EH, A=None, C=None, R=None, x=None, nIt=300, tolType="Energy", tol=1e-5,
             method="fft", dtype=np.float64):
    """Reconstruction/CGsolver.m:26-109 with E.Je=1 (encodedecode). Returns
    (x, En, nn) with En the 2 x k energies sampled every NitTest=2 iterations
    (empty unless tolType is 'Energy')."""
    NitTest = 2
    tolTyp = stopCondition(tolType)
    b = constrain(enc.decode(y, EH, E, method, dtype), C)  # :46
    if x is None:  # :53
        x = np.zeros_like(b)
        EHE = np.zeros_like(b)
    else:  # :55
        x = np.asarray(x, dtype=b.dtype)
        EHE = constrain(enc.encodedecode(x, E, EH, method, dtype) + regularize(x, R), C)
    bnorm2 = None
    if tolTyp not in (6, 7):  # :58-62
        zb = precondition(b, A)
        zb = np.conj(zb) * b
        bnorm2 = np.sum(np.abs(zb))
    r = b - EHE  # :64
    z = precondition(r, A)
    p = z
    zr = np.conj(z) * r
    rsold = np.sum(zr)
    En = np.zeros((2, 0))
    if abs(rsold) < 1e-6:  # :70-75
        return x, En, 0
    err = np.inf
    if tolTyp == 6:
        En = np.full((2, nIt), np.inf)
    n = 0
    for n in range(1, nIt + 1):  # :79-104
        EHE = constrain(enc.encodedecode(p, E, EH, method, dtype) + regularize(p, R), C)
        g = rsold / np.sum(np.conj(p) * EHE)
        x = x + g * p
        if n % NitTest == 1 and tolTyp == 6:
            En[:, n - 1] = enc.computeEnergy(y, x, E, R, EH, method, dtype=dtype)
        r = r - g * EHE
        z = precondition(r, A)
        zr = np.conj(z) * r
        rs = np.sum(zr)
        d = rs / (rsold + EPS)
        p = z + d * p
        rsold = rs
        if tolTyp == 1:
            err = np.sqrt(np.sum(np.abs(zr)) / bnorm2)
        elif tolTyp == 6 and n % NitTest == 1 and n > 1:
            err = np.sum(En[:, n - 1 - NitTest] - En[:, n - 1]) / np.sum(En[:, n - 1 - NitTest])
        if err < tol or abs(rs) < 1e-6:
            break
    nn = n
    if tolTyp == 6:  # :108-109
        En = En[:, :n]
    En = En[:, ::NitTest]
    return x, En, nn



def CSsolver(y, E, EH, A=None, C=None, R=None, x=None, nIt=300, tolType="Energy", tol=1e-5, nOu=2, noise=None,
             method="fft", dtype=np.float64):
    """Reconstruction/CSsolver.m:21-89 (same grid in and out, so the
    resampling steps :41-48,74 are identities). R.Ti is R.Ti.la and must be
    given when C is empty (:47,72). noise(shape) draws the trace-estimation
    probes. Returns (x, lambda)."""
    from .encoding import Struct
    if x is None:  # :33-38
        EH0 = EH.copy(We=np.ones_like(np.asarray(EH.We, np.float64))) if EH.has("We") else EH
        if EH0.has("Mbe"):
            EH0 = EH0.copy(Mbe=np.ones_like(np.asarray(EH0.Mbe, np.float64)))
        x, _, _ = CGsolver(y, E, EH0, A, C, R, None, nIt, tolType, tol, method, dtype)
    if EH.has("Mbe"):
        EH = EH.copy(Mbe=np.ones_like(np.asarray(EH.Mbe, np.float64)))
    x = np.asarray(x)
    NN = x.shape[:3]
    if C is not None and C.has("Ma"):
        C = C.copy(Ma=(np.asarray(C.Ma) > 0.5).astype(np.float64))  # :46
    epsil, p = 1e-2, 1.0  # :51-53
    S = buildShearlet(list(NN), 1, [1], "kos")["S"]  # :54
    We = (compute_shearlet(x.reshape(NN), S) + epsil) ** (p - 2)  # :58-59
    Sh = Struct(S=S, We=We, la=0.0, p=p)
    Rr = (R or Struct()).copy(Sh=Sh)
    trFid, _ = trace_estimation(x, E, EH, C, None, 1e-2, 4, noise)  # :63
    trReg, _ = trace_estimation(x, None, None, C, Rr, 1e-2, 4, noise)  # :64
    la = (2 / p) * trFid / (trReg + EPS)  # :65
    lam = [la]
    for n in range(1, nOu + 1):  # :69-88
        Se = np.sum(np.abs(np.asarray(E.Sf, np.complex128)) ** 2, axis=3)
        if C is None or not C.has("Ma"):
            Se = Se + R.Ti.reshape(Se.shape)
        Se = (Se + la * p / 2) ** -1
        Rr = Rr.copy(Sh=Sh.copy(la=la))
        x, _, _ = CGsolver(y, E, EH, Struct(Se=Se.reshape(x.shape)), C, Rr, x, 3, "None", tol, method, dtype)
        if n != nOu:
            Sh = Sh.copy(We=(compute_shearlet(x.reshape(NN), S) + epsil) ** (p - 2))
            Rr = Rr.copy(Sh=Sh)
            trReg, _ = trace_estimation(x, None, None, C, Rr, 1e-2, 4, noise)
            la = (2 / p) * trFid / (trReg + EPS)
            lam.append(la)
            Sh = Sh.copy(la=la)
    return x, np.array(lam + [0.0] * (nOu + 1 - len(lam)))

# Hessian index pairs ha (LMsolver.m:26): 6 diagonal entries then nchoosek(1:6,2)
HA = [(i, i) for i in range(6)] + list(itertools.combinations(range(6), 2))


def _state_samples(E, vA):
    return np.concatenate([np.arange(int(E.nEc[s]), int(E.nEc[s + 1])) for s in vA]) if len(vA) else np.zeros(0, int)


def _encode_sub(xT, E, vA, method):
    Es = E.copy(Tr=None, vA=list(vA))
    return enc.encode(xT, Es, method)


def LMsolver(y, E, x, C=None, method="fft", dtype=np.float64, deb=0):
    """Reconstruction/LMsolver.m:15-226 (E.Fs branch). Returns an updated copy
    of E with Tr, cT, w and En set as the reference sets them (:217-225).

    Fields used: E.Tr (S x 6), E.cT (S,), E.w (S,), E.winit, E.tL (2,),
    E.nF (readout indices, optional), E.Sf, E.ky/E.kz/E.nEc, E.mSt, E.grids.
    """
    E = E.copy()
    T = np.asarray(E.Tr, dtype=np.float32).copy()
    S = T.shape[0]
    ndG, ndH = 6, len(HA)
    flagw = np.zeros(S, bool)
    multA, multB = 1.2, 2.0
    NElY = y.size  # numel(y) before the readout crop (:32)
    if E.has("nF"):  # :33
        nF = np.asarray(E.nF)
        E = E.copy(Sf=E.Sf[:, :, nF])
        y = y[:, nF]
    else:
        nF = None
    cTFull = np.asarray(E.cT, bool).copy()
    w = np.asarray(E.w, np.float64).copy()
    dH = np.zeros((S, ndH))
    dG = np.zeros((S, ndG))
    dGEff = np.zeros((S, ndG))
    EnPrev = np.zeros(S)
    ind2EstOr = np.flatnonzero(~cTFull)  # :49
    vA = list(ind2EstOr)

    def crop(v):
        return v[:, :, nF] if nF is not None else v

    if vA:
        indY = _state_samples(E, vA)
        Tf, Tg = precomputeFactorsSincRigidTransform(E.grids, T[vA], 1, 1, dtype)  # :60
        xT, xB = sincRigidTransform(x, Tf, 1, keep_intermediates=True)  # :66
        r = _encode_sub(crop(xT), E, vA, method) - y[indY]  # :72
        ry = np.sum(np.abs(r) ** 2, axis=(1, 2)) / NElY  # :82
        mst = np.asarray(E.mSt)[indY]
        EnPrev[vA] = np.bincount(mst, ry, minlength=S)[vA]  # :83,93
        G = sincRigidTransformGradient(xB, Tf, Tg)  # :96
        Genc = [_encode_sub(crop(g), E, vA, method) for g in G]  # :97-99
        for gi in range(ndG):  # :106
            v = np.sum(np.real(Genc[gi] * np.conj(r)), axis=(1, 2))
            dG[vA, gi] = np.bincount(mst, v, minlength=S)[vA]
        for h, (a_, b_) in enumerate(HA):  # :115
            v = np.sum(np.real(Genc[a_] * np.conj(Genc[b_])), axis=(1, 2))
            dH[vA, h] = np.bincount(mst, v, minlength=S)[vA]

    En = EnPrev.copy()
    MH = np.eye(ndG)
    fina = False
    Tupr = np.zeros_like(T)
    Tup = T
    while not fina:  # :129-215
        for a in np.flatnonzero(~cTFull & (w < 1e10)):
            for h, (p_, q_) in enumerate(HA):
                if p_ == q_:
                    MH[p_, q_] = (1 + w[a]) * dH[a, h]
                else:
                    MH[p_, q_] = dH[a, h]
                    MH[q_, p_] = dH[a, h]
            GJ = np.linalg.solve(MH, dG[a])
            dGEff[a] = -(E.winit / w[a]) * GJ
        Tupr = dGEff.astype(np.float32)
        Tup = restrictTransform(T + Tupr)  # :143
        ecT = cTFull | flagw  # :146
        vE = list(np.flatnonzero(~ecT))
        if vE:
            indY = _state_samples(E, vE)
            Tf, _ = precomputeFactorsSincRigidTransform(E.grids, Tup[vE], 1, 0, dtype)
            xT = sincRigidTransform(x, Tf, 1)
            r = _encode_sub(crop(xT), E, vE, method) - y[indY]
            ry = np.sum(np.abs(r) ** 2, axis=(1, 2)) / NElY
            mst = np.asarray(E.mSt)[indY]
            En[vE] = np.bincount(mst, ry, minlength=S)[vE]
        En[w > 1e10] = EnPrev[w > 1e10]  # :195
        flagw[En <= EnPrev] = True  # :196
        if deb >= 2:
            print("Energy before: %0.6g / Energy after: %0.6g" % (EnPrev.sum(), En.sum()))
        if np.any(~flagw):  # :199-200
            sel = (En > EnPrev) & ~cTFull
            w[sel] = w[sel] * multB
        else:  # :201-213
            w[~cTFull] = w[~cTFull] / multA
            w[w < 1e-8] = multA * w[w < 1e-8]
            T = Tup
            fina = True
            traDiff = np.abs(Tupr[:, 0:3])
            rotDiff = np.abs(Tupr[:, 3:6] * 180 / np.pi)
            cTFull[(traDiff.max(axis=1) < E.tL[0]) & (rotDiff.max(axis=1) < E.tL[1])] = True
    Enmin = np.minimum(EnPrev, En)  # :224-225
    if E.has("En"):
        Eo = np.asarray(E.En, float).copy()
        Eo[ind2EstOr] = Enmin[ind2EstOr]
    else:
        Eo = Enmin
    return E.copy(Tr=T.astype(np.float32), cT=cTFull, w=w, En=Eo, EnPrev=EnPrev)


def alternating_reconstruction(y, E, n_outer=10, n_cg=3, n_lm=1, winit=1e-3, tL=(0.05, 0.02), reg=1e-9,
                               on_stage=None, method="fft", dtype=np.float64):
    """The fixed-schedule alignment at one resolution (the small simulation
    case): n_outer times CGsolver (n_cg iterations, RelativeResidual2Error
    with tolerance 0, from the current image, A.Se = 1/(sum_c |S_c|^2 + reg),
    Reconstruction/solveXT.m:231-233,431), then n_lm LMsolver iterations
    (solveXT.m:507), with the motion-convergence resets of solveXT.m:379-384.
    E carries Sf, the sampling fields and the grids (E.Tr is ignored: motion
    starts at zero). on_stage(stage, n, x, E) after every update. Returns (x, E)."""
    S = int(E.NMs)
    Se = 1.0 / (np.sum(np.abs(E.Sf) ** 2, axis=3) + reg)
    A = enc.Struct(Se=Se)
    E = E.copy(Tr=np.zeros((S, 6), np.float32), w=np.full(S, winit), cT=np.zeros(S, bool), winit=winit,
               tL=list(tL))
    Sf = E.Sf
    x = None
    nReset, cont = 0, 0
    for n in range(n_outer):
        if nReset == 0 or cont % nReset == 0 or np.all(E.cT):
            nReset += 1
            cont = 0
            E = E.copy(cT=np.zeros(S, bool))
        cont += 1
        x, _, _ = CGsolver(y, E, None, A, None, None, x, n_cg, "RelativeResidual2Error", 0.0, method, dtype)
        if on_stage:
            on_stage("cg", n, x, E)
        for _ in range(n_lm):
            E = LMsolver(y, E.copy(Sf=Sf), x, method=method, dtype=dtype)
        E = E.copy(Sf=Sf)
        if on_stage:
            on_stage("lm", n, x, E)
    return x, E
