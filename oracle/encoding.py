"""Encoding operators: encode, decode, encodedecode, computeEnergy (oracle).

TEST INFRASTRUCTURE ONLY. Restates the hot-path fields of
Reconstruction/encode.m:1-147, Reconstruction/decode.m:1-160,
Reconstruction/encodedecode.m:1-250 and Reconstruction/computeEnergy.m:34-80.

Supported structure fields (the ones the aligned reconstruction sets):
  E.Tr (NMs x 6), E.NMs, E.NSe, E.Sf (N1,N2,N3,C), E.Fs (given as per-sample
  DFT row indices ky/kz with segment offsets E.nEc), E.vA, E.kG/E.rkG (grids),
  E.nF (readout crop, LMsolver only); EH.We (per-sample weights), EH.Mb and
  EH.Mbe (readout masks). Folding E.Uf/EH.Ub is the identity when the
  reconstruction and acquisition grids agree (Methods/fold.m:20), which is the
  only case supported.

Two evaluation methods give the same operator:
  method="rows": the reference's literal per-sample DFT rows
    (encode.m:120-136, decode.m:42-58, encodedecode.m:119-143), cost
    O(Ns*N1*N2*N3*C); small sizes only.
  method="fft": the separable full 2-D DFT plus gather/scatter of the same
    unitary DFT (DC-first rows of build1DFTM(N,1), buildHarmonicSampling.m:30,39).
Samples y have shape (Ns_total, N3, C) (the reference's [Ns 1 N3 C]).
"""

import numpy as np

from .grids import build1DFTM, fftGPU, ifftGPU
from .transform import precomputeFactorsSincRigidTransform, sincRigidTransform


class Struct:
    """A MATLAB-struct-like bag of fields."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def has(self, name):
        return getattr(self, name, None) is not None

    def copy(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return Struct(**d)


def _segments(E):
    if E.has("vA"):
        return list(E.vA)
    return list(range(E.NSe))


def _any_motion(E):
    return E.has("Tr") and np.any(np.asarray(E.Tr) != 0)


def transform_states(x, E, segs, di, dtype=np.float64):
    """The RIGID TRANSFORM block of encode.m:59-80 for the segments segs:
    transformed copies of x for motion segments (< NMs), untransformed copies
    for the outer segments. Returns (N1,N2,N3,1,len(segs))."""
    x5 = x.reshape(x.shape[:3] + (1, 1))
    mot = [s for s in segs if s < E.NMs]
    outs = []
    if mot:
        if _any_motion(E):
            et, _ = precomputeFactorsSincRigidTransform(E.grids, np.asarray(E.Tr)[mot], di, 0, dtype)
            outs.append(sincRigidTransform(x5, et, di))
        else:
            outs.append(np.repeat(x5, len(mot), axis=4))
    n_out = len(segs) - len(mot)
    if n_out:
        outs.append(np.repeat(x5, n_out, axis=4))
    return np.concatenate(outs, axis=4)


def _dft_rows(E):
    N1, N2 = E.Sf.shape[0], E.Sf.shape[1]
    F1, _ = build1DFTM(N1, 1)
    F2, _ = build1DFTM(N2, 1)
    return F1, F2


def _encode_states(xT, E, segs, method):
    """Coil profiles + FOURIER DOMAIN (SEGMENTS) of encode.m:90-136 for the
    transformed states xT (N1,N2,N3,1,len(segs)); returns (Ns, N3, C)."""
    S = E.Sf
    N1, N2, N3, C = S.shape
    outs = []
    if method == "rows":
        F1, F2 = _dft_rows(E)
    for j, s in enumerate(segs):
        a, b = int(E.nEc[s]), int(E.nEc[s + 1])
        if b == a:
            continue
        ky, kz = E.ky[a:b], E.kz[a:b]
        xS = xT[:, :, :, 0, j][..., None] * S  # (N1,N2,N3,C)
        if method == "rows":
            xQ = np.einsum("in,nmrc->imrc", F1[ky], xS)  # aplGPU(F1rows, x, 1)
            yq = np.einsum("imrc,im->irc", xQ, F2[kz])  # sum(xQ.*F2rows, 2)
        else:
            X = fftGPU(fftGPU(xS, 0), 1) / np.sqrt(N1 * N2)
            yq = X[ky, kz]
        outs.append(yq)
    if not outs:
        return np.zeros((0, N3, C), dtype=np.result_type(xT, S))
    return np.concatenate(outs, axis=0)


def encode(x, E, method="fft", dtype=np.float64):
    """Reconstruction/encode.m:1-147 (hot fields). x is one volume
    (N1,N2,N3) or, when E has no Tr, already-transformed states
    (N1,N2,N3,1,S) aligned with the segments (LMsolver calls it that way)."""
    segs = _segments(E)
    if E.has("Tr"):
        xT = transform_states(x, E, segs, 1, dtype)
    else:
        xT = x if x.ndim == 5 else x.reshape(x.shape[:3] + (1, 1))
        if xT.shape[4] == 1 and len(segs) > 1:
            xT = np.repeat(xT, len(segs), axis=4)
    return _encode_states(xT, E, segs, method)


def _sample_weights(EH, a, b):
    if EH is not None and EH.has("We") and len(EH.We):
        return np.asarray(EH.We)[a:b]
    return None


def _decode_states(y, E, EH, segs, method, apply_we=True):
    """FOURIER DOMAIN (SEGMENTS) + COIL PROFILES of decode.m:42-58,78-85: per
    segment F^H of its samples, times conj(S), summed over coils."""
    S = E.Sf
    N1, N2, N3, C = S.shape
    out = np.zeros((N1, N2, N3, 1, len(segs)), dtype=np.result_type(y, S, np.complex64))
    if method == "rows":
        F1, F2 = _dft_rows(E)
    for j, s in enumerate(segs):
        a, b = int(E.nEc[s]), int(E.nEc[s + 1])
        if b == a:
            continue
        yR = y[a:b]
        we = _sample_weights(EH, a, b) if apply_we else None
        if we is not None:
            yR = yR * we[:, None, None]
        ky, kz = E.ky[a:b], E.kz[a:b]
        if method == "rows":
            xQ = yR[:, None, :, :] * np.conj(F2[kz])[:, :, None, None]  # (Ns,N2,N3,C)
            xo = np.einsum("in,imrc->nmrc", np.conj(F1[ky]), xQ)
        else:
            K = np.zeros((N1, N2, N3, C), dtype=out.dtype)
            np.add.at(K, (ky, kz), yR)
            xo = ifftGPU(ifftGPU(K, 0), 1) * np.sqrt(N1 * N2)
        out[:, :, :, 0, j] = np.sum(xo * np.conj(S), axis=3)
    return out


def _inverse_and_sum(xo, E, segs, dtype):
    """RIGID TRANSFORM (MOTION STATES) of decode.m:95-113: inverse transform of
    the motion segments (sumR=0), then sum over all segments."""
    mot = [j for j, s in enumerate(segs) if s < E.NMs]
    if E.has("Tr") and _any_motion(E) and mot:
        et, _ = precomputeFactorsSincRigidTransform(E.grids, np.asarray(E.Tr)[[segs[j] for j in mot]], 0, 0, dtype)
        xo = xo.copy()
        xo[..., mot] = sincRigidTransform(xo[..., mot], et, 0, sumR=0)
    return np.sum(xo, axis=(3, 4))


def decode(y, EH, E, method="fft", dtype=np.float64):
    """Reconstruction/decode.m:1-160 (hot fields). Returns (N1,N2,N3)."""
    if EH is not None and EH.has("Mb"):
        y = y * np.asarray(EH.Mb)[None, :, None]  # decode.m:23
    segs = _segments(E)
    xo = _decode_states(y, E, EH, segs, method)
    return _inverse_and_sum(xo, E, segs, dtype)


def encodedecode(x, E, EH, method="fft", dtype=np.float64):
    """Reconstruction/encodedecode.m:1-212 (hot fields): the normal operator
    sum_s T_s^H sum_c S_c^H F_s^H W_s F_s S_c T_s x. EH.We weights the
    samples between the forward and adjoint DFT (:133); EH.Mb is NOT applied
    here (the reference applies it in decode only)."""
    segs = _segments(E)
    xT = transform_states(x, E, segs, 1, dtype) if E.has("Tr") else np.repeat(
        x.reshape(x.shape[:3] + (1, 1)), len(segs), axis=4)
    yk = _encode_states(xT, E, segs, method)
    # samples of all segments, concatenated in segment order, are decoded back
    Esub = E
    if E.has("vA"):
        # re-index offsets to the concatenated block
        offs = [0]
        for s in segs:
            offs.append(offs[-1] + int(E.nEc[s + 1] - E.nEc[s]))
        ky = np.concatenate([E.ky[int(E.nEc[s]):int(E.nEc[s + 1])] for s in segs])
        kz = np.concatenate([E.kz[int(E.nEc[s]):int(E.nEc[s + 1])] for s in segs])
        Esub = E.copy(nEc=np.array(offs), ky=ky, kz=kz, vA=None)
        EHs = None
        if EH is not None and EH.has("We") and len(EH.We):
            We = np.concatenate([np.asarray(EH.We)[int(E.nEc[s]):int(E.nEc[s + 1])] for s in segs])
            EHs = Struct(We=We)
        xo = _decode_states(yk, Esub, EHs, list(range(len(segs))), method)
    else:
        xo = _decode_states(yk, Esub, EH, segs, method)
    return _inverse_and_sum(xo, E, segs, dtype)


def computeEnergy(y, x, E, R=None, EH=None, method="fft", per_sample=False, dtype=np.float64):
    """Reconstruction/computeEnergy.m:34-80 for no=2 (least squares).

    Returns [fidelity, regularisation]: fidelity = sum |sqrt(Mb) sqrt(Mbe)
    (E x - y)|^2 (:34-39,55-57), regularisation = |sum (R.Ti.la x) conj(x)|
    (:72-76, regularize.m:24). With per_sample (the avdi form used at
    solveXT.m:443) returns the per-sample sums over readout and coils.
    """
    res = encode(x, E, method, dtype) - y
    if EH is not None and EH.has("Mb"):
        res = res * np.sqrt(np.asarray(EH.Mb))[None, :, None]
    if EH is not None and EH.has("Mbe"):
        res = res * np.sqrt(np.asarray(EH.Mbe))[None, :, None]
    fi2 = np.abs(res) ** 2
    if per_sample:
        return np.sum(fi2, axis=(1, 2))
    fid = float(np.sum(fi2))
    reg = 0.0
    if R is not None and R.has("Ti"):
        reg = float(abs(np.sum(np.asarray(R.Ti) * x * np.conj(x))))
    return np.array([fid, reg])
