"""Sinc-interpolated rigid transform, its factors and its gradient (oracle).

TEST INFRASTRUCTURE ONLY. Restates
  Methods/precomputeFactorsSincRigidTransform.m:24-133 (di, cg in {0,1}, gr=1, sh=1),
  Methods/sincRigidTransform.m:21-116,
  Methods/sincRigidTransformGradient.m:19-149,
  Methods/flipping.m:11-22, Methods/shifting.m:25-49,
  Methods/wrapToPiHalf.m:9-12, Methods/restrictTransform.m:28-32 and the
  Mapping Toolbox function wrapToPi (restated from its documented definition:
  angles outside [-pi, pi] are mapped to mod(x+pi, 2*pi)-pi, with positive odd
  multiples of pi mapped to +pi).

Volumes are 5-D arrays (N1, N2, N3, 1, S): motion states on axis 4 as in the
reference (dim 5). T is an (S, 6) float32 array: 3 translations (voxels of the
full-resolution grid) then 3 rotations (radians), the reference's
[1 1 1 1 S 6] layout (Reconstruction/solveXT.m:173).
"""

import numpy as np

from .grids import PER, along, fftGPU, ifftGPU, generateGrid

TR = np.array([[0, 2, 1], [1, 0, 2]])  # tr = [1 3 2; 2 1 3] (sincRigidTransform.m:33-34)


def wrapToPi(x):
    """Mapping Toolbox wrapToPi, restated from its definition."""
    x = np.array(x, copy=True)
    q = (x < -np.pi) | (np.pi < x)
    if np.any(q):
        y = x[q] + np.pi
        w = np.mod(y, 2 * np.pi)
        w[(w == 0) & (y > 0)] = 2 * np.pi
        x[q] = w - np.pi
    return x


def wrapToPiHalf(x):
    """Methods/wrapToPiHalf.m:9-12."""
    x = np.mod(x, np.pi).astype(x.dtype)
    ind = x > np.pi / 2
    x[ind] = x[ind] - np.asarray(np.pi, dtype=x.dtype)
    return x


def restrictTransform(T):
    """Methods/restrictTransform.m:28-32 (nargin<2 branch): wrap rotations into
    [-pi, pi] by repeated +-2*pi."""
    T = np.array(T, copy=True)
    a = T[:, 3:6]
    while np.any(a > np.pi):
        a[a > np.pi] -= 2 * np.pi
    while np.any(a < -np.pi):
        a[a < -np.pi] += 2 * np.pi
    T[:, 3:6] = a
    return T


class Factors:
    """Output of precomputeFactorsSincRigidTransform with gr=1 (per-axis
    translation factors) and sh=1. All tables carry the state axis (4)."""


def precomputeFactorsSincRigidTransform(grids_, T, di=1, cg=0, dtype=np.float64, cGrid=None):
    """Methods/precomputeFactorsSincRigidTransform.m:24-133 with gr=1, sh=1.

    Returns (et, etg) where et.e1[m], et.e2[m], et.e3[m] are the translation,
    tan-shear and sin-shear factors (et{1}{m}, et{2}{m}, et{3}{m}), et.flip[m]
    the per-state flip flags (et{5}{m}) and et.cent[m] the flip centres
    (et{4}{m}); etg carries the derivative factors (etg{1..3}{m}) when cg=1.
    dtype=float64 evaluates the reference's single-precision inputs in double
    precision; dtype=float32 emulates the reference's single arithmetic.
    """
    rdt = np.dtype(dtype)
    cdt = np.complex128 if rdt == np.float64 else np.complex64
    T = np.asarray(T, dtype=np.float32)
    S = T.shape[0]
    N = grids_.N
    if cGrid is None:
        cGrid = [n / 2.0 + 1 for n in N]  # :31
    Td = T.astype(rdt)
    t = ((-1) ** di) * 1j * Td[:, 0:3]  # :45
    theta = wrapToPi(Td[:, 3:6])  # :46
    et = Factors()
    et.flip = [np.abs(theta[:, n]) > np.pi / 2 for n in range(3)]  # :48-51
    et.cent = [{PER[0, n]: cGrid[PER[0, n]], PER[1, n]: cGrid[PER[1, n]]} for n in range(3)]  # :52
    theta = wrapToPiHalf(theta)  # :54
    tantheta2 = np.tan(theta / 2)  # :56-57
    tantheta2j = ((-1) ** (di - 1)) * 1j * tantheta2  # :58
    sintheta = ((-1) ** di) * 1j * np.sin(theta)  # :59-60
    if cg > 0:
        tanthetacuad = (1 + tantheta2 * tantheta2) / 2  # :63-64
        costheta = np.cos(theta)  # :65
    st = lambda v: along(v, 4)  # noqa: E731  states on axis 4
    et.e2, et.e3 = [], []
    for m in range(3):  # :78-81
        rk1 = grids_.rk(1, m).astype(rdt)
        rk2 = grids_.rk(2, m).astype(rdt)
        et.e2.append(np.exp(st(tantheta2j[:, m]) * rk1).astype(cdt))
        et.e3.append(np.exp(st(sintheta[:, m]) * rk2).astype(cdt))
    etg = None
    if cg > 0:
        etg = Factors()
        etg.e2, etg.e3 = [], []
        for m in range(3):  # :88-102
            rk1 = grids_.rk(1, m).astype(rdt)
            rk2 = grids_.rk(2, m).astype(rdt)
            etg.e2.append((1j * st(tanthetacuad[:, m]) * rk1 * et.e2[m]).astype(cdt))
            etg.e3.append((-1j * st(costheta[:, m]) * rk2 * et.e3[m]).astype(cdt))
    et.e1 = []
    for m in range(3):  # :114-115 (gr=1)
        k = along(grids_.kGrid[m].astype(rdt), m)
        et.e1.append(np.exp(st(t[:, m]) * k).astype(cdt))
    if cg > 0:
        etg.e1 = [(-1j * along(grids_.kGrid[m].astype(rdt), m)).astype(cdt) for m in range(3)]  # :120-125
    et.S = S
    et.N = N
    return et, etg


def shifting(x, H):
    """Methods/shifting.m:25-49 (f=0, zp=0) for complex x. H maps axis ->
    scalar shift. Integer shifts are circular index shifts (:29-37);
    others are DFT phase ramps exp(-i*k*h) with k the ifftshifted grid
    (2*pi/N)((1:N)-ceil((N+1)/2)) (:38-47)."""
    for m, hh in sorted(H.items()):
        n = x.shape[m]
        if float(hh) == np.round(hh):
            if n != 1:
                x = np.roll(x, int(round(hh)), axis=m)
        else:
            g, _ = generateGrid([n], nor=2 * np.pi, cent=[np.ceil((n + 1) / 2.0)])
            k = -1j * np.fft.ifftshift(g[0].astype(np.float64))
            ph = along(np.exp(hh * k), m, x.ndim).astype(x.dtype)
            x = ifftGPU(fftGPU(x, m) * ph, m)
    return x


def flipping(x, H):
    """Methods/flipping.m:11-22: shift by -c+0.5, flip, shift back by c-0.5."""
    H1 = {m: -c + 0.5 for m, c in H.items()}
    x = shifting(x, H1)
    H2 = {}
    for m in sorted(H1):
        H2[m] = -H1[m]
        x = np.flip(x, axis=m)
    return shifting(x, H2)


def _apply_flip(x, et, m):
    f = along(et.flip[m].astype(np.float64), 4).astype(x.real.dtype)
    return x * (1 - f) + flipping(x, et.cent[m]) * f


def _as5(x):
    x = np.asarray(x)
    while x.ndim < 5:
        x = x[..., None]
    return x


def sincRigidTransform(x, et, di=1, sumR=1, useFull=1, keep_intermediates=False):
    """Methods/sincRigidTransform.m:21-116 with gr=1 factors.

    x: volume (N1,N2,N3) or (N1,N2,N3,1,S). Returns the transformed states
    (N1,N2,N3,1,S) (forward) or, for di=0, the inverse transform summed over
    states when sumR (:113). With keep_intermediates the list xB{1..5}
    (:39,45,62/69) is returned as well.
    """
    x = _as5(x)
    if x.dtype not in (np.complex64, np.complex128):
        x = x.astype(np.complex128)
    if di == 1:
        xB = [None] * 5
        xB[4] = x
        if useFull != 0:
            for m in range(3):  # :42-54
                if np.any(et.flip[m]):
                    x = _apply_flip(x, et, m)
                x = fftGPU(x, TR[0, m])
                xB[m] = x
                x = x * et.e2[m]
                x = ifftGPU(x, TR[0, m])
                x = fftGPU(x, TR[1, m])
                x = x * et.e3[m]
                x = ifftGPU(x, TR[1, m])
                x = fftGPU(x, TR[0, m])
                x = x * et.e2[m]
                if m != 2:
                    x = ifftGPU(x, TR[0, m])
        if useFull != -1:  # :57-72
            for m in range(3):
                if m != TR[0, 2] or useFull == 0:
                    x = fftGPU(x, m)
            xB[3] = x
            for m in range(3):
                x = x * et.e1[m]
            for m in (2, 1, 0):
                x = ifftGPU(x, m)
        else:
            x = ifftGPU(x, TR[0, 2])  # :74
        if keep_intermediates:
            return x, xB
        return x
    # inverse (:76-113)
    if useFull != -1:
        for m in range(3):  # :86-90 (gr=1)
            x = fftGPU(x, m)
            x = x * et.e1[m]
            if m != TR[0, 2] or useFull == 0:
                x = ifftGPU(x, m)
    else:
        x = fftGPU(x, TR[0, 2])  # :94
    if useFull != 0:
        for m in (2, 1, 0):  # :99-111
            if m != 2:
                x = fftGPU(x, TR[0, m])
            x = x * et.e2[m]
            x = ifftGPU(x, TR[0, m])
            x = fftGPU(x, TR[1, m])
            x = x * et.e3[m]
            x = ifftGPU(x, TR[1, m])
            x = fftGPU(x, TR[0, m])
            x = x * et.e2[m]
            x = ifftGPU(x, TR[0, m])
            if np.any(et.flip[m]):
                x = _apply_flip(x, et, m)
    if sumR:
        x = np.sum(x, axis=(3, 4), keepdims=True)  # :113 multDimSum(x,4:ndT)
    return x


def sincRigidTransformGradient(xB, et, etg):
    """Methods/sincRigidTransformGradient.m:19-149 (gr=1 factors).

    Returns G[0..5]: derivatives of the forward transform with respect to
    the 3 translations and the 3 rotations, each (N1,N2,N3,1,S). The final
    crop (:149) is a no-op because the transform grid equals the volume grid.
    """
    G = [None] * 6
    for m in range(3):  # translations :29-36
        x1 = xB[3] * etg.e1[m]
        for n in range(3):
            x1 = x1 * et.e1[n]
        for n in range(3):
            x1 = ifftGPU(x1, n)
        G[m] = x1

    # first rotation :39-85
    x1 = xB[0] * et.e2[0]
    x2 = xB[0] * etg.e2[0]
    x1 = fftGPU(ifftGPU(x1, 0), 1)
    x2 = fftGPU(ifftGPU(x2, 0), 1)
    x2 = x1 * etg.e3[0] + x2 * et.e3[0]
    x1 = x1 * et.e3[0]
    x1 = fftGPU(ifftGPU(x1, 1), 0)
    x2 = fftGPU(ifftGPU(x2, 1), 0)
    x1 = x1 * etg.e2[0] + x2 * et.e2[0]
    x1 = ifftGPU(x1, 0)
    if np.any(et.flip[1]):
        x1 = _apply_flip(x1, et, 1)
    x1 = fftGPU(x1, 2)
    x1 = x1 * et.e2[1]
    x1 = ifftGPU(x1, 2)
    x1 = fftGPU(x1, 0)
    x1 = x1 * et.e3[1]
    x1 = ifftGPU(x1, 0)
    x1 = fftGPU(x1, 2)
    x1 = x1 * et.e2[1]
    x1 = ifftGPU(x1, 2)
    if np.any(et.flip[2]):
        x1 = _apply_flip(x1, et, 2)
    x1 = fftGPU(x1, 1)
    x1 = x1 * et.e2[2]
    x1 = ifftGPU(x1, 1)
    x1 = fftGPU(x1, 2)
    x1 = x1 * et.e3[2]
    x1 = ifftGPU(x1, 2)
    x1 = fftGPU(x1, 1)
    x1 = x1 * et.e2[2]
    G[3] = _translate_tail(x1, et)

    # second rotation :88-122
    x1 = xB[1] * et.e2[1]
    x2 = xB[1] * etg.e2[1]
    x1 = fftGPU(ifftGPU(x1, 2), 0)
    x2 = fftGPU(ifftGPU(x2, 2), 0)
    x2 = x1 * etg.e3[1] + x2 * et.e3[1]
    x1 = x1 * et.e3[1]
    x1 = fftGPU(ifftGPU(x1, 0), 2)
    x2 = fftGPU(ifftGPU(x2, 0), 2)
    x1 = x1 * etg.e2[1] + x2 * et.e2[1]
    x1 = ifftGPU(x1, 2)
    if np.any(et.flip[2]):
        x1 = _apply_flip(x1, et, 2)
    x1 = fftGPU(x1, 1)
    x1 = x1 * et.e2[2]
    x1 = ifftGPU(x1, 1)
    x1 = fftGPU(x1, 2)
    x1 = x1 * et.e3[2]
    x1 = ifftGPU(x1, 2)
    x1 = fftGPU(x1, 1)
    x1 = x1 * et.e2[2]
    G[4] = _translate_tail(x1, et)

    # third rotation :125-147
    x1 = xB[2] * et.e2[2]
    x2 = xB[2] * etg.e2[2]
    x1 = fftGPU(ifftGPU(x1, 1), 2)
    x2 = fftGPU(ifftGPU(x2, 1), 2)
    x2 = x1 * etg.e3[2] + x2 * et.e3[2]
    x1 = x1 * et.e3[2]
    x1 = fftGPU(ifftGPU(x1, 2), 1)
    x2 = fftGPU(ifftGPU(x2, 2), 1)
    x1 = x1 * etg.e2[2] + x2 * et.e2[2]
    G[5] = _translate_tail(x1, et)
    return G


def _translate_tail(x1, et):
    """The common tail (sincRigidTransformGradient.m:77-84 and repeats):
    DFT along dims 1 and 3, translation factors, inverse DFT along 3,2,1."""
    x1 = fftGPU(x1, 0)
    x1 = fftGPU(x1, 2)
    for m in range(3):
        x1 = x1 * et.e1[m]
    for m in (2, 1, 0):
        x1 = ifftGPU(x1, m)
    return x1
