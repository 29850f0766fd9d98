"""Synthetic scans built on the GPU by the library's own kernels
(disorder_synth_phantom, disorder_synth_coils, disorder_add_noise).

The random parameters are drawn on the host with the same generator calls, in
the same order, as the NumPy recipe in disorder_b200.synth (phantom: per
ellipsoid centre, semi-axes, rotation angles and magnitude, then four phase
terms; coils: per coil a wave vector and a phase), so a scan built here from
numpy.random.default_rng(seed) matches synth.phantom / synth.coil_maps from
the same seed up to single-precision rounding. Sampling and motion come from
disorder_b200.synth (host, cheap); the noise is drawn on the device.
"""

import ctypes as C
import math

import numpy as np

from . import _lib
from .synth import _rot


def phantom_params(n_ellipsoids, rng):
    """(ellipsoids (n, 16) float32, phase terms (4, 5) float32) drawn as
    synth.phantom draws them."""
    ell = np.zeros((n_ellipsoids, 16), np.float32)
    for q in range(n_ellipsoids):
        c = rng.uniform(-0.2, 0.2, 3)
        ax = rng.uniform(0.04, 0.25, 3)
        R = _rot(*rng.uniform(-np.pi, np.pi, 3)).astype(np.float32)
        ell[q, 0:3] = c
        ell[q, 3:6] = ax
        ell[q, 6:15] = R.reshape(-1)
        ell[q, 15] = np.float32(rng.uniform(0.2, 1.0))
    ph = np.zeros((4, 5), np.float32)
    for q in range(4):
        ph[q, 0:3] = rng.uniform(0.3, 1.5, 3)
        ph[q, 3] = rng.uniform(-np.pi, np.pi)
        ph[q, 4] = rng.uniform(0.2, 0.6)
    return ell, ph


def coil_params(n_coils, rng):
    """(n_coils, 7) float32: centre on a sphere (Fibonacci directions, radius
    0.6), wave vector and phase, as synth.coil_maps draws them."""
    cp = np.zeros((n_coils, 7), np.float32)
    ga = np.pi * (3 - np.sqrt(5))
    for c in range(n_coils):
        zc = 1 - 2 * (c + 0.5) / n_coils
        rc = np.sqrt(max(0.0, 1 - zc * zc))
        th = ga * c
        cp[c, 0:3] = 0.6 * np.array([rc * np.cos(th), rc * np.sin(th), zc])
        cp[c, 3:6] = rng.uniform(-2, 2, 3)
        cp[c, 6] = rng.uniform(-np.pi, np.pi)
    return cp


def phantom(ctx, N, n_ellipsoids, rng, normalise=True):
    """The ellipsoid phantom as a device volume (N1, N2, N3), unit L2 norm
    when normalise (fig0506.m:95)."""
    ell, ph = phantom_params(n_ellipsoids, rng)
    out = ctx.empty(tuple(N))
    Nc = (C.c_int32 * 3)(*[int(n) for n in N])
    ctx.check(ctx.lib.disorder_synth_phantom(ctx.h, Nc, int(n_ellipsoids), ell.ctypes.data_as(_lib.FP), 4,
                                             ph.ctypes.data_as(_lib.FP), 1 if normalise else 0, out.ptr))
    return out


def coil_maps(ctx, N, n_coils, rng, width=0.45):
    """Gaussian-bump coil maps (N1, N2, N3, C) with unit root sum of squares."""
    cp = coil_params(n_coils, rng)
    S = ctx.empty(tuple(N) + (int(n_coils),))
    Nc = (C.c_int32 * 3)(*[int(n) for n in N])
    ctx.check(ctx.lib.disorder_synth_coils(ctx.h, Nc, int(n_coils), cp.ctypes.data_as(_lib.FP), float(width), S.ptr))
    return S


def add_noise(ctx, y, sigma, seed):
    """y += sigma * (n1 + i n2) in place (Methods/plugNoise.m:17)."""
    ctx.check(ctx.lib.disorder_add_noise(ctx.h, y.ptr, int(np.prod(y.shape)), float(sigma), int(seed) & (2**64 - 1)))


def snr_sigma(snr_db, V, ridge=1e-3):
    """synth.snr_to_sigma for a unit-norm image of V voxels and coils with unit
    root sum of squares: mean |x|^2 = 1/V and mean 1/(sum|S|^2 + 1e-3) =
    1/(1 + 1e-3) (Simulation/SNRToLevels.m:23-33, unitary encoding)."""
    meanN = (1.0 / V) / (10 ** (snr_db / 10))
    return float(math.sqrt(meanN / (2.0 / (1.0 + ridge))))
