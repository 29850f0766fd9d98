"""Seeded synthetic scans for the aligned reconstruction (input recipe).

The reference's own experiments load a ground-truth image and coil maps from
files that are not distributed (fig0506.m:53-56), so the phantom and coil
maps here are new: a sum of random ellipsoids with a smooth random phase and
Gaussian-bump coil sensitivities on a sphere, normalised to unit root sum of
squares. The sampling, motion and noise follow the reference's simulation
recipe:
  * shot orders: 'Random-checkered' (Simulation/synthesizeEncoding.m:86-106):
    the ky-kz grid is tiled with b1 x b2 tiles, b1*b2 = number of shots, and
    every tile gives each shot exactly one position through an independent
    random permutation; the mask is ifftshifted so DC comes first (:127).
    A square tile (b1 = b2 = sqrt(shots)) is the reference's case; for a
    non-square shot count the most square factorisation is used.
  * motion: Simulation/synthesizeT.m:36-40: uniform rotations and
    translations, mean removed over the shots (:40). The 3-D scans here draw
    all six parameters.
  * noise: Simulation/SNRToLevels.m:23-33 and Methods/plugNoise.m:17:
    complex Gaussian samples with sigma from the prescribed SNR in dB.
  * data: Simulation/synthesizeY.m:82-84: y = sum over shots of the encoded
    moved object plus noise (the encoding is done by the caller, on the GPU
    through disorder_b200.encode or on the CPU by the oracle).
Everything is NumPy and seeded with numpy.random.default_rng(seed).
"""

import numpy as np


def _rot(a, b, c):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    Rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def phantom(N, n_ellipsoids, rng, dtype=np.complex64):
    """Sum of random ellipsoids (magnitudes U(0.2,1)) times exp(i*phase) with
    a smooth random phase (a few random low-frequency cosines)."""
    N = tuple(int(n) for n in N)
    axes = [np.linspace(-0.5, 0.5, n, endpoint=False, dtype=np.float32) for n in N]
    mag = np.zeros(N, np.float32)
    X, Y, Z = np.meshgrid(*axes, indexing="ij", sparse=True)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.2, 0.2, 3)
        ax = rng.uniform(0.04, 0.25, 3)
        R = _rot(*rng.uniform(-np.pi, np.pi, 3)).astype(np.float32)
        dx, dy, dz = X - c[0], Y - c[1], Z - c[2]
        u = (R[0, 0] * dx + R[0, 1] * dy + R[0, 2] * dz) / ax[0]
        v = (R[1, 0] * dx + R[1, 1] * dy + R[1, 2] * dz) / ax[1]
        w = (R[2, 0] * dx + R[2, 1] * dy + R[2, 2] * dz) / ax[2]
        mag += np.float32(rng.uniform(0.2, 1.0)) * ((u * u + v * v + w * w) <= 1.0)
    ph = np.zeros(N, np.float32)
    for _ in range(4):
        f = rng.uniform(0.3, 1.5, 3)
        p0 = rng.uniform(-np.pi, np.pi)
        a = rng.uniform(0.2, 0.6)
        ph += np.float32(a) * np.cos(2 * np.pi * (f[0] * X + f[1] * Y + f[2] * Z) + p0).astype(np.float32)
    return (mag * np.exp(1j * ph)).astype(dtype)


def coil_maps(N, n_coils, rng, width=0.45, dtype=np.complex64):
    """Gaussian-bump sensitivities centred on a sphere around the volume
    (Fibonacci directions, radius 0.6 FOV), each with a random smooth phase,
    normalised so that sqrt(sum_c |S_c|^2) = 1 everywhere. Returns (N1,N2,N3,C)."""
    N = tuple(int(n) for n in N)
    axes = [np.linspace(-0.5, 0.5, n, endpoint=False, dtype=np.float32) for n in N]
    X, Y, Z = np.meshgrid(*axes, indexing="ij", sparse=True)
    S = np.zeros(N + (n_coils,), dtype)
    ga = np.pi * (3 - np.sqrt(5))
    for c in range(n_coils):
        zc = 1 - 2 * (c + 0.5) / n_coils
        rc = np.sqrt(max(0.0, 1 - zc * zc))
        th = ga * c
        cen = 0.6 * np.array([rc * np.cos(th), rc * np.sin(th), zc])
        d2 = (X - cen[0]) ** 2 + (Y - cen[1]) ** 2 + (Z - cen[2]) ** 2
        g = np.exp(-d2 / (2 * width ** 2)).astype(np.float32)
        k = rng.uniform(-2, 2, 3)
        ph = (2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) * 0.25 + rng.uniform(-np.pi, np.pi)).astype(np.float32)
        S[..., c] = g * np.exp(1j * ph)
    rss = np.sqrt(np.sum(np.abs(S) ** 2, axis=3, keepdims=True))
    return (S / rss).astype(dtype)


def tile_shape(n_shots):
    """Tile (b1, b2) with b1*b2 = n_shots: square when n_shots is a perfect
    square (the reference's requirement, synthesizeEncoding.m:87,93),
    otherwise the most square factorisation."""
    b1 = int(np.floor(np.sqrt(n_shots)))
    while n_shots % b1:
        b1 -= 1
    return b1, n_shots // b1


def random_checkered(NY, n_shots, rng, truncate=False):
    """Simulation/synthesizeEncoding.m:86-106,127: returns the (NY1, NY2)
    array of 1-based shot indices with DC first (ifftshifted).

    The reference requires tiles that divide the grid. With truncate=True a
    grid that the b1 x b2 tile does not divide is covered by
    ceil(NY1/b1) x ceil(NY2/b2) tiles whose last row and column are cut at the
    grid edge: every full tile still gives each shot one position, and an edge
    tile gives its positions to the shots of its permutation that land
    inside the grid (the rectangular variant used for shot counts such as 96
    on a 128 x 160 grid)."""
    b1, b2 = tile_shape(n_shots)
    NY1, NY2 = int(NY[0]), int(NY[1])
    if (NY1 % b1 or NY2 % b2) and not truncate:
        raise ValueError("grid %dx%d is not tiled by %dx%d" % (NY1, NY2, b1, b2))
    H = np.zeros((NY1, NY2), np.int32)
    for o in range(-(-NY1 // b1)):
        for p in range(-(-NY2 // b2)):
            perm = rng.permutation(n_shots)  # indRand = randperm(NNT)
            IR, JR = np.unravel_index(perm, (b1, b2), order="F")  # ind2sub
            s = np.arange(n_shots)
            r, c = IR + o * b1, JR + p * b2
            keep = (r < NY1) & (c < NY2)
            H[r[keep], c[keep]] = s[keep] + 1
    return np.fft.ifftshift(H)


def motion(n_shots, rot_deg, trans_vox, rng):
    """Simulation/synthesizeT.m:36-40 for all six parameters: rotations
    U(-rot_deg, rot_deg) (radians) and translations U(-trans_vox, trans_vox),
    mean over shots removed. Returns (n_shots, 6) float32 [t1 t2 t3 r1 r2 r3]."""
    T = np.zeros((n_shots, 6))
    T[:, 3:6] = np.pi * (2 * rot_deg) * (rng.random((n_shots, 3)) - 0.5) / 180
    T[:, 0:3] = (2 * trans_vox) * (rng.random((n_shots, 3)) - 0.5)
    T -= T.mean(axis=0, keepdims=True)
    return T.astype(np.float32)


def snr_to_sigma(snr_db, x_gt, S):
    """Simulation/SNRToLevels.m:23-33, for the unitary encoding of the aligned
    reconstruction. The reference divides the noise amplification by
    numel(xGT) (:31) because its simulation encoder applies the unnormalised
    DFT; with the unitary DFT of encode.m (build1DFTM(N,1)) the same image
    SNR needs that factor left out, i.e. sigma is the reference's divided by
    sqrt(numel(xGT))."""
    meanS = np.mean(np.abs(x_gt) ** 2)
    meanN = meanS / (10 ** (snr_db / 10))
    P = np.mean(1.0 / (np.sum(np.abs(S) ** 2, axis=3) + 1e-3))
    return float(np.sqrt(meanN / (2 * P)))


def plug_noise(shape, sigma, rng, dtype=np.complex64):
    """Methods/plugNoise.m:17 scaled by sigma: sigma*(randn + 1i*randn)."""
    return (sigma * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))).astype(dtype)


def sample_lists(H, n_shots):
    """Per-sample (ky, kz) row indices grouped by shot, in the order of
    Methods/buildHarmonicSampling.m:36-44 (shots 1..S then the unassigned
    points as segment S+1; column-major order inside a shot). Returns
    (ky, kz, nEc offsets of length S+2, mSt segment of each sample, iSt
    column-major linear index of each sample)."""
    Hf = np.asarray(H).reshape(-1, order="F")
    idx, seg = [], []
    for s in range(1, n_shots + 2):
        ind = np.flatnonzero(Hf == (s % (n_shots + 1)))
        idx.append(ind)
        seg.append(np.full(len(ind), s - 1, np.int32))
    iSt = np.concatenate(idx)
    ky, kz = np.unravel_index(iSt, np.asarray(H).shape, order="F")
    nEc = np.concatenate([[0], np.cumsum([len(i) for i in idx])]).astype(np.int64)
    return ky.astype(np.int32), kz.astype(np.int32), nEc, np.concatenate(seg), iSt


class Scan:
    """A synthetic scan: x_gt (N), coils S (N + (C,)), shot map H, per-sample
    lists, ground-truth motion T_gt, noise sigma."""


def make_scan(N, n_coils, n_shots, rot_deg, trans_vox, snr_db, n_ellipsoids, seed,
              dtype=np.complex64):
    rng = np.random.default_rng(seed)
    sc = Scan()
    sc.N = tuple(int(n) for n in N)
    x = phantom(N, n_ellipsoids, rng, dtype)
    x = (x / np.linalg.norm(x.ravel())).astype(dtype)  # fig0506.m:95
    sc.x_gt = x
    sc.S = coil_maps(N, n_coils, rng, dtype=dtype)
    sc.H = random_checkered(N[:2], n_shots, rng)
    sc.n_shots = n_shots
    sc.ky, sc.kz, sc.nEc, sc.mSt, sc.iSt = sample_lists(sc.H, n_shots)
    sc.T_gt = motion(n_shots, rot_deg, trans_vox, rng)
    sc.sigma = snr_to_sigma(snr_db, x, sc.S)
    sc.noise_seed = seed + 7919
    return sc


def add_noise(y, sigma, seed):
    rng = np.random.default_rng(seed)
    return (y + plug_noise(y.shape, sigma, rng, y.dtype)).astype(y.dtype)
