"""Fast synthesis of large scans on the GPU with torch (same recipe as
disorder_b200.synth, used by the benchmark to build 256x256x176 inputs in
seconds). Only the phantom and coil maps are built here; sampling, motion and
noise levels come from disorder_b200.synth."""

import numpy as np


def _grid(N, dev):
    import torch
    ax = [torch.linspace(-0.5, 0.5, n + 1, device=dev, dtype=torch.float32)[:-1] for n in N]
    return torch.meshgrid(*ax, indexing="ij")


def phantom_torch(N, n_ellipsoids, rng, dev="cuda"):
    import torch
    from .synth import _rot
    X, Y, Z = _grid(N, dev)
    mag = torch.zeros(N, device=dev)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.2, 0.2, 3)
        ax = rng.uniform(0.04, 0.25, 3)
        R = _rot(*rng.uniform(-np.pi, np.pi, 3))
        dx, dy, dz = X - c[0], Y - c[1], Z - c[2]
        u = (R[0, 0] * dx + R[0, 1] * dy + R[0, 2] * dz) / ax[0]
        v = (R[1, 0] * dx + R[1, 1] * dy + R[1, 2] * dz) / ax[1]
        w = (R[2, 0] * dx + R[2, 1] * dy + R[2, 2] * dz) / ax[2]
        mag += float(rng.uniform(0.2, 1.0)) * ((u * u + v * v + w * w) <= 1.0).float()
    ph = torch.zeros(N, device=dev)
    for _ in range(4):
        f = rng.uniform(0.3, 1.5, 3)
        p0 = rng.uniform(-np.pi, np.pi)
        a = rng.uniform(0.2, 0.6)
        ph += float(a) * torch.cos(2 * np.pi * (f[0] * X + f[1] * Y + f[2] * Z) + float(p0))
    x = torch.polar(mag, ph)
    return x / torch.linalg.vector_norm(x)


def coils_torch(N, n_coils, rng, width=0.45, dev="cuda"):
    import torch
    X, Y, Z = _grid(N, dev)
    S = torch.zeros(tuple(N) + (n_coils,), device=dev, dtype=torch.complex64)
    ga = np.pi * (3 - np.sqrt(5))
    for c in range(n_coils):
        zc = 1 - 2 * (c + 0.5) / n_coils
        rc = np.sqrt(max(0.0, 1 - zc * zc))
        th = ga * c
        cen = 0.6 * np.array([rc * np.cos(th), rc * np.sin(th), zc])
        d2 = (X - cen[0]) ** 2 + (Y - cen[1]) ** 2 + (Z - cen[2]) ** 2
        g = torch.exp(-d2 / (2 * width ** 2))
        k = rng.uniform(-2, 2, 3)
        ph = 2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) * 0.25 + float(rng.uniform(-np.pi, np.pi))
        S[..., c] = torch.polar(g, ph)
    rss = torch.sqrt(torch.sum(torch.abs(S) ** 2, dim=3, keepdim=True))
    return S / rss


def to_fortran_numpy(t):
    """torch tensor (MATLAB dim order) -> Fortran-ordered numpy array."""
    return np.asfortranarray(t.detach().cpu().numpy())
