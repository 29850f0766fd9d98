"""Motion-proposal network (oracle; test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of the learned motion proposal's
forward and backward kernels. The network has no counterpart in the
reference, so it is restated from its own definition:
  input  (B, n3, n2, n1, 4): a state's back-projected residual times s_in and
         the current image times s_ref (shared by the batch), each read as
         real/imaginary channels (``features``);
  4 x    conv 3x3x3, stride 2, zero padding 1 (channels 16, 32, 64, 64),
         bias, exact GELU z*Phi(z);
  global average pool -> fc 64->128, GELU -> fc 128->6;
  loss   sum_b sum_k (out - target)^2 / B.
Parameters are one flat FP32 vector in the order the C ABI documents (per
convolution the weights [tap=(kz*3+ky)*3+kx][c_in][c_out] then the bias; fc1
[64][128] and bias; fc2 [128][6] and bias). The device computes with the
parameters rounded to BF16, so ``bf16_round`` is applied before the FP64
arithmetic here. ``grad`` is exact backpropagation, pinned against central
finite differences of ``forward`` by the tests.
"""

import numpy as np
from scipy.special import erf

CH = (4, 16, 32, 64, 64)
HID = 128
OUT = 6


def layout():
    """Offsets (w, b) per convolution, then fc1 w/b and fc2 w/b; total count."""
    o = 0
    conv = []
    for l in range(4):
        w = o
        o += 27 * CH[l] * CH[l + 1]
        b = o
        o += CH[l + 1]
        conv.append((w, b))
    f1w = o
    o += CH[4] * HID
    f1b = o
    o += HID
    f2w = o
    o += HID * OUT
    f2b = o
    o += OUT
    return conv, (f1w, f1b, f2w, f2b), o


def param_count():
    return layout()[2]


def bf16_round(p):
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    u = np.ascontiguousarray(p, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def init_params(rng):
    """He-style initialisation (weights N(0, 2/fan_in), zero bias), FP32."""
    conv, (f1w, f1b, f2w, f2b), P = layout()
    p = np.zeros(P, np.float32)
    for l, (w, b) in enumerate(conv):
        fan = 27 * CH[l]
        p[w:b] = rng.standard_normal(b - w) * np.sqrt(2.0 / fan)
    p[f1w:f1b] = rng.standard_normal(f1b - f1w) * np.sqrt(2.0 / CH[4])
    p[f2w:f2b] = rng.standard_normal(f2b - f2w) * np.sqrt(1.0 / HID)
    return p


def _gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def _gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _unpack(p, rnd=True):
    conv, (f1w, f1b, f2w, f2b), _ = layout()
    q = (bf16_round(p) if rnd else np.asarray(p)).astype(np.float64)
    Ws = [q[w:b].reshape(27, CH[l], CH[l + 1]) for l, (w, b) in enumerate(conv)]
    bs = [q[b:b + CH[l + 1]] for l, (w, b) in enumerate(conv)]
    return Ws, bs, q[f1w:f1b].reshape(CH[4], HID), q[f1b:f2w], q[f2w:f2b].reshape(HID, OUT), q[f2b:f2b + OUT]


def _out_size(n):
    return (n + 1) // 2


def _taps(a, O):
    """Views of the zero-padded input a (B, I3, I2, I1, C) at 2o-1+k per axis."""
    B, I3, I2, I1, C = a.shape
    O3, O2, O1 = O
    pad = np.zeros((B, 2 * O3 + 1, 2 * O2 + 1, 2 * O1 + 1, C))
    pad[:, 1:I3 + 1, 1:I2 + 1, 1:I1 + 1] = a
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                yield (kz * 3 + ky) * 3 + kx, pad[:, kz:kz + 2 * O3:2, ky:ky + 2 * O2:2, kx:kx + 2 * O1:2]


def _conv(a, W, b):
    O = tuple(_out_size(n) for n in a.shape[1:4])
    z = np.zeros(a.shape[:1] + O + (W.shape[2],))
    for t, v in _taps(a, O):
        z += v @ W[t]
    return z + b


def features(vols, ref=None, s_in=1.0, s_ref=1.0):
    """(B, N1, N2, N3) complex volumes and one (N1, N2, N3) reference volume
    (MATLAB order) -> (B, n3, n2, n1, 4) network input."""
    v = np.transpose(np.asarray(vols, np.complex128), (0, 3, 2, 1)) * s_in
    r = np.zeros(v.shape[1:], np.complex128) if ref is None else np.transpose(np.asarray(ref, np.complex128)) * s_ref
    r = np.broadcast_to(r, v.shape)
    return np.stack([v.real, v.imag, r.real, r.imag], axis=-1)


def forward(p, x, rnd=True):
    """x: (B, n3, n2, n1, 4) input. Returns (out (B, 6), cache). rnd=False
    skips the BF16 rounding of the parameters (for finite differences)."""
    Ws, bs, W1, b1, W2, b2 = _unpack(p, rnd)
    a = np.asarray(x, np.float64)
    acts, pres = [a], []
    for l in range(4):
        z = _conv(acts[-1], Ws[l], bs[l])
        pres.append(z)
        acts.append(_gelu(z))
    g = acts[-1].mean(axis=(1, 2, 3))
    hp = g @ W1 + b1
    h = _gelu(hp)
    out = h @ W2 + b2
    return out, (acts, pres, g, hp, h)


def loss(p, x, target, rnd=True):
    out, _ = forward(p, x, rnd)
    return float(np.sum((out - target) ** 2) / out.shape[0])


def grad(p, x, target, rnd=True):
    """Gradient of ``loss`` with respect to the (BF16-rounded) parameters."""
    conv, (f1w, f1b, f2w, f2b), P = layout()
    Ws, bs, W1, b1, W2, b2 = _unpack(p, rnd)
    out, (acts, pres, g, hp, h) = forward(p, x, rnd)
    B = out.shape[0]
    G = np.zeros(P)
    dout = 2.0 * (out - target) / B
    G[f2w:f2b] = (h.T @ dout).ravel()
    G[f2b:f2b + OUT] = dout.sum(0)
    dhp = (dout @ W2.T) * _gelu_grad(hp)
    G[f1w:f1b] = (g.T @ dhp).ravel()
    G[f1b:f2w] = dhp.sum(0)
    dg = dhp @ W1.T
    nvox = np.prod(pres[3].shape[1:4])
    dz = np.broadcast_to(dg[:, None, None, None, :] / nvox, pres[3].shape) * _gelu_grad(pres[3])
    for l in range(3, -1, -1):
        a = acts[l]
        O = dz.shape[1:4]
        w, b = conv[l]
        dW = np.zeros_like(Ws[l])
        da = np.zeros((B, 2 * O[0] + 1, 2 * O[1] + 1, 2 * O[2] + 1, a.shape[4]))
        for t, v in _taps(a, O):
            dW[t] = np.einsum("bzyxi,bzyxo->io", v, dz)
            kz, ky, kx = t // 9, (t // 3) % 3, t % 3
            da[:, kz:kz + 2 * O[0]:2, ky:ky + 2 * O[1]:2, kx:kx + 2 * O[2]:2] += dz @ Ws[l][t].T
        G[w:b] = dW.ravel()
        G[b:b + CH[l + 1]] = dz.sum(axis=(0, 1, 2, 3))
        if l > 0:
            I3, I2, I1 = a.shape[1:4]
            dz = da[:, 1:I3 + 1, 1:I2 + 1, 1:I1 + 1] * _gelu_grad(pres[l - 1])
    return G, out
