"""Learned motion proposal (no counterpart in the reference).

A small 3-D convolutional network, run and trained by the library's own
kernels (``disorder_net_*`` in include/disorder.h), proposes each motion
state's update from that state's back-projected k-space residual at the
coarsest pyramid level. The plain Levenberg-Marquardt step
(Reconstruction/LMsolver.m) still decides: ``propose_step`` keeps a
proposal only for the states whose energy it lowers (the energy LMsolver.m
evaluates at :82-83 and :196), and the LM step then runs from the kept
motion, so a poor proposal costs at most the evaluation.

Training data are simulated by the method itself: phantom, coils and
DISORDER random-checkered shots as Simulation/synthesizeEncoding.m and
synthesizeT.m / synthesizeY.m build them, encoded with the library's encode,
a few CG iterations at a perturbed motion, and the per-state back-projection
of the residual (``backproject_states``).
"""

import ctypes as C
import math
import os
import time

import numpy as np

from . import _lib, api, synth

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "proposal_64x64x44.npz")

CH = (4, 16, 32, 64, 64)
HID = 128
OUT = 6
# network output units: translations in voxels of the level's grid / 2,
# rotations in radians / (8 deg)
TRANS_UNIT = 2.0
ROT_UNIT = 8.0 * math.pi / 180


def param_count():
    return int(_lib.load().disorder_net_param_count())


def init_params(rng):
    """He-style initial parameters in the ABI's flat order (FP32): conv
    weights N(0, 2/fan_in), fc1 N(0, 2/64), fc2 N(0, 1/128), zero biases."""
    parts = []
    for l in range(4):
        n = 27 * CH[l] * CH[l + 1]
        parts += [rng.standard_normal(n) * math.sqrt(2.0 / (27 * CH[l])), np.zeros(CH[l + 1])]
    parts += [rng.standard_normal(CH[4] * HID) * math.sqrt(2.0 / CH[4]), np.zeros(HID)]
    parts += [rng.standard_normal(HID * OUT) * math.sqrt(1.0 / HID), np.zeros(OUT)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == param_count()
    return p


class MotionNet:
    """The proposal network on one context. D: input volume (n1, n2, n3)."""

    def __init__(self, ctx, D, max_batch=64, params=None, gain=1.0):
        self.ctx = ctx
        self.D = tuple(int(d) for d in D)
        self.max_batch = int(max_batch)
        self.gain = float(gain)
        h = C.c_void_p()
        Dv = (C.c_int32 * 3)(*self.D)
        ctx.check(ctx.lib.disorder_net_create(ctx.h, Dv, self.max_batch, C.byref(h)))
        self.h = h
        ctx.adopt(self)
        self.P = param_count()
        self.step = 0
        self.set_params(init_params(np.random.default_rng(0)) if params is None else params)

    def close(self):
        if getattr(self, "h", None) is not None and self.ctx.h is not None:
            self.ctx.lib.disorder_net_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.P:
            raise ValueError("expected %d parameters, got %d" % (self.P, p.size))
        self.ctx.check(self.ctx.lib.disorder_net_set_params(self.ctx.h, self.h, p.ctypes.data_as(_lib.FP)))
        self.step = 0

    def get_params(self):
        p = np.empty(self.P, np.float32)
        self.ctx.check(self.ctx.lib.disorder_net_get_params(self.ctx.h, self.h, p.ctypes.data_as(_lib.FP)))
        return p

    def forward(self, vols, ref, batch, s_in, s_ref, out=None):
        """vols: device complex volumes (batch of size D), ref: one device
        complex volume or None. Returns (batch, 6) outputs on the host; out
        (device, batch x 6 FP32) also receives them."""
        o = out if out is not None else self.ctx.empty((OUT, batch), np.float32)
        self.ctx.check(self.ctx.lib.disorder_net_forward(self.ctx.h, self.h, vols.ptr,
                                                         ref.ptr if ref is not None else None, int(batch),
                                                         float(s_in), float(s_ref), o.ptr))
        self._inputs = (vols, ref)  # backward reads the first layer's inputs again
        return o.numpy().T.copy()

    def backward(self, target, batch, grad):
        """Gradient of the loss of the last forward into grad (device FP32 P).
        target: device (6, batch) FP32 array (row-major batch x 6)."""
        loss = C.c_double()
        self.ctx.check(self.ctx.lib.disorder_net_backward(self.ctx.h, self.h, target.ptr, int(batch), grad.ptr,
                                                          C.byref(loss)))
        return float(loss.value)

    def adam(self, grad, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        self.ctx.check(self.ctx.lib.disorder_net_adam(self.ctx.h, self.h, grad.ptr, float(lr), float(beta1),
                                                      float(beta2), float(eps), self.step))

    def propose(self, y, E, x, nF=None):
        """Proposed update (n_states, 6) in T's units for every motion state."""
        ctx = self.ctx
        p = api._plan(E, ctx)
        yd, _ = api._dev(ctx, y, np.complex64)
        xd, _ = api._dev(ctx, x, np.complex64)
        Sd, _ = api._dev(ctx, E.Sf, np.complex64)
        Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
        lo, hi = _range(E, nF)
        S = p.n_mot
        Tf = np.asfortranarray(np.asarray(E.Tr, np.float32))
        dT = np.zeros((S, 6), np.float32, order="F")
        ctx.check(ctx.lib.disorder_propose_motion(ctx.h, p.h, self.h, yd.ptr, Sd.ptr, Cn, xd.ptr,
                                                  Tf.ctypes.data_as(_lib.FP), lo, hi, self.gain,
                                                  dT.ctypes.data_as(_lib.FP)))
        return np.array(dT)

    def save(self, path, meta=None):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.get_params(), D=np.array(self.D), gain=np.float64(self.gain),
                 **(meta or {}))

    @classmethod
    def load(cls, ctx, path=WEIGHTS, max_batch=64):
        z = np.load(path)
        return cls(ctx, tuple(int(d) for d in z["D"]), max_batch, params=z["params"], gain=float(z["gain"]))


def _range(E, nF):
    nF = nF if nF is not None else (E.nF if E.has("nF") else None)
    if nF is None:
        return 0, 0
    nF = np.asarray(nF)
    return int(nF[0]), int(nF[-1]) + 1


def _dev_args(y, E, x, ctx):
    p = api._plan(E, ctx)
    yd, _ = api._dev(ctx, y, np.complex64)
    xd, _ = api._dev(ctx, x, np.complex64)
    Sd, _ = api._dev(ctx, E.Sf, np.complex64)
    Cn = Sd.shape[3] if len(Sd.shape) > 3 else 1
    Tf = np.asfortranarray(np.asarray(E.Tr, np.float32))
    return p, yd, xd, Sd, Cn, Tf


def state_energies(y, E, x, nF=None, ctx=None):
    """Per-state energy of the residual encode(T_s x) - y over the readout rows
    nF, normalised as LMsolver.m:82-83 does. Returns (n_states,) float64."""
    ctx = ctx or api.default_context()
    p, yd, xd, Sd, Cn, Tf = _dev_args(y, E, x, ctx)
    lo, hi = _range(E, nF)
    En = (C.c_double * max(p.n_mot, 1))()
    ctx.check(ctx.lib.disorder_state_energies(ctx.h, p.h, yd.ptr, Sd.ptr, Cn, xd.ptr, Tf.ctypes.data_as(_lib.FP),
                                              lo, hi, En))
    return np.array(En[:p.n_mot])


def backproject_states(y, E, x, nF=None, ctx=None):
    """Per-state adjoint of the residual, T_s^H sum_c S_c^H F^H (E_s x - y_s):
    a device array (N1, N2, N3, n_states)."""
    ctx = ctx or api.default_context()
    p, yd, xd, Sd, Cn, Tf = _dev_args(y, E, x, ctx)
    lo, hi = _range(E, nF)
    out = ctx.empty(tuple(p.N) + (p.n_mot,))
    ctx.check(ctx.lib.disorder_backproject_states(ctx.h, p.h, yd.ptr, Sd.ptr, Cn, xd.ptr,
                                                  Tf.ctypes.data_as(_lib.FP), lo, hi, out.ptr))
    return out


def restrict(T):
    """Methods/restrictTransform.m:28-32: rotations wrapped to (-pi, pi]."""
    T = np.array(T, np.float32)
    T[:, 3:] = np.float32(np.angle(np.exp(1j * T[:, 3:].astype(np.float64))))
    return T


def propose_step(net, y, E, x, nF=None, ctx=None, refresh=None):
    """One proposal round for the states not yet converged: returns (E with
    the accepted proposals applied to Tr, accepted mask). A proposal is kept
    only where it lowers the state's energy. The energies are compared at the
    current image x, or, with refresh = (EH, A) of the image update, at x
    refreshed by one CG iteration (CGsolver.m) with the proposed motion: the
    current image is a blur of all shots' poses, which favours the average
    pose over each shot's own."""
    ctx = ctx or net.ctx
    act = ~np.asarray(E.cT, bool)
    if not act.any():
        return E, np.zeros_like(act)
    dT = net.propose(y, E, x, nF)
    T0 = np.asarray(E.Tr, np.float32)
    T1 = T0.copy()
    T1[act] = T0[act] + dT[act]
    T1 = restrict(T1)
    xg = x
    if refresh is not None:
        EH, A = refresh
        xg = ctx.empty(x.shape)
        ctx.check(ctx.lib.disorder_memcpy_d2d(ctx.h, xg.ptr, x.ptr, x.nbytes))
        xg, _, _ = api.CGsolver(y, E.copy(Tr=T1), EH, A, None, None, xg, 1, "RelativeResidual2Error", 0.0, ctx=ctx)
    En0 = state_energies(y, E, xg, nF, ctx=ctx)
    En1 = state_energies(y, E.copy(Tr=T1), xg, nF, ctx=ctx)
    acc = act & (En1 < En0)
    T = T0.copy()
    T[acc] = T1[acc]
    return E.copy(Tr=T), acc


# ---------------------------------------------------------------- training data
LEVEL_N = (64, 64, 44)
FULL_N = (256, 256, 176)


def simulate_level(ctx, rng, N=LEVEL_N, N_full=FULL_N, n_shots=64, n_coils=16, max_deg=8.0, max_vox=8.0,
                   snr_db=25.0, n_ellipsoids=40, redFOV=1.0 / 3):
    """One simulated scan on the coarsest pyramid level's grid (translations
    in voxels of the full grid N_full, as the driver's T): phantom, coils,
    random-checkered shots, motion U(-max_deg, max_deg) deg and
    U(-max_vox, max_vox) voxels, noisy samples. Returns a Struct with x_gt
    (host), y (device), E (true motion in Tr), the readout rows nF and the
    preconditioner Se."""
    xh = synth.phantom(N, n_ellipsoids, rng)
    xh = (xh / np.linalg.norm(xh.ravel())).astype(np.complex64)
    Sh = synth.coil_maps(N, n_coils, rng)
    sigma = synth.snr_to_sigma(snr_db, xh, Sh)
    H = synth.random_checkered(N[:2], n_shots, rng)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, n_shots)
    T_true = synth.motion(n_shots, max_deg, max_vox, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = api.generateTransformGrids(N_full, N, cent, sh=1)
    Sd = ctx.upload(Sh)
    nF = np.arange(0, int(math.floor((1 - redFOV) * N[2])))
    E = api.Struct(Tr=T_true, NMs=n_shots, NSe=n_shots + 1, Sf=Sd, grids=grids, ky=ky, kz=kz, nEc=nEc, mSt=mSt,
                   nF=nF)
    y = api.encode(ctx.upload(xh), E, ctx=ctx)
    y = ctx.upload(synth.add_noise(y.numpy(), sigma, int(rng.integers(1 << 30))))
    Mbe = ctx.upload(np.isin(np.arange(N[2]), nF).astype(np.float32))
    return api.Struct(x_gt=xh, y=y, E=E, nF=nF, Se=api.precondition_weights(Sd, 1e-9, ctx=ctx), Mbe=Mbe,
                      N=tuple(N), N_full=tuple(N_full), T_true=T_true)


def simulate_shots(ctx, rng, **kw):
    """One simulated scan and its training shots: the per-state
    back-projections of the residual at a current estimate (no motion, as in
    the first outer iteration, or the truth minus a mean-free error of random
    size; the image from 1-5 CG iterations at that motion). Returns
    (features device (N + (n_shots,)), image x device (N), 1/rms(x), targets
    (n_shots, 6) in network units)."""
    sim = simulate_level(ctx, rng, **kw)
    E, T_true, N = sim.E, sim.T_true, sim.N
    n_shots = T_true.shape[0]
    if rng.random() < 0.5:
        T_cur = np.zeros_like(T_true)
    else:
        a = rng.uniform(0.1, 1.0)
        err = synth.motion(n_shots, a * kw.get("max_deg", 8.0), a * kw.get("max_vox", 8.0), rng)
        T_cur = restrict(T_true - err)
    Ec = E.copy(Tr=T_cur)
    n_cg = int(rng.choice([1, 2, 3, 5]))
    x_cur, _, _ = api.CGsolver(sim.y, Ec, api.Struct(Mbe=sim.Mbe), api.Struct(Se=sim.Se), None, None, None, n_cg,
                               "RelativeResidual2Error", 0.0, ctx=ctx)
    feats = backproject_states(sim.y, Ec, x_cur, sim.nF, ctx=ctx)
    xv = x_cur.numpy()
    rms = float(np.sqrt(np.mean(np.abs(xv) ** 2)))
    d = (T_true - T_cur).astype(np.float64)
    d[:, 3:] = np.angle(np.exp(1j * d[:, 3:])) / ROT_UNIT
    d[:, :3] *= np.asarray(N, float) / np.asarray(sim.N_full, float) / TRANS_UNIT  # full-grid -> level voxels
    return feats, x_cur, 1.0 / rms, d.astype(np.float32)


def motion_error(T, T_true):
    """Largest translation (full-grid voxels) and rotation (degrees) error
    after removing the common offset (the image absorbs a global pose)."""
    d = np.asarray(T, float) - np.asarray(T_true, float)
    d[:, 3:] = np.angle(np.exp(1j * d[:, 3:]))
    d -= d.mean(axis=0, keepdims=True)
    return float(np.abs(d[:, :3]).max()), float(np.degrees(np.abs(d[:, 3:]).max()))


def level_run(ctx, sim, net=None, n_outer=9, winit=1e-3, traLimXT=(0.05, 0.02), resIso=None, refresh=False):
    """Motion estimation on one level as the driver runs it (solveXT.m:379-388,
    431, 507): outer iterations of one CG iteration and one LM step, with
    the proposal round before the LM step when net is given. Returns a dict
    of per-iteration motion errors, LM state-steps, accepted proposals and
    the device time."""
    E0 = sim.E
    S = E0.NMs
    resIso = resIso if resIso is not None else math.sqrt(2) * float(np.asarray(sim.N_full)[0]) / sim.N[0]
    E = E0.copy(Tr=np.zeros((S, 6), np.float32), w=np.full(S, winit, np.float32), cT=np.zeros(S, bool),
                winit=winit, tL=list(np.asarray(traLimXT) * resIso))
    x = ctx.empty(sim.N)
    ctx.check(ctx.lib.disorder_memset(ctx.h, x.ptr, 0, x.nbytes))
    out = dict(err_vox=[], err_deg=[], lm_states=0, accepted=0, iters=0)
    nReset, cont = 0, 0
    ctx.synchronize()
    ctx.event(8)
    for n in range(n_outer):
        if nReset == 0 or cont % nReset == 0 or np.all(E.cT):
            nReset += 1
            cont = 0
            E.cT = np.zeros(S, bool)
        cont += 1
        x, _, _ = api.CGsolver(sim.y, E, api.Struct(Mbe=sim.Mbe), api.Struct(Se=sim.Se), None, None, x, 1,
                               "RelativeResidual2Error", 0.0, ctx=ctx)
        if net is not None:
            E, acc = propose_step(net, sim.y, E, x, sim.nF, ctx=ctx,
                                  refresh=(api.Struct(Mbe=sim.Mbe), api.Struct(Se=sim.Se)) if refresh else None)
            out["accepted"] += int(acc.sum())
        out["lm_states"] += int(np.sum(~np.asarray(E.cT, bool)))
        E = api.LMsolver(sim.y, E, x, ctx=ctx)
        ev, ed = motion_error(E.Tr, sim.T_true)
        out["err_vox"].append(ev)
        out["err_deg"].append(ed)
        out["iters"] = n + 1
        if np.all(E.cT):
            break
    ctx.event(9)
    out["time_s"] = ctx.elapsed_ms(8, 9) * 1e-3
    return out


def compare(ctx, net, n_scans=4, seed=9000, n_outer=9, max_deg=5.0, max_vox=5.0, refresh=False):
    """level_run with and without the proposal on n_scans simulated scans with
    config-2 motion (U(-5, 5) deg / voxels). Returns (plain runs, learned runs)."""
    rng = np.random.default_rng(seed)
    plain, learned = [], []
    for _ in range(n_scans):
        sim = simulate_level(ctx, rng, max_deg=max_deg, max_vox=max_vox)
        plain.append(level_run(ctx, sim, None, n_outer))
        learned.append(level_run(ctx, sim, net, n_outer, refresh=refresh))
    return plain, learned


def make_dataset(ctx, n_scans, seed, **kw):
    """n_scans simulated scans: a list of (features, image, 1/rms(image), targets)."""
    rng = np.random.default_rng(seed)
    return [simulate_shots(ctx, rng, **kw) for _ in range(n_scans)]


def calibrate_gain(ctx, data, net_D=LEVEL_N):
    """The feature gain that gives the training inputs unit RMS on average."""
    r = []
    for feats, _, sc, _ in data[:8]:
        v = feats.numpy()
        r.append(sc * float(np.sqrt(np.mean(np.abs(v) ** 2))))
    return 1.0 / float(np.median(r))


def train(ctx, net, data, epochs, lr=1e-3, seed=0, log=None, lr_end=1e-4, it0=0, total=None):
    """Adam over the scans (one scan's shots per batch), cosine learning rate
    from lr to lr_end over `total` steps (default: this call's), starting at
    step it0. Returns (mean training loss of each epoch, next step)."""
    rng = np.random.default_rng(seed)
    grad = ctx.empty((net.P,), np.float32)
    hist = []
    total = total if total is not None else epochs * len(data)
    it = it0
    tg = [ctx.upload(np.ascontiguousarray(t).T.copy(order="F")) for _, _, _, t in data]
    for ep in range(epochs):
        losses = []
        for j in rng.permutation(len(data)):
            feats, x, sc, t = data[j]
            B = t.shape[0]
            net.forward(feats, x, B, sc * net.gain, sc)
            losses.append(net.backward(tg[j], B, grad))
            f = min(it / max(total - 1, 1), 1.0)
            net.adam(grad, lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * f)))
            it += 1
        hist.append(float(np.mean(losses)))
        if log:
            log("epoch %d loss %.4f" % (ep, hist[-1]))
    return hist, it


def evaluate(net, data):
    """Mean loss of the network and of the zero proposal on data."""
    ln, lz = [], []
    for feats, x, sc, t in data:
        out = net.forward(feats, x, t.shape[0], sc * net.gain, sc)
        ln.append(np.sum((out - t) ** 2) / t.shape[0])
        lz.append(np.sum(t ** 2) / t.shape[0])
    return float(np.mean(ln)), float(np.mean(lz))


def main():
    """Train the proposal network on simulated shots and write its weights:
    python -m disorder_b200.proposal [--scans 320] [--rounds 1] [--epochs 16] [--out PATH]
    Each round simulates --scans fresh scans and trains --epochs on them; one
    cosine learning-rate schedule spans all rounds."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--scans", type=int, default=320)
    ap.add_argument("--rounds", type=int, default=1)
    ap.add_argument("--val", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=5000)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args()
    ctx = api.Context(0)
    val = make_dataset(ctx, a.val, a.seed + 1)
    net = MotionNet(ctx, LEVEL_N, 64, params=init_params(np.random.default_rng(a.seed)))
    total = a.rounds * a.epochs * a.scans
    it, hist, t_gen, t_train = 0, [], 0.0, 0.0
    for r in range(a.rounds):
        t0 = time.time()
        data = make_dataset(ctx, a.scans, a.seed if r == 0 else a.seed + 7919 * r)
        t_gen += time.time() - t0
        if r == 0:
            net.gain = calibrate_gain(ctx, data)
        print("round %d: %d training shots, gain %.4g" % (r, a.scans * 64, net.gain), flush=True)
        t0 = time.time()
        h, it = train(ctx, net, data, a.epochs, a.lr, seed=a.seed + r, log=lambda s: print(s, flush=True),
                      it0=it, total=total)
        t_train += time.time() - t0
        hist += h
        vl, vz = evaluate(net, val)
        print("round %d: validation loss %.4f (zero proposal %.4f)" % (r, vl, vz), flush=True)
        del data
    print("simulated %d shots in %.1f s, trained in %.1f s; validation loss %.4f (zero proposal %.4f)"
          % (a.rounds * a.scans * 64, t_gen, t_train, vl, vz), flush=True)
    net.save(a.out, meta=dict(train_loss=np.array(hist), val_loss=np.float64(vl), val_zero=np.float64(vz),
                              scans=np.int64(a.scans * a.rounds), epochs=np.int64(a.epochs),
                              rounds=np.int64(a.rounds), seed=np.int64(a.seed)))


if __name__ == "__main__":
    main()
