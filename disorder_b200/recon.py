"""Aligned reconstruction driver (the caller of the hot path).

Follows the level / outer-iteration structure of Reconstruction/solveXT.m:
coil compression (:61), resolution pyramid (pyramidPlan, :38), per level the
Fourier-cropped image, coils and samples (downsampleOperators, :333-342),
then outer iterations of CGsolver (:431) and LMsolver (:507) with the
reference's motion-convergence resets (:379-388) and, once the motion has
converged or at the last level, a final CGsolver to the energy tolerance
(:414-425, nIt=300, 'Energy', tolerSolve). Before every image update the
motion states are binned by compressMotion (:392); from the levels with
leff >= 0 on, the image updates weight the shots by the outlier rejection
(:440-482). NIfTI output, the CS/shearlet reconstruction and the
Gibbs/B-spline filters of the reference driver are not part of this path.
"""

import json
import math
import os
import shutil
import time

import numpy as np

from . import api

# ---------------------------------------------------------------- checkpoints
CHECKPOINT_VERSION = 1


def save_state(path, meta, arrays):
    """Write a checkpoint directory: state.json (the scalars in `meta`, and
    for each array its file, dtype, shape and order) and one raw
    little-endian file per array in column-major order (readable by
    numpy.fromfile and MATLAB fread). The directory is replaced as a whole:
    the new state is written beside it and renamed into place."""
    tmp = path + ".tmp"
    shutil.rmtree(tmp, ignore_errors=True)
    os.makedirs(tmp)
    files = {}
    for name, a in arrays.items():
        if a is None:
            continue
        a = a.numpy() if hasattr(a, "numpy") else np.asarray(a)
        with open(os.path.join(tmp, name + ".raw"), "wb") as f:
            f.write(np.asfortranarray(a.astype(a.dtype.newbyteorder("<"))).tobytes(order="F"))
        files[name] = {"file": name + ".raw", "dtype": a.dtype.name, "shape": list(a.shape), "order": "F"}
    with open(os.path.join(tmp, "state.json"), "w") as f:
        json.dump(dict(meta, version=CHECKPOINT_VERSION, arrays=files), f, indent=1)
    old = path + ".old"
    shutil.rmtree(old, ignore_errors=True)
    if os.path.exists(path):
        os.rename(path, old)
    os.rename(tmp, path)
    shutil.rmtree(old, ignore_errors=True)


def load_state(path):
    """(meta, {name: array}) of a checkpoint written by save_state."""
    with open(os.path.join(path, "state.json")) as f:
        meta = json.load(f)
    if meta.get("version") != CHECKPOINT_VERSION:
        raise ValueError("checkpoint %s: version %r, expected %d" % (path, meta.get("version"), CHECKPOINT_VERSION))
    arrays = {}
    for name, d in meta["arrays"].items():
        a = np.fromfile(os.path.join(path, d["file"]), dtype=np.dtype(d["dtype"]).newbyteorder("<"))
        arrays[name] = a.reshape(d["shape"], order="F").astype(d["dtype"])
    return meta, arrays


def pyramidPlan(voxSiz, resolMax=4.0, NWend=1, accel=(1, 0)):
    """Methods/pyramidPlan.m:19-33. Returns (resPyr, L, estT, resIso)."""
    voxSiz = np.asarray(voxSiz, float)
    Lr = int(round(math.log2(max(resolMax / voxSiz.min(), 1)))) + 1
    resPyr = 1.0 / np.flip(2.0 ** np.arange(Lr))
    L = Lr + int(round(math.log2(NWend)))
    resPyr = np.concatenate([resPyr, np.ones(L - Lr)])
    estT = np.ones(L, int)
    estT[max(L - accel[0], 0):L] = 0
    resIso = math.sqrt(2) * (np.prod(voxSiz) ** (1 / 3)) / resPyr
    L = max(L - accel[1], 1)
    return resPyr[:L], L, estT[:L], resIso[:L]


def _signed(j, n):
    return ((j + n // 2) % n) - n // 2


def level_sampling(H, n_states, NYres):
    """Crop the DC-first shot map H to the central NYres frequencies (the
    k-space crop of resampling(A, NYres, 1), Methods/downsampleOperators.m:53)
    and list the level's samples as buildHarmonicSampling does. Returns (ky,
    kz, nEc, mSt, src) with src the row of every level sample in the
    full-resolution sample array."""
    N1, N2 = H.shape
    f1 = np.array([_signed(j, NYres[0]) % N1 for j in range(NYres[0])])
    f2 = np.array([_signed(j, NYres[1]) % N2 for j in range(NYres[1])])
    Hres = H[np.ix_(f1, f2)]
    full_lin = f1[:, None] + N1 * f2[None, :]
    Hf = Hres.reshape(-1, order="F")
    Lf = full_lin.reshape(-1, order="F")
    idx, seg = [], []
    for s in range(1, n_states + 2):
        ind = np.flatnonzero(Hf == (s % (n_states + 1)))
        idx.append(ind)
        seg.append(np.full(len(ind), s - 1, np.int32))
    lin = np.concatenate(idx)
    ky, kz = np.unravel_index(lin, Hres.shape, order="F")
    nEc = np.concatenate([[0], np.cumsum([len(i) for i in idx])]).astype(np.int64)
    # rows of the full-resolution sample array: its samples are the grid points
    # ordered by shot in the same way (H at full size)
    Hfull = H.reshape(-1, order="F")
    full_order = np.concatenate([np.flatnonzero(Hfull == (s % (n_states + 1))) for s in range(1, n_states + 2)])
    row_of = np.empty(H.size, np.int64)
    row_of[full_order] = np.arange(full_order.size)
    return ky.astype(np.int32), kz.astype(np.int32), nEc, np.concatenate(seg), row_of[Lf[lin]]


def _haar_dec(x, levels):
    """Multi-level orthonormal Haar decomposition with half-point symmetric
    extension at odd lengths (the pair (x[n-1], x[n-1])): returns the
    coefficient list [a_L, d_L, ..., d_1] and the length of each level."""
    a = np.asarray(x, np.float64)
    details, lengths = [], [a.size]
    s = math.sqrt(0.5)
    for _ in range(levels):
        if a.size % 2:
            a = np.append(a, a[-1])
        details.append((a[0::2] - a[1::2]) * s)
        a = (a[0::2] + a[1::2]) * s
        lengths.append(a.size)
    return [a] + details[::-1], lengths


def _haar_rec(coefs, lengths):
    s = math.sqrt(0.5)
    a = coefs[0]
    for j, d in enumerate(coefs[1:]):
        x = np.empty(2 * a.size)
        x[0::2] = (a + d) * s
        x[1::2] = (a - d) * s
        a = x[:lengths[-2 - j]]
    return a


def compressMotion(T, nEc, res, traLimX=(0.05, 0.02)):
    """Methods/compressMotion.m:19-80: bin the motion states for the image
    update. Each parameter's trajectory over the states is Haar-decomposed
    (floor(log2(n)) levels, :30-33), coefficients below the binning limit
    (traLimX(1)*res voxels, traLimX(2)*res degrees, :32) are zeroed, and the
    trajectory is rebuilt (:34-35). Runs of consecutive states whose rebuilt
    transforms agree to 1e-6 form one bin (:40-53) with the mean transform
    (:56-65); their samples, consecutive already, form one segment. The outer
    segments follow unchanged (:66-72).
    T: (n, 6); nEc: offsets of the n motion segments then the outer ones.
    Returns (T_bins (nb, 6) float32, nEc of the bins then the outer
    segments, bin of each state)."""
    T = np.asarray(T, np.float64)
    n = T.shape[0]
    nEc = np.asarray(nEc, np.int64)
    if n <= 1:
        return T.astype(np.float32), nEc.copy(), np.zeros(n, np.int64)
    levels = int(math.floor(math.log2(n)))
    Test = np.empty_like(T)
    for m in range(6):
        th = traLimX[0] * res if m < 3 else math.radians(traLimX[1] * res)
        C, L = _haar_dec(T[:, m], levels)
        C = [np.where(np.abs(c) < th, 0.0, c) for c in C]
        Test[:, m] = _haar_rec(C, L)
    bins = np.zeros(n, np.int64)
    starts = [0]
    for s in range(1, n):
        if np.any(np.abs(Test[s] - Test[starts[-1]]) > 1e-6):
            starts.append(s)
        bins[s] = len(starts) - 1
    starts.append(n)
    Tb = np.stack([Test[a:b].mean(axis=0) for a, b in zip(starts[:-1], starts[1:])])
    off = np.concatenate([nEc[starts], nEc[n + 1:]])
    return Tb.astype(np.float32), off, bins


def binned(E, res, traLimX=(0.05, 0.02)):
    """E with its motion states binned by compressMotion (solveXT.m:392): the
    structure for the image update; the motion update keeps E itself
    (solveXT.m:495)."""
    Tb, off, _ = compressMotion(E.Tr, E.nEc, res, traLimX)
    nb = Tb.shape[0]
    if nb == E.NMs:
        return E.copy(Tr=Tb)
    mSt = np.repeat(np.arange(len(off) - 1, dtype=np.int32), np.diff(off))
    return E.copy(Tr=Tb, NMs=nb, NSe=len(off) - 1, nEc=off, mSt=mSt, plan_cache=None)


def outlier_weights(Re, sweeps, n_sweeps, leff, percRobustShot=(0.125, 0.25), enerRobustShot=0.95):
    """Shot weights of the outlier rejection (Reconstruction/solveXT.m:447-466).
    Re: per-sample residual energies (computeEnergy with avdi=1); sweeps: the
    shot of every sample (n_sweeps and above: outer samples, ignored).
    Percentiles of each shot's log residuals (MATLAB prctile, the midpoint
    rule) are standardised by a robust spread taken from the lower
    percentiles across shots; a shot's weight is the tail probability of its
    mean score over (1 - enerRobustShot) / n_sweeps, capped at 1."""
    from statistics import NormalDist
    nd = NormalDist()
    Re = np.maximum(np.asarray(Re, np.float64), np.finfo(np.float64).tiny)
    sweeps = np.asarray(sweeps)
    lo, hi = (0.15, 0.85) if leff > 0 else (0.3, 0.7)
    percUse = 100 * np.round(np.arange(lo, hi + 1e-9, 0.05), 10)
    WeO = np.zeros((n_sweeps, percUse.size))
    for s in range(n_sweeps):
        v = np.log(Re[sweeps == s])
        WeO[s] = np.percentile(v, percUse, method="hazen") if v.size else 0.0
    pr = np.asarray(percRobustShot, np.float64)
    q = np.percentile(WeO, 100 * pr, axis=0, method="hazen")
    Westd = (q[1] - q[0]) / (nd.inv_cdf(pr[1]) - nd.inv_cdf(pr[0]))
    pm = float(pr.mean())
    # the centre sits -norminv(pm) spreads above the pm-th percentile; the
    # reference adds sqrt(2)*erfcinv(2*pm)*Westd, the same quantity (:462)
    Wmea = np.percentile(WeO, 100 * pm, axis=0, method="hazen") - Westd * nd.inv_cdf(pm)
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.mean((WeO - Wmea) / Westd, axis=1)
    z = np.where(np.isfinite(z), z, -np.inf)
    tail = np.array([1.0 - nd.cdf(v) if np.isfinite(v) else 1.0 for v in z])
    return np.minimum(tail / ((1.0 - enerRobustShot) / n_sweeps), 1.0)


def unsampled_states(nEc, n_states):
    """The motion states with no samples in a level's sampling (the check of
    Reconstruction/solveXT.m:355): any such state means the acquisition is
    probably not DISORDER, and the reference returns without correcting."""
    return np.flatnonzero(np.diff(np.asarray(nEc, np.int64))[:n_states] == 0)


def _sample_weights(We_shot, mSt, n_states):
    """Per-sample EH.We from shot weights; outer samples keep 1 (solveXT.m:480-481)."""
    w = np.ones(len(mSt), np.float32)
    inner = np.asarray(mSt) < n_states
    w[inner] = np.asarray(We_shot)[np.asarray(mSt)[inner]]
    return w


def _uncorrected(ctx, S, y, H, n_states, N, tolerSolve):
    """CGsolver at zero motion and full resolution to the energy tolerance
    (solveXT.m:243), preconditioned by A.Se (solveXT.m:231-233)."""
    ky, kz, nEc, mSt, _ = level_sampling(H, n_states, N[:2])
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    E = api.Struct(Tr=np.zeros((n_states, 6), np.float32), NMs=n_states, NSe=n_states + 1, Sf=S,
                   grids=api.generateTransformGrids(N, N, cent, sh=1), ky=ky, kz=kz, nEc=nEc, mSt=mSt)
    A = api.Struct(Se=api.precondition_weights(S, 1e-9, ctx=ctx))
    x, _, _ = api.CGsolver(y, E, None, A, None, None, None, 300, "Energy", tolerSolve, ctx=ctx)
    return x


class ReconLog:
    """The structured log of a reconstruction: one event per step (cg, lm,
    proposal, outliers, compress, resume, stopped, abort) with its level,
    outer iteration, step figures (CG iterations, LM energy and unconverged
    states, proposals kept, shots down-weighted) and the host time since the
    start (the solver calls synchronise, so it includes their device time).
    The figures the reference prints (CGsolver.m:88,102, LMsolver.m:198,
    210-212) as JSON lines instead."""

    def __init__(self, path=None):
        self.events = []
        self.t0 = time.perf_counter()
        self.path = path  # when set, every event is appended to this file as one JSON line

    def add(self, **kw):
        kw["t"] = time.perf_counter() - self.t0
        self.events.append(kw)
        if self.path:
            with open(self.path, "a") as f:
                f.write(json.dumps(kw, default=_json_default) + "\n")


def _json_default(v):
    if isinstance(v, np.generic):
        return v.item()
    if isinstance(v, np.ndarray):
        return v.tolist()
    raise TypeError("%r is not JSON serialisable" % type(v))


def reset_schedule():
    """The motion-convergence resets of solveXT.m:379-384 as a closure: call
    it at the start of every outer iteration with the current convergence
    flags; it returns True when they are to be cleared."""
    st = {"nReset": 0, "cont": 0}

    def due(cT):
        reset = st["nReset"] == 0 or st["cont"] % st["nReset"] == 0 or bool(np.all(cT))
        if reset:
            st["nReset"] += 1
            st["cont"] = 0
        st["cont"] += 1
        return reset

    return due


def alternating_reconstruction(ctx, S, y, ky, kz, nEc, mSt, n_states, N, n_outer=10, n_cg=3, n_lm=1, winit=1e-3,
                               tL=(0.05, 0.02), reg=1e-9, log=None, on_stage=None):
    """Aligned reconstruction at one resolution with a fixed schedule (the
    small simulation case): n_outer times an image update by CGsolver, n_cg
    iterations from the current image with the preconditioner
    A.Se = 1 / (sum_c |S_c|^2 + reg) (solveXT.m:231-233,431), then a motion
    update by n_lm LMsolver iterations (solveXT.m:507), with the
    motion-convergence resets of solveXT.m:379-384.

    S: coil maps (N1,N2,N3,C) device array; y: samples (Ns,N3,C) ordered by
    segment as (ky, kz, nEc, mSt) list them; n_states motion states, then the
    outer segment. on_stage(stage, n, x, E) is called after every update
    ("cg" or "lm", outer iteration n). Returns (x device volume, T, log)."""
    log = log if log is not None else ReconLog()
    N = tuple(int(n) for n in N)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = api.generateTransformGrids(N, N, cent, sh=1)
    x = ctx.empty(N)
    ctx.check(ctx.lib.disorder_memset(ctx.h, x.ptr, 0, x.nbytes))
    E = api.Struct(Tr=np.zeros((n_states, 6), np.float32), NMs=n_states, NSe=len(nEc) - 1, Sf=S, grids=grids,
                   ky=ky, kz=kz, nEc=nEc, mSt=mSt, w=np.full(n_states, winit, np.float32),
                   cT=np.zeros(n_states, bool), winit=winit, tL=list(tL))
    A = api.Struct(Se=api.precondition_weights(S, reg, ctx=ctx))
    due = reset_schedule()
    for n in range(n_outer):
        if due(E.cT):
            E.cT = np.zeros(n_states, bool)
        x, _, nn = api.CGsolver(y, E, None, A, None, None, x, n_cg, "RelativeResidual2Error", 0.0, ctx=ctx)
        log.add(step="cg", level=0, it=n, iters=nn, states=n_states)
        if on_stage:
            on_stage("cg", n, x, E)
        for _ in range(n_lm):
            E = api.LMsolver(y, E, x, ctx=ctx)
        log.add(step="lm", level=0, it=n, unconverged=int(np.sum(~E.cT)), energy=float(np.sum(E.En)))
        if on_stage:
            on_stage("lm", n, x, E)
    return x, E.Tr, log


def aligned_reconstruction(ctx, S, y, H, n_states, N, voxSiz=(1.0, 1.0, 1.0), perc=16, resolMax=4.0,
                           nExtern=20, winit=1e-3, traLimXT=(0.05, 0.02), redFOV=1.0 / 3, echoesMin=4,
                           tolerSolve=1e-3, log=None, proposal=None, levels=None, traLimX=(0.05, 0.02), outliers=True,
                           checkpoint=None, resume=False, stop_after=None):
    """Motion-corrected reconstruction of one scan on the GPU.

    S: coil maps (N1,N2,N3,C) device array; y: samples (Ns,N3,C) device array
    on the full k-space grid, ordered by shot as sample_lists(H) orders them
    (unitary DFT along the phase encodes, image space along the readout); H:
    (N1,N2) shot map, 1-based, DC first. perc: coil compression (count if >= 1,
    energy share if < 1). proposal: a proposal.MotionNet; at the motion levels
    whose grid is its input size, each outer iteration first offers its
    proposals and keeps those that lower a state's energy, then runs the LM
    step from there (no counterpart in the reference). levels: run only
    the first levels of the pyramid. traLimX: motion binning limits of the
    image update (compressMotion; None: no binning). outliers: the shot
    weights of the outlier rejection (rec.Alg.AlignedRec=2, solveXT.m:440-482),
    computed after each image update at the levels with leff >= 0 and applied
    to the later image updates of that level and to the final one.
    checkpoint: a directory that holds the latest state (save_state): after
    every outer iteration of a level its image, motion, LM damping and
    convergence flags, reset counters and shot weights; after every level
    the full-size image. resume: continue from that state (the result is the
    one the run without a stop gives). stop_after = (level, iteration) returns
    right after the checkpoint of that outer iteration, or of the end of the
    level when iteration is None (a staged run, e.g. a job with a time limit).
    Returns (x device volume, T (n_states, 6), log).
    """
    log = log if log is not None else ReconLog()
    N = tuple(int(n) for n in N)
    # coil compression (solveXT.m:61)
    Sc, yc, Ck, _, _ = api.compressCoils(S, perc, y, ctx=ctx)
    log.add(step="compress", coils=Ck)
    resPyr, L, estT, resIso = pyramidPlan(voxSiz, resolMax, 1, (1, 0))
    ky_full = None
    x = ctx.empty(N)
    ctx.check(ctx.lib.disorder_memset(ctx.h, x.ptr, 0, x.nbytes))
    T = np.zeros((n_states, 6), np.float32)
    E = None
    n_coarse = int(np.sum(resPyr != 1))
    We_shot = None
    n_run = L if levels is None else min(L, levels)
    start_level, mid = 0, None  # mid: a checkpoint taken inside a level
    if checkpoint and resume and os.path.exists(os.path.join(checkpoint, "state.json")):
        meta, arr = load_state(checkpoint)
        if meta["N"] != list(N) or meta["n_states"] != n_states:
            raise ValueError("checkpoint %s holds a %s scan with %d states" % (checkpoint, meta["N"], meta["n_states"]))
        T = np.ascontiguousarray(arr["T"], np.float32)
        We_shot = arr.get("We")
        if meta["iteration"] is None:
            start_level = meta["level"] + 1
            x = ctx.upload(arr["x"])
        else:
            start_level, mid = meta["level"], (meta, arr)
        log.add(step="resume", level=meta["level"], it=meta["iteration"])

    def save(l, n, xs, E_=None, est_=None, nReset_=0, cont_=0):
        if not checkpoint:
            return
        meta = {"N": list(N), "n_states": n_states, "level": l, "iteration": n, "est": est_, "nReset": nReset_,
                "cont": cont_}
        arrays = {"x": xs, "T": T if E_ is None else E_.Tr, "We": We_shot}
        if E_ is not None:
            arrays["w"] = np.asarray(E_.w, np.float32)
            arrays["cT"] = np.asarray(E_.cT, np.uint8)
        save_state(checkpoint, meta, arrays)

    for l in range(start_level, n_run):
        leff = l + 1 - n_coarse  # solveXT.m:269
        NXres = tuple(int(math.ceil(n * resPyr[l])) for n in N)
        # level operators (downsampleOperators, solveXT.m:333-342)
        resumed = mid is not None and l == start_level
        xRes = ctx.upload(mid[1]["x"]) if resumed else api.resampling(x, NXres, ctx=ctx)
        SRes = api.resampling(Sc, NXres, ctx=ctx)
        ky, kz, nEc, mSt, src = level_sampling(H, n_states, NXres[:2])
        empty = unsampled_states(nEc, n_states)
        if empty.size:
            # "Probably not DISORDER, returning without performing
            # corrections" (solveXT.m:355): the result is the uncorrected
            # reconstruction of solveXT.m:243 (zero motion, full resolution)
            log.add(step="abort", level=l, states=[int(v) for v in empty],
                    reason="Probably not DISORDER: motion states without samples at this level")
            return _uncorrected(ctx, Sc, yc, H, n_states, N, tolerSolve), np.zeros((n_states, 6), np.float32), log
        scale = math.sqrt(NXres[0] / N[0] * NXres[1] / N[1])
        ysel = api.gather_samples(yc, src, scale, ctx=ctx)
        yRes = api.resampling(ysel, (len(src), NXres[2], Ck), ctx=ctx) if NXres[2] != N[2] else ysel
        cent = [math.ceil((n + 1) / 2.0) for n in NXres]
        grids = api.generateTransformGrids(N, NXres, cent, sh=1)
        Se = api.precondition_weights(SRes, 1e-9, ctx=ctx)
        # readout region for motion estimation and energy (solveXT.m:345-346)
        nF = np.arange(0, int(math.floor((1 - redFOV) * NXres[2])))
        Mbe = np.zeros(NXres[2], np.float32)
        Mbe[nF] = 1
        Mbe_d = ctx.upload(Mbe)
        nSa = np.diff(nEc)[:n_states]
        cT0 = np.zeros(n_states, bool)
        if estT[l]:
            cT0[nSa < echoesMin] = True
        E = api.Struct(Tr=T, NMs=n_states, NSe=n_states + 1, Sf=SRes, grids=grids, ky=ky, kz=kz, nEc=nEc,
                       mSt=mSt, w=np.full(n_states, winit, np.float32), cT=cT0.copy(), winit=winit,
                       tL=list(np.asarray(traLimXT) * resIso[l]), nF=nF)
        EH = api.Struct(Mbe=Mbe_d)
        if not estT[l] and leff > 0 and We_shot is not None and np.any(We_shot < 1):
            # soft shot weights in the final image update (solveXT.m:411-415)
            EH = api.Struct(Mbe=Mbe_d, We=_sample_weights(We_shot, mSt, n_states))
        A = api.Struct(Se=Se)
        est = bool(estT[l])
        use_net = proposal is not None and est and tuple(NXres) == tuple(proposal.D)
        rres = None  # the sample residual of the image updates at the outlier levels
        nReset, cont, n0 = 0, 0, 0
        if resumed:
            meta, arr = mid
            E.w = arr["w"].astype(np.float32)
            E.cT = arr["cT"].astype(bool)
            est, nReset, cont, n0 = bool(meta["est"]), int(meta["nReset"]), int(meta["cont"]), int(meta["iteration"])
            if outliers and leff >= 0 and l < n_run - 1 and We_shot is not None and np.any(We_shot < 1):
                EH = api.Struct(Mbe=Mbe_d, We=_sample_weights(We_shot, mSt, n_states))
        for n in range(n0, nExtern):
            if nReset == 0 or cont % nReset == 0 or np.all(E.cT):  # solveXT.m:379-384
                nReset += 1
                cont = 0
                E.cT = cT0.copy()
            cont += 1
            if est:
                nX, tolType, tol = 1, "RelativeResidual2Error", 0.0  # nIt(2)=1 at motion levels
            else:
                nX, tolType, tol = 300, "Energy", tolerSolve
            Ex = binned(E, resIso[-1], traLimX) if traLimX is not None else E  # solveXT.m:392
            detect = outliers and leff >= 0 and l < n_run - 1
            if detect and rres is None:
                rres = ctx.empty((int(nEc[-1]), NXres[2], Ck))
            xRes, EnX, nn = api.CGsolver(yRes, Ex, EH, A, None, None, xRes, nX, tolType, tol, ctx=ctx,
                                         residual=rres if detect else None)
            log.add(step="cg", level=l, it=n, iters=nn, tolType=tolType, states=int(Ex.NMs))
            if detect:
                # residual energy per sample and outlier detection after every
                # image update, the level's last one included (solveXT.m:440-466),
                # from the residual the image update leaves; the final level's
                # weights are not used again
                Re = api.residualSampleEnergies(rres, Ex, EH, ctx=ctx)
                We_shot = outlier_weights(Re, mSt, n_states, leff)
                log.add(step="outliers", level=l, it=n, rejected=int(np.sum(We_shot < 1)))
                # soft shot weights for the next image updates of this level (:478-482)
                EH = api.Struct(Mbe=Mbe_d, We=_sample_weights(We_shot, mSt, n_states)) if np.any(We_shot < 1) \
                    else api.Struct(Mbe=Mbe_d)
            if not est:
                break
            if use_net:
                # a proposal that lowers a state's energy moves that state's
                # motion; the LM step then runs from there for every state
                from .proposal import propose_step
                E, acc = propose_step(proposal, yRes, E, xRes, nF, ctx=ctx)
                log.add(step="proposal", level=l, it=n, accepted=int(acc.sum()))
            n_lm = int(np.sum(~np.asarray(E.cT, bool)))
            E = api.LMsolver(yRes, E, xRes, ctx=ctx)
            T = E.Tr
            log.add(step="lm", level=l, it=n, unconverged=int(np.sum(~E.cT)), lm_states=n_lm,
                    energy=float(np.sum(E.En)))
            if np.all(E.cT):  # weak convergence (solveXT.m:530-534)
                est = False
            save(l, n + 1, xRes, E, est, nReset, cont)
            if stop_after is not None and tuple(stop_after) == (l, n):
                log.add(step="stopped", level=l, it=n)
                return api.resampling(xRes, N, ctx=ctx), T, log
        x = api.resampling(xRes, N, ctx=ctx)
        save(l, None, x)
        if stop_after is not None and tuple(stop_after) == (l, None):
            log.add(step="stopped", level=l)
            return x, T, log
    return x, T, log
