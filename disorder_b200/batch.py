"""Batched aligned reconstruction of many independent scans of uneven size.

The reference's only batching is memory blocking over motion states and coils
inside one scan (Reconstruction/encode.m:13-17,55,90; solveXT.m:194-195). Here
a whole batch of scans, each with its own matrix size, coil count and shot
count, is reconstructed on one GPU by K workers, each a library context with
its own CUDA stream driven by its own host thread (the library's calls release
the interpreter lock while they run, so the workers' launch sequences and
their host round trips interleave). Scans are handed out longest first (the
LPT rule on a cost model of voxels x shots x coils), so the batch ends
balanced.

Autotuning (tune()): for each worker count K in the candidate list and each
engine of the strided line passes (TMA bulk tensor copies, or cp.async
pipelines; disorder_ctx_set_tuning), a probe batch of the largest scans is
reconstructed and timed; the fastest setting is kept and reported.

The synthetic batch (uneven_specs) follows the simulation recipe of
disorder_b200.synth with per-scan sizes drawn from the given sets; shot counts
whose checkered tile does not divide the grid use the truncated-tile variant
of synth.random_checkered.
"""

import math
import queue
import threading
import time

import numpy as np

from . import api, recon, synth, synth_gpu

SIZES = (96, 128, 160, 192, 256)
COILS = (8, 16, 32)
SHOTS = (16, 32, 64, 96)


def uneven_specs(n_scans=32, seed=4000, sizes=SIZES, coils=COILS, shots=SHOTS):
    """Per-scan (N, coils, shots, seed): sizes drawn per axis, coil and shot
    counts drawn from their sets, with numpy.random.default_rng(seed); scan i
    is then synthesised from default_rng(seed + i)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scans):
        N = tuple(int(v) for v in rng.choice(sizes, 3))
        out.append({"N": N, "coils": int(rng.choice(coils)), "shots": int(rng.choice(shots)), "seed": seed + i})
    return out


def cost(spec):
    """Relative cost of one reconstruction (voxels x shots x kept coils)."""
    return float(np.prod(spec["N"])) * spec["shots"] * min(spec["coils"], 16)


class Scan:
    pass


def build(ctx, spec, rot_deg=5.0, trans_vox=5.0, snr_db=25.0, n_ell=40):
    """One synthetic scan on the device: phantom and coils from the library's
    generator kernels, a random-checkered sampling (truncated tiles where the
    tile does not divide the grid), uniform per-shot motion, samples
    y = encode(x_gt, T) + noise."""
    N, C, NS = tuple(spec["N"]), spec["coils"], spec["shots"]
    rng = np.random.default_rng(spec["seed"])
    sc = Scan()
    sc.spec = spec
    sc.N = N
    sc.x_gt = synth_gpu.phantom(ctx, N, n_ell, rng)
    sc.x_gt_host = sc.x_gt.numpy()
    sc.S = synth_gpu.coil_maps(ctx, N, C, rng)
    sc.H = synth.random_checkered(N[:2], NS, rng, truncate=True)
    ky, kz, nEc, mSt, _ = synth.sample_lists(sc.H, NS)
    sc.T_gt = synth.motion(NS, rot_deg, trans_vox, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    E = api.Struct(Tr=sc.T_gt, NMs=NS, NSe=NS + 1, Sf=sc.S, grids=api.generateTransformGrids(N, N, cent), ky=ky,
                   kz=kz, nEc=nEc, mSt=mSt)
    sc.y = api.encode(sc.x_gt, E, ctx=ctx)
    synth_gpu.add_noise(ctx, sc.y, synth_gpu.snr_sigma(snr_db, int(np.prod(N))), spec["seed"] + 7919)
    ctx.synchronize()
    return sc


def reconstruct(ctx, sc, perc=16, proposal=None):
    """One scan's aligned reconstruction (recon.aligned_reconstruction);
    returns (x, T, log)."""
    return recon.aligned_reconstruction(ctx, sc.S, sc.y, sc.H, sc.spec["shots"], sc.N, perc=perc, proposal=proposal)


class BatchRunner:
    """K worker contexts on one device, each with its own stream and host
    thread. precision: the contexts' tensor-core setting; tma: the strided
    pass engine (disorder_ctx_set_tuning)."""

    def __init__(self, workers=4, device=0, precision="fp32", tma=1):
        self.ctxs = [api.Context(device) for _ in range(workers)]
        self.configure(precision, tma)

    def configure(self, precision="fp32", tma=1):
        self.precision, self.tma = precision, int(tma)
        for c in self.ctxs:
            c.set_precision(precision)
            c.check(c.lib.disorder_ctx_set_tuning(c.h, 0, self.tma))

    def run(self, scans, workers=None, nrmse=True):
        """Reconstruct every scan (scans built on any of the contexts' device)
        with `workers` of the contexts (all by default). Returns a dict with
        the batch wall time, scans/s, per-scan seconds (start to end of its
        reconstruction on its worker), p50/p99 and per-scan NRMSE."""
        ctxs = self.ctxs[:workers] if workers else self.ctxs
        order = sorted(range(len(scans)), key=lambda i: -cost(scans[i].spec))
        q = queue.Queue()
        for i in order:
            q.put(i)
        per = [None] * len(scans)
        err = [None] * len(scans)
        fails = []

        def work(ctx):
            while True:
                try:
                    i = q.get_nowait()
                except queue.Empty:
                    return
                try:
                    t0 = time.perf_counter()
                    x, T, _ = reconstruct(ctx, scans[i])
                    ctx.synchronize()
                    per[i] = time.perf_counter() - t0
                    if nrmse:
                        xh = x.numpy()
                        g = scans[i].x_gt_host
                        err[i] = float(np.linalg.norm(xh - g) / np.linalg.norm(g))
                except Exception as e:  # noqa: BLE001 - reported, the batch carries on
                    fails.append((i, repr(e)))

        for c in ctxs:
            c.synchronize()
        t0 = time.perf_counter()
        th = [threading.Thread(target=work, args=(c,)) for c in ctxs]
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
        done = [p for p in per if p is not None]
        return {"wall_s": wall, "scans": len(scans), "workers": len(ctxs), "scans_per_s": len(done) / wall,
                "p50_s": float(np.percentile(done, 50)) if done else None,
                "p99_s": float(np.percentile(done, 99)) if done else None, "per_scan_s": per, "nrmse": err,
                "failures": fails, "precision": self.precision, "tma": self.tma}


def tune(runner, scans, worker_counts=(1, 2, 4), engines=(1, 0), probe=4):
    """Pick the worker count and strided-pass engine by reconstructing the
    `probe` costliest scans under each setting (one untimed warm-up pass of
    the probe first). Returns (best setting, all timings)."""
    big = sorted(scans, key=lambda s: -cost(s.spec))[:probe]
    runner.run(big, workers=max(worker_counts), nrmse=False)
    trials = []
    for tma in engines:
        runner.configure(runner.precision, tma)
        for k in worker_counts:
            if k > len(runner.ctxs):
                continue
            r = runner.run(big, workers=k, nrmse=False)
            trials.append({"workers": k, "tma": tma, "wall_s": r["wall_s"]})
    best = min(trials, key=lambda t: t["wall_s"])
    runner.configure(runner.precision, best["tma"])
    return best, trials
