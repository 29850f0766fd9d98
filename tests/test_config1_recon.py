"""The small aligned reconstruction end to end, on the GPU and in the FP64 oracle.

Scan: 64x64x64, 12 ellipsoids, 8 coils, 16 random-checkered shots (4x4
tiles), rotations U(-3,3) deg and translations U(-3,3) voxels, 30 dB SNR.
Schedule: 10 outer iterations of CGsolver (3 iterations) then LMsolver (1
iteration) from zero motion, the whole reconstruction at one resolution.
Both runs start from the same single-precision samples; after every stage the
image and the motion of the library are compared with the oracle's
(relative L2 error), and the convergence flags must agree. The per-stage
errors are printed.
"""

import json
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_SOLVER = 1e-4


def config1_scan(seed=1001):
    """The seeded scan and its samples y = encode(x_gt, T_gt) + noise, encoded
    by the oracle in FP64 and rounded to single precision."""
    from disorder_b200 import synth
    from oracle import encoding as oenc
    from oracle.encoding import Struct as OStruct
    from oracle.grids import generateTransformGrids as ogrids
    N, C, S = (64, 64, 64), 8, 16
    sc = synth.make_scan(N, C, S, 3.0, 3.0, 30.0, 12, seed)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    Eo = OStruct(Tr=sc.T_gt, NMs=S, NSe=S + 1, Sf=sc.S.astype(np.complex128), ky=sc.ky, kz=sc.kz, nEc=sc.nEc,
                 mSt=sc.mSt, grids=ogrids(N, N, cent, sh=1), cent=cent)
    y = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
    y = synth.add_noise(y.astype(np.complex64), sc.sigma, sc.noise_seed)
    return sc, Eo, y


def test_small_aligned_reconstruction_matches_the_oracle():
    import disorder_b200 as db
    from disorder_b200 import recon
    from oracle import grids as og
    from oracle import solvers as osol
    og.WORKERS = os.cpu_count() or 1
    sc, Eo, y = config1_scan()
    ctx = db.Context(0)
    gpu, ora = [], []

    def rec_gpu(stage, n, x, E):
        gpu.append((stage, n, np.array(x.numpy()), np.array(E.Tr), np.array(E.cT)))

    def rec_ora(stage, n, x, E):
        ora.append((stage, n, np.array(x), np.array(E.Tr), np.array(E.cT)))

    S = ctx.upload(sc.S)
    yd = ctx.upload(y)
    recon.alternating_reconstruction(ctx, S, yd, sc.ky, sc.kz, sc.nEc, sc.mSt, sc.n_shots, sc.N, on_stage=rec_gpu)
    osol.alternating_reconstruction(y.astype(np.complex128), Eo, on_stage=rec_ora)
    assert len(gpu) == len(ora) == 20
    report = []
    for (st, n, xg, Tg, cg), (st2, n2, xo, To, co) in zip(gpu, ora):
        assert (st, n) == (st2, n2)
        ex = float(np.linalg.norm(xg - xo) / np.linalg.norm(xo))
        eT = float(np.linalg.norm(Tg - To) / max(np.linalg.norm(To), 1e-30)) if st == "lm" else 0.0
        nrmse = float(np.linalg.norm(xg - sc.x_gt) / np.linalg.norm(sc.x_gt))
        report.append({"stage": st, "outer": n, "x_rel_err": ex, "T_rel_err": eT, "nrmse_gpu": nrmse,
                       "nrmse_oracle": float(np.linalg.norm(xo - sc.x_gt) / np.linalg.norm(sc.x_gt))})
        assert np.array_equal(cg, co), (st, n)
    print("per-stage error vs the FP64 oracle:", json.dumps(report))
    for r in report:
        assert r["x_rel_err"] < TOL_SOLVER and r["T_rel_err"] < TOL_SOLVER, r
    # the reconstruction gets better than its first image
    assert report[-1]["nrmse_gpu"] < report[0]["nrmse_gpu"]
