"""Failure detection without a GPU fault.

Every failure here is made on the host or by a bounded wait that runs out:
- an unsupported structure field is rejected before any device work
  (disorder:UNSUPPORTED_FIELD, the gateway's MATLAB error);
- a sampling with an empty motion state is "probably not DISORDER"
  (Reconstruction/solveXT.m:355): the driver returns the uncorrected image;
- disorder_ctx_inject_fault arms one fault on a context: a TMA line pass that
  issues no tile loads, so its bounded waits run out with nothing in flight
  and disorder_synchronize reports DISORDER_TIMEOUT, or a workspace growth
  that fails as a failed cudaMalloc would (DISORDER_OOM); the context stays
  usable and the next call gives the right answer;
- non-finite samples make CG and LM stop with DISORDER_NONFINITE.
"""

import math

import numpy as np
import pytest


def _sequential_shots(N12, n_shots):
    """A non-DISORDER ordering: each shot is a contiguous band of ky rows
    (DC first), so the central crop of a coarse level misses whole shots."""
    H = np.zeros(N12, np.int32)
    rows = np.array_split(np.arange(N12[0]), n_shots)
    order = np.fft.ifftshift(np.arange(N12[0]))  # DC-first row of each centred row
    for s, r in enumerate(rows):
        H[order[r], :] = s + 1
    return H


def test_unsupported_field_is_rejected_before_device_work():
    import disorder_b200 as db
    from disorder_b200._lib import DisorderError
    E = db.Struct(Tr=np.zeros((2, 6), np.float32), NMs=2, NSe=2, Af=np.ones(3))
    with pytest.raises(DisorderError) as ei:
        db.api.encode(np.zeros((4, 4, 4), np.complex64), E, ctx=object())
    assert ei.value.status == 2 and "UNSUPPORTED_FIELD" in str(ei.value)
    with pytest.raises(DisorderError) as ei:
        db.api.decode(np.zeros((1, 4, 1), np.complex64), db.Struct(Fms=np.ones(2)), E, ctx=object())
    assert ei.value.status == 2


def test_unsampled_state_is_detected_at_a_coarse_level():
    from disorder_b200 import recon, synth
    n = 16
    H = _sequential_shots((64, 64), n)
    # full resolution: every shot has samples
    _, _, nEc, _, _ = recon.level_sampling(H, n, (64, 64))
    assert recon.unsampled_states(nEc, n).size == 0
    # the 16x16 centre holds only the central ky bands
    _, _, nEc, _, _ = recon.level_sampling(H, n, (16, 16))
    assert recon.unsampled_states(nEc, n).size > 0
    # a random-checkered sampling keeps every shot at the coarsest level
    Hd = synth.random_checkered((64, 64), n, np.random.default_rng(0))
    _, _, nEc, _, _ = recon.level_sampling(Hd, n, (16, 16))
    assert recon.unsampled_states(nEc, n).size == 0


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    return db.Context(0)


@pytest.mark.gpu
def test_tma_wait_that_runs_out_is_reported_and_the_context_recovers(ctx):
    import disorder_b200 as db
    from disorder_b200 import _lib, api, synth
    N, S = (64, 64, 44), 3
    rng = np.random.default_rng(12)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    T = np.asfortranarray(synth.motion(S, 5.0, 3.0, rng))
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    plan = api._transform_plan(ctx, db.generateTransformGrids(N, N, cent))
    xd, out = ctx.upload(x), ctx.empty(N + (S,))
    Tp = T.ctypes.data_as(_lib.FP)
    L = ctx.lib
    assert L.disorder_ctx_inject_fault(ctx.h, 1) == 0
    assert L.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out.ptr) == 0
    assert L.disorder_synchronize(ctx.h) == 5  # DISORDER_TIMEOUT
    assert b"ran out" in L.disorder_last_error(ctx.h)
    # the fault was one-shot and the context still works
    ctx.check(L.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out.ptr))
    assert L.disorder_synchronize(ctx.h) == 0
    et, _ = db.precomputeFactorsSincRigidTransform(db.generateTransformGrids(N, N, cent), T, 1)
    ref, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    assert np.array_equal(out.numpy(), ref)


@pytest.mark.gpu
def test_tensor_core_pass_wait_that_runs_out_is_reported(ctx):
    """The same injected fault on a tensor-core (BF16x3) line pass: its tile
    wait runs out before any MMA is issued, the kernel frees its tensor
    memory and stops, and the context gives the clean result afterwards."""
    import disorder_b200 as db
    from disorder_b200 import _lib, api, synth
    N, S = (16, 256, 16), 2  # 256-point strided lines: the tensor-core pass
    rng = np.random.default_rng(31)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    T = np.asfortranarray(synth.motion(S, 4.0, 2.0, rng))
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = db.generateTransformGrids(N, N, cent)
    plan = api._transform_plan(ctx, grids)
    xd, out = ctx.upload(x), ctx.empty(N + (S,))
    Tp = T.ctypes.data_as(_lib.FP)
    L = ctx.lib
    ctx.set_precision("bf16x3")
    try:
        assert L.disorder_ctx_inject_fault(ctx.h, 1) == 0
        assert L.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out.ptr) == 0
        assert L.disorder_synchronize(ctx.h) == 5  # DISORDER_TIMEOUT
        assert b"ran out" in L.disorder_last_error(ctx.h)
        ctx.check(L.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out.ptr))
        assert L.disorder_synchronize(ctx.h) == 0
        y1 = out.numpy()
        ctx.check(L.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out.ptr))
        assert L.disorder_synchronize(ctx.h) == 0
        y2 = out.numpy()
    finally:
        ctx.set_precision("fp32")
    assert np.array_equal(y1, y2)
    et, _ = db.precomputeFactorsSincRigidTransform(grids, T, 1)
    ref, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    err = np.linalg.norm(y1 - ref) / np.linalg.norm(ref)
    assert 1e-7 < err < 1e-4  # the BF16x3 result (not the FP32 one)


@pytest.mark.gpu
def test_injected_allocation_failure_returns_oom():
    import disorder_b200 as db
    from conftest import make_problem
    from disorder_b200._lib import DisorderError
    ctx = db.Context(0)  # fresh: its workspace has not grown yet
    N = (24, 20, 16)
    sc, Eo = make_problem(N=N, C=2, S=4, seed=3)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    E = db.Struct(Tr=sc.T_gt, NMs=4, NSe=5, Sf=ctx.upload(sc.S, np.complex64),
                  grids=db.generateTransformGrids(N, N, cent), ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    assert ctx.lib.disorder_ctx_inject_fault(ctx.h, 2) == 0
    with pytest.raises(DisorderError) as ei:
        db.encode(sc.x_gt, E, ctx=ctx)
    assert ei.value.status == 3 and "injected" in str(ei.value)
    y = db.encode(sc.x_gt, E, ctx=ctx)
    assert np.all(np.isfinite(y)) and np.linalg.norm(y) > 0


@pytest.mark.gpu
def test_nonfinite_samples_stop_the_solvers(ctx):
    import disorder_b200 as db
    from conftest import make_problem
    from disorder_b200._lib import DisorderError
    N = (16, 16, 12)
    sc, Eo = make_problem(N=N, C=2, S=4, seed=9)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    E = db.Struct(Tr=sc.T_gt, NMs=4, NSe=5, Sf=ctx.upload(sc.S, np.complex64),
                  grids=db.generateTransformGrids(N, N, cent), ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
    y = db.encode(sc.x_gt.astype(np.complex64), E, ctx=ctx)
    y[5, 3, 1] = np.nan
    with pytest.raises(DisorderError) as ei:
        db.CGsolver(y, E, None, None, None, None, None, 3, "RelativeResidual2Error", 0.0, ctx=ctx)
    assert ei.value.status == 6
    El = E.copy(Tr=np.zeros_like(sc.T_gt), cT=np.zeros(4, bool), w=np.full(4, 1e-3, np.float32), winit=1e-3,
                tL=[0.05, 0.02])
    with pytest.raises(DisorderError) as ei:
        db.LMsolver(y, El, sc.x_gt, ctx=ctx)
    assert ei.value.status == 6


@pytest.mark.gpu
def test_reconstruction_of_a_non_disorder_sampling_returns_uncorrected(ctx):
    """A sequential shot ordering loses whole shots at the coarse levels: the
    driver returns the uncorrected reconstruction with zero motion."""
    import disorder_b200 as db
    from disorder_b200 import recon, synth
    N, n = (64, 64, 32), 16
    rng = np.random.default_rng(4)
    x = synth.phantom(N, 6, rng)
    x = (x / np.linalg.norm(x)).astype(np.complex64)
    Sm = synth.coil_maps(N, 4, rng)
    H = _sequential_shots(N[:2], n)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, n)
    cent = [math.ceil((v + 1) / 2.0) for v in N]
    Sd = ctx.upload(Sm)
    E = db.Struct(Tr=np.zeros((n, 6), np.float32), NMs=n, NSe=n + 1, Sf=Sd,
                  grids=db.generateTransformGrids(N, N, cent), ky=ky, kz=kz, nEc=nEc, mSt=mSt)
    y = db.encode(ctx.upload(x), E, ctx=ctx)
    xr, T, log = recon.aligned_reconstruction(ctx, Sd, y, H, n, N, perc=4)
    assert any(e["step"] == "abort" for e in log.events)
    assert not np.any(T)
    err = np.linalg.norm(xr.numpy() - x) / np.linalg.norm(x)
    assert err < 0.05  # noise-free, motion-free data: the uncorrected image is the image
