"""The allocation-free sinc rigid transform (disorder_sinc_rigid_transform_static).

Callers that reserve their device memory up front and cannot let a library
call cudaMalloc use this entry point; its scratch lives in a static device
array of the library. This test calls it through the C ABI and checks it
against the regular entry point, which builds the same tables in the
context's workspace, on two calls in a row (the static array keeps the
previous call's contents, so the second call checks that nothing stale leaks
through). It sits in a file that pytest collects last and creates its own
context, so it passes alone in a fresh process and after the other tests.
"""

import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the FP32 tolerance of the other GPU parity tests


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_static_scratch_transform_matches_workspace_transform():
    import disorder_b200 as db
    from disorder_b200 import _lib

    ctx = db.Context(0)
    lib = ctx.lib
    N = (64, 64, 44)
    rng = np.random.default_rng(2024)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = db.generateTransformGrids(N, N, cent)
    plan = db.Plan(ctx, grids, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int64), 0)
    V = int(np.prod(N))
    free_before = None
    for call in range(2):
        S = 8 + 4 * call
        x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        T = np.zeros((S, 6), np.float32)
        T[:, :3] = rng.uniform(-4, 4, (S, 3))
        T[:, 3:] = np.radians(rng.uniform(-8, 8, (S, 3)))
        Tf = np.asfortranarray(T)
        xd = ctx.upload(x)
        out_ref = ctx.empty(N + (S,))
        out_st = ctx.empty(N + (S,))
        Tp = Tf.ctypes.data_as(_lib.FP)
        ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out_ref.ptr))
        ctx.synchronize()
        if call == 1:
            try:
                import torch
                free_before = torch.cuda.mem_get_info(0)[0]
            except Exception:
                free_before = None
        ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, out_st.ptr))
        ctx.synchronize()
        if call == 1 and free_before is not None:
            import torch
            assert free_before - torch.cuda.mem_get_info(0)[0] < (1 << 20)
        a, b = out_st.numpy(), out_ref.numpy()
        assert _rel(a, b) < TOL, call
        # inverse without the state sum, also against the regular entry point
        inv_ref = ctx.empty(N + (S,))
        inv_st = ctx.empty(N + (S,))
        ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, out_ref.ptr, S, Tp, S, 0, 0, 1, inv_ref.ptr))
        ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, out_ref.ptr, S, Tp, S, 0, 1, inv_st.ptr))
        ctx.synchronize()
        assert _rel(inv_st.numpy(), inv_ref.numpy()) < TOL, call
    # requests beyond the static limit fail cleanly
    Sbig = 300
    Tbig = np.zeros((Sbig, 6), np.float32, order="F")
    big = ctx.empty((1,))
    st = lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, big.ptr, 1, Tbig.ctypes.data_as(_lib.FP), Sbig, 1,
                                                  1, big.ptr)
    assert st == 1
    assert b"at most" in lib.disorder_last_error(ctx.h)
