"""The allocation-free sinc rigid transform (disorder_sinc_rigid_transform_static).

Some callers cannot let a library call cudaMalloc in the middle of their
pipeline: an application that reserves its whole device-memory budget at
start-up and serves buffers from its own allocator, where an allocation can
fail once the budget is taken and synchronises the device. They use this entry
point, whose scratch lives in a static device array of the library that is
committed when the context is created.

Two checks, both through the C ABI:
- in a fresh process (a child started by the test, with eager module loading
  so that no kernel module loads mid-call) the first GPU work after the
  caller's own set-up is two static calls: the device's free memory and the
  context's workspace must not change, and only then is the result compared
  with the regular entry point;
- in this process, after whatever tests ran before, two calls in a row against
  the regular entry point (the array keeps the previous call's contents, so the
  second call checks that nothing stale leaks through), and the two size limits.
The file is collected last, so a run that stops at the first failure has run
every other test before it.
"""

import json
import math
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the FP32 tolerance of the other GPU parity tests
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def _setup(db, N):
    ctx = db.Context(0)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = db.generateTransformGrids(N, N, cent)
    plan = db.Plan(ctx, grids, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(1, np.int64), 0)
    return ctx, plan


def _motion(rng, S):
    T = np.zeros((S, 6), np.float32)
    T[:, :3] = rng.uniform(-4, 4, (S, 3))
    T[:, 3:] = np.radians(rng.uniform(-8, 8, (S, 3)))
    return np.asfortranarray(T)


# Runs in the child process: prints one JSON line.
_CHILD = r"""
import json, math, sys
import numpy as np
sys.path.insert(0, ROOT)
import torch
import disorder_b200 as db
from disorder_b200 import _lib
from tests.test_zz_no_alloc import _setup, _motion, _rel
N, S = (128, 128, 88), 40
ctx, plan = _setup(db, N)
lib = ctx.lib
rng = np.random.default_rng(77)
x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
T = _motion(rng, S)
Tp = T.ctypes.data_as(_lib.FP)
xd = ctx.upload(x)
fwd, inv = ctx.empty(N + (S,)), ctx.empty(N + (S,))
ctx.synchronize()
torch.cuda.mem_get_info(0)  # torch's own context set-up, before the reading
free0 = torch.cuda.mem_get_info(0)[0]
ws0 = lib.disorder_workspace_bytes(ctx.h)
ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, fwd.ptr))
ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, fwd.ptr, S, Tp, S, 0, 1, inv.ptr))
ctx.synchronize()
free1 = torch.cuda.mem_get_info(0)[0]
ws1 = lib.disorder_workspace_bytes(ctx.h)
ref_f, ref_i = ctx.empty(N + (S,)), ctx.empty(N + (S,))
ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, ref_f.ptr))
ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, ref_f.ptr, S, Tp, S, 0, 0, 1, ref_i.ptr))
ctx.synchronize()
print(json.dumps({"free_before": free0, "free_after": free1, "ws_before": ws0, "ws_after": ws1,
                  "ws_regular": lib.disorder_workspace_bytes(ctx.h),
                  "err_fwd": _rel(fwd.numpy(), ref_f.numpy()), "err_inv": _rel(inv.numpy(), ref_i.numpy())}))
"""


def test_static_call_allocates_nothing_in_a_fresh_process():
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    env.pop("DISORDER_POOL_RESERVE_GB", None)
    code = "ROOT = %r\n" % ROOT + _CHILD
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if not lines:
        pytest.skip("the child process could not measure free device memory: " + r.stderr[-500:])
    d = json.loads(lines[-1])
    # the static calls grew no workspace and took no device memory
    assert d["ws_after"] == d["ws_before"], d
    assert d["free_after"] == d["free_before"], d
    # (the regular entry point, run afterwards, does grow the workspace: the
    # check above would see a static path that used it)
    assert d["ws_regular"] > d["ws_after"], d
    assert d["err_fwd"] < TOL and d["err_inv"] < TOL, d


def test_static_scratch_transform_matches_workspace_transform():
    import disorder_b200 as db
    from disorder_b200 import _lib

    N = (64, 64, 44)
    ctx, plan = _setup(db, N)
    lib = ctx.lib
    rng = np.random.default_rng(2024)
    for call in range(2):
        S = 8 + 4 * call
        x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
        Tf = _motion(rng, S)
        Tp = Tf.ctypes.data_as(_lib.FP)
        xd = ctx.upload(x)
        out_ref, out_st = ctx.empty(N + (S,)), ctx.empty(N + (S,))
        ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, out_st.ptr))
        ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, xd.ptr, 1, Tp, S, 1, 1, 1, out_ref.ptr))
        ctx.synchronize()
        assert _rel(out_st.numpy(), out_ref.numpy()) < TOL, call
        # inverse without the state sum, also against the regular entry point
        inv_ref, inv_st = ctx.empty(N + (S,)), ctx.empty(N + (S,))
        ctx.check(lib.disorder_sinc_rigid_transform(ctx.h, plan.h, out_ref.ptr, S, Tp, S, 0, 0, 1, inv_ref.ptr))
        ctx.check(lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, out_ref.ptr, S, Tp, S, 0, 1, inv_st.ptr))
        ctx.synchronize()
        assert _rel(inv_st.numpy(), inv_ref.numpy()) < TOL, call
    big = ctx.empty((1,))
    # more states than the per-call limit
    Tbig = np.zeros((300, 6), np.float32, order="F")
    st = lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, big.ptr, 1, Tbig.ctypes.data_as(_lib.FP), 300, 1,
                                                  1, big.ptr)
    assert st == 1
    assert b"at most" in lib.disorder_last_error(ctx.h)
    # within the state limit, but the tables of 250 states at 64x64x44 (about
    # 39 MB) exceed the 32 MiB array
    T250 = np.zeros((250, 6), np.float32, order="F")
    st = lib.disorder_sinc_rigid_transform_static(ctx.h, plan.h, big.ptr, 1, T250.ctypes.data_as(_lib.FP), 250, 1,
                                                  1, big.ptr)
    assert st == 1
    assert b"bytes of scratch" in lib.disorder_last_error(ctx.h)
