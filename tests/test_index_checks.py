"""Device index checks.

- Indices that come from the caller (disorder_gather_samples' row indices)
  are checked in every build: an index outside its array gives a zero row,
  disorder_synchronize reports BAD_ARG with the check's site, nothing is read
  out of bounds, and the context stays usable.
- The build with -DDISORDER_CHECKS (libdisorder_checks.so, loaded with
  DISORDER_LIB=checks) also checks the library's own sample indices; a child
  process runs encode, decode, encodedecode and CG through it against the
  FP64 oracle and requires no check to fire.
"""

import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_caller_index_outside_the_array_is_skipped_and_reported():
    import disorder_b200 as db
    ctx = db.Context(0)
    L = ctx.lib
    rng = np.random.default_rng(3)
    n_in, rows = 10, 3
    y = (rng.standard_normal((n_in, rows)) + 1j * rng.standard_normal((n_in, rows))).astype(np.complex64)
    yd = ctx.upload(y)
    idx = np.array([0, 5, n_in, 9, -1], np.int32)
    idd = ctx.upload(idx)
    out = ctx.empty((len(idx), rows))
    assert L.disorder_gather_samples(ctx.h, yd.ptr, n_in, rows, idd.ptr, len(idx), 2.0, out.ptr) == 0
    assert L.disorder_synchronize(ctx.h) == 1  # DISORDER_BAD_ARG
    assert b"index check failed (site 1)" in L.disorder_last_error(ctx.h)
    o = out.numpy()
    good = np.array([0, 1, 3])
    assert np.array_equal(o[good], 2.0 * y[idx[good]])
    assert not np.any(o[[2, 4]])
    # the report was cleared and the context works
    ok = ctx.upload(np.array([1, 2], np.int32))
    out2 = ctx.empty((2, rows))
    assert L.disorder_gather_samples(ctx.h, yd.ptr, n_in, rows, ok.ptr, 2, 1.0, out2.ptr) == 0
    assert L.disorder_synchronize(ctx.h) == 0
    assert np.array_equal(out2.numpy(), y[[1, 2]])


_CHILD = r"""
import math, sys
import numpy as np
sys.path.insert(0, ROOT)
import disorder_b200 as db
from disorder_b200 import _lib, synth
from oracle import encoding as oenc
from oracle.encoding import Struct as OStruct
from oracle.grids import generateTransformGrids as ogrids
assert _lib.LIB_PATH.endswith("libdisorder_checks.so"), _lib.LIB_PATH
N, C, S = (48, 48, 32), 4, 16
sc = synth.make_scan(N, C, S, 4.0, 2.0, 30.0, 8, seed=7)
cent = [math.ceil((n + 1) / 2.0) for n in N]
ctx = db.Context(0)
E = db.Struct(Tr=sc.T_gt, NMs=S, NSe=S + 1, Sf=ctx.upload(sc.S), grids=db.generateTransformGrids(N, N, cent),
              ky=sc.ky, kz=sc.kz, nEc=sc.nEc, mSt=sc.mSt)
Eo = OStruct(Tr=sc.T_gt, NMs=S, NSe=S + 1, Sf=sc.S.astype(np.complex128), ky=sc.ky, kz=sc.kz, nEc=sc.nEc,
             mSt=sc.mSt, grids=ogrids(N, N, cent, sh=1))
rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
we = np.random.default_rng(2).uniform(0.5, 1.5, sc.ky.size).astype(np.float32)
y = db.encode(sc.x_gt, E, ctx=ctx)
yo = oenc.encode(sc.x_gt.astype(np.complex128), Eo)
d = db.decode(y, db.Struct(We=we), E, ctx=ctx)
do = oenc.decode(y.astype(np.complex128), Eo.__class__(We=we.astype(np.float64)), Eo)
ed = db.encodedecode(sc.x_gt, E, db.Struct(We=we), ctx=ctx)
edo = oenc.decode(yo * we.astype(np.float64)[:, None, None], None, Eo)
xc, _, nn = db.CGsolver(y, E, None, None, None, None, None, 2, "RelativeResidual2Error", 0.0, ctx=ctx)
st = ctx.lib.disorder_synchronize(ctx.h)
print("checks build: encode %.2e decode %.2e encodedecode %.2e, synchronize %d" % (rel(y, yo), rel(d, do),
                                                                                    rel(ed, edo), st))
assert st == 0, ctx.lib.disorder_last_error(ctx.h)
assert rel(y, yo) < 1e-5 and rel(d, do) < 1e-5 and rel(ed, edo) < 1e-5 and nn == 2
"""


def test_checks_build_runs_the_operators_without_a_failed_check():
    lib = os.path.join(ROOT, "disorder_b200", "libdisorder_checks.so")
    if not os.path.exists(lib):
        pytest.skip("libdisorder_checks.so not built (python -m disorder_b200.build --debug)")
    env = dict(os.environ, DISORDER_LIB="checks")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + _CHILD], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "synchronize 0" in r.stdout
