"""The kernel variants of one operation agree: the TMA tile-copy passes (and
the TMA gather / scatter of encode and decode), the
cp.async-pipelined passes (DISORDER_NO_TMA=1), the one-tile-per-CTA
kernels (DISORDER_NO_PIPE=1), and the sample-sum coil stage against the
three-pass one (DISORDER_SUM_COIL=1) compute the same arithmetic with
different data movement, so the sinc rigid transform and the encoding
operators must match to rounding. The environment switches are read once per
process, so each variant runs in a child process."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, math, numpy as np
sys.path.insert(0, sys.argv[1])
import disorder_b200 as db
from disorder_b200 import synth
out = sys.argv[2]
N, S, C = (96, 128, 44), 8, 3
rng = np.random.default_rng(7)
ctx = db.Context(0)
x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
T = synth.motion(S, 6, 3, rng)
cent = [math.ceil((n + 1) / 2.0) for n in N]
g = db.generateTransformGrids(N, N, cent)
et, _ = db.precomputeFactorsSincRigidTransform(g, T, 1)
fw, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
inv, _ = db.sincRigidTransform(fw, et, 0, sumR=1, ctx=ctx)
Sf = (rng.standard_normal(N + (C,)) + 1j * rng.standard_normal(N + (C,))).astype(np.complex64)
H = synth.random_checkered(N[:2], S, rng)
ky, kz, nEc, mSt, _ = synth.sample_lists(H, S)
E = db.Struct(Tr=T, NMs=S, NSe=S + 1, Sf=ctx.upload(Sf), grids=g, ky=ky, kz=kz, nEc=nEc, mSt=mSt)
we = rng.uniform(0.5, 1.5, int(nEc[-1])).astype(np.float32)
ed = db.encodedecode(x, E, db.Struct(We=we), ctx=ctx)
yy = db.encode(x, E, ctx=ctx)
mb = rng.uniform(0.0, 1.0, N[2]).astype(np.float32)
dd = db.decode(yy, db.Struct(We=we, Mb=mb), E, ctx=ctx)
ctx.synchronize()
np.savez(out, fw=fw, inv=inv, ed=ed, y=yy, dec=dd)
"""


def _run(tmp_path, name, env_extra):
    out = str(tmp_path / (name + ".npz"))
    env = dict(os.environ)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, out], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_tma_pipe_and_tile_kernels_agree(tmp_path):
    tma = _run(tmp_path, "tma", {})
    pipe = _run(tmp_path, "pipe", {"DISORDER_NO_TMA": "1"})
    tile = _run(tmp_path, "tile", {"DISORDER_NO_PIPE": "1"})
    sums = _run(tmp_path, "sums", {"DISORDER_SUM_COIL": "1"})
    for k in ("fw", "inv", "ed", "y", "dec"):
        assert _rel(tma[k], pipe[k]) < 1e-6, k
        # the one-tile kernels read full phase tables (single-precision grid
        # products) where the pipelined ones use per-row seeds
        assert _rel(tma[k], tile[k]) < 1e-5, k
        # the dim-2 DFT of the coil stage as FFTs with a gather (three passes,
        # the default) or as per-tile sample sums: different summation orders
        assert _rel(tma[k], sums[k]) < 2e-6, k
