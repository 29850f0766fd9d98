"""Checkpoint / resume of the reconstruction driver (recon.save_state,
load_state and aligned_reconstruction(checkpoint=..., resume=...,
stop_after=...)): the state files are raw little-endian column-major arrays
with a JSON header, and a run stopped after any outer iteration or level and
resumed gives the image and motion of the run without a stop, bit for bit."""

import json
import os

import numpy as np
import pytest


def test_state_files_round_trip_and_are_plain_raw(tmp_path):
    from disorder_b200 import recon
    rng = np.random.default_rng(0)
    x = (rng.standard_normal((5, 4, 3)) + 1j * rng.standard_normal((5, 4, 3))).astype(np.complex64)
    T = rng.standard_normal((7, 6)).astype(np.float32)
    cT = np.array([1, 0, 1, 1, 0, 0, 1], np.uint8)
    path = str(tmp_path / "ckpt")
    recon.save_state(path, {"level": 1, "iteration": 3, "est": True}, {"x": x, "T": T, "cT": cT, "We": None})
    meta, arr = recon.load_state(path)
    assert meta["level"] == 1 and meta["iteration"] == 3 and meta["est"] is True
    assert set(arr) == {"x", "T", "cT"}
    assert np.array_equal(arr["x"], x) and np.array_equal(arr["T"], T) and np.array_equal(arr["cT"], cT)
    # the raw file is the column-major little-endian array (what MATLAB fread reads)
    raw = np.fromfile(os.path.join(path, "T.raw"), "<f4")
    assert np.array_equal(raw, T.ravel(order="F"))
    with open(os.path.join(path, "state.json")) as f:
        assert json.load(f)["arrays"]["x"] == {"file": "x.raw", "dtype": "complex64", "shape": [5, 4, 3],
                                                 "order": "F"}
    # a second save replaces the state as a whole
    recon.save_state(path, {"level": 2, "iteration": None}, {"x": x[:2]})
    meta, arr = recon.load_state(path)
    assert meta["iteration"] is None and set(arr) == {"x"} and arr["x"].shape == (2, 4, 3)
    assert not os.path.exists(path + ".tmp") and not os.path.exists(path + ".old")


@pytest.mark.gpu
@pytest.mark.parametrize("stop", [(0, 1), (1, None)])
def test_staged_reconstruction_equals_the_uninterrupted_one(tmp_path, stop):
    import disorder_b200 as db
    from disorder_b200 import recon, synth
    N, C, S = (48, 48, 32), 6, 16
    rng = np.random.default_rng(8)
    x = synth.phantom(N, 8, rng)
    x = (x / np.linalg.norm(x)).astype(np.complex64)
    Sm = synth.coil_maps(N, C, rng)
    H = synth.random_checkered(N[:2], S, rng)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, S)
    T = synth.motion(S, 3.0, 3.0, rng)
    ctx = db.Context(0)
    Sd = ctx.upload(Sm)
    cent = [int(np.ceil((n + 1) / 2.0)) for n in N]
    E = db.Struct(Tr=T, NMs=S, NSe=S + 1, Sf=Sd, grids=db.generateTransformGrids(N, N, cent), ky=ky, kz=kz,
                  nEc=nEc, mSt=mSt)
    y = db.encode(ctx.upload(x), E, ctx=ctx)
    xa, Ta, _ = recon.aligned_reconstruction(ctx, Sd, y, H, S, N, perc=C)
    path = str(tmp_path / "ckpt")
    _, _, log1 = recon.aligned_reconstruction(ctx, Sd, y, H, S, N, perc=C, checkpoint=path, stop_after=stop)
    assert log1.events[-1]["step"] == "stopped"
    xb, Tb, log2 = recon.aligned_reconstruction(ctx, Sd, y, H, S, N, perc=C, checkpoint=path, resume=True)
    assert any(e["step"] == "resume" for e in log2.events)
    assert np.array_equal(Tb, Ta)
    assert np.array_equal(xb.numpy(), xa.numpy())


def test_log_events_as_json_lines(tmp_path):
    from disorder_b200 import recon
    path = str(tmp_path / "log.jsonl")
    log = recon.ReconLog(path)
    log.add(step="cg", level=0, it=1, iters=np.int64(3), energy=np.float32(2.5))
    log.add(step="lm", level=0, it=1, unconverged=4, states=[1, 2])
    lines = [json.loads(l) for l in open(path)]
    assert [l["step"] for l in lines] == ["cg", "lm"]
    assert lines[0]["iters"] == 3 and lines[0]["energy"] == 2.5 and lines[1]["states"] == [1, 2]
    assert lines[1]["t"] >= lines[0]["t"] >= 0
