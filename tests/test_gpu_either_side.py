"""Either side of the aligned reconstruction, on the GPU: a scan whose shot
map comes from the DISORDER trajectory generator (disorder_b200.sampling,
random-checkered, alternating zig-zag) is reconstructed by the driver, and
the image and motion are written with writeData and read back with readNII
(disorder_b200.nifti)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trajectory_to_reconstruction_to_nifti(tmp_path):
    import disorder_b200 as db
    from disorder_b200 import nifti, recon, sampling, synth
    N, C, S = (48, 48, 32), 6, 16
    rng = np.random.default_rng(21)
    x = synth.phantom(N, 8, rng)
    x = (x / np.linalg.norm(x)).astype(np.complex64)
    Sm = synth.coil_maps(N, C, rng)
    _, NP, _, _, Shot, _ = sampling.samplingDISORDER(sampling.cartesian_points(N[:2]), (4, 4), "RandomCheckered",
                                                     rng=np.random.default_rng(5))
    assert NP == N[0] * N[1] and Shot.min() == 1
    H = sampling.shot_map(Shot)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, S)
    T = synth.motion(S, 3.0, 3.0, rng)
    ctx = db.Context(0)
    Sd = ctx.upload(Sm)
    cent = [int(np.ceil((n + 1) / 2.0)) for n in N]
    E = db.Struct(Tr=T, NMs=S, NSe=S + 1, Sf=Sd, grids=db.generateTransformGrids(N, N, cent), ky=ky, kz=kz,
                  nEc=nEc, mSt=mSt)
    y = db.encode(ctx.upload(x), E, ctx=ctx)
    xr, Tr, log = recon.aligned_reconstruction(ctx, Sd, y, H, S, N, perc=C)
    assert not any(e["step"] == "abort" for e in log.events)
    # the motion-corrected image beats the uncorrected one (zero motion, solveXT.m:243)
    xu = recon._uncorrected(ctx, Sd, y, H, S, N, 1e-3)
    err = float(np.linalg.norm(xr.numpy() - x) / np.linalg.norm(x))
    err_u = float(np.linalg.norm(xu.numpy() - x) / np.linalg.norm(x))
    print("NRMSE corrected %.4f, uncorrected %.4f" % (err, err_u))
    assert np.isfinite(err) and err < 0.7 * err_u, (err, err_u)
    dat = str(tmp_path / "scan")
    nifti.writeData(dat, xr, Tr, np.diag([1.0, 1.0, 1.0, 1.0]))
    back, MS, _ = nifti.readNII(dat, ["Aq"])
    xh = xr.numpy()
    assert back[0].shape == N
    assert np.linalg.norm(back[0] - xh) / np.linalg.norm(xh) < 1e-6
    assert np.allclose(MS[0], [1.0, 1.0, 1.0])
