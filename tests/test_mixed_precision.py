"""The mixed-precision (tensor-core) contractions against the FP64 oracle.

BF16x3 and 3xTF32 split each operand into two tensor-core parts and keep
hi*hi + hi*lo + lo*hi in an FP32 accumulator (tcgen05 MMAs). Tolerances:
1e-4 relative for BF16x3 (about 16 significant bits per operand) and 1e-5
for 3xTF32 (about 21), the mixed-precision bar of the encoded k-space.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-4, "tf32x3": 1e-5}


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    c = db.Context(0)
    yield c
    c.set_precision("fp32")


@pytest.mark.parametrize("mode", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("N,Cin", [((24, 20, 16), 12), ((128, 128, 88), 32)])
def test_coil_compression_gram_on_tensor_cores(ctx, mode, N, Cin):
    """compressCoils (Methods/compressCoils.m:76-118) with its Gram matrix
    contracted on the tensor cores: the matrix (rebuilt from the returned
    eigenpairs), the kept coil count and subspace, and the compressed data."""
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle.prep import compressCoils
    rng = np.random.default_rng(Cin)
    S = synth.coil_maps(N, Cin, rng)
    S = S + 0.05 * (rng.standard_normal(S.shape) + 1j * rng.standard_normal(S.shape)).astype(np.complex64)
    ctx.set_precision(mode)
    try:
        So, _, C, D, U = db.compressCoils(S, 0.95, None, ctx=ctx)
    finally:
        ctx.set_precision("fp32")
    _, _, Co, Do, Uo, Po = compressCoils(S.astype(np.complex128), [0.95], None)
    P = (U * D[None, :]) @ U.conj().T
    assert rel(P, Po) < TOL[mode]
    assert C == Co[0]
    Pk = U[:, :C] @ U[:, :C].conj().T
    Pko = Uo[:, :C] @ Uo[:, :C].conj().T
    assert np.max(np.abs(Pk - Pko)) < 10 * TOL[mode]
    A = U[:, :C].conj().T
    assert rel(So, np.tensordot(S, A, axes=([3], [1]))) < 1e-5


@pytest.mark.parametrize("mode", ["bf16x3", "tf32x3"])
def test_transform_with_tensor_core_dft_passes(ctx, mode):
    """The sinc rigid transform at 256x256x176 with its strided line passes
    (256-point lines along dim 2, 176-point lines along dim 3) as tensor-core
    DFT GEMMs: forward to 2 states and the inverse with the state sum, against
    the FP64 oracle; the CUDA-core FFT result is printed beside it."""
    import math
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle.grids import generateTransformGrids as ogrids
    from oracle import grids as og
    from oracle.transform import precomputeFactorsSincRigidTransform as opf
    from oracle.transform import sincRigidTransform as ost
    import os
    og.WORKERS = os.cpu_count() or 1
    N, S = (256, 256, 176), 2
    rng = np.random.default_rng(77)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    T = synth.motion(S, 5.0, 5.0, rng)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    grids = db.generateTransformGrids(N, N, cent)
    et, _ = db.precomputeFactorsSincRigidTransform(grids, T, 1)
    eti, _ = db.precomputeFactorsSincRigidTransform(grids, T, 0)
    og_ = ogrids(N, N, cent, sh=1)
    yo = ost(x.astype(np.complex128).reshape(N + (1, 1)), opf(og_, T, 1, 0)[0], 1)[:, :, :, 0, :]
    u = (rng.standard_normal(N + (S,)) + 1j * rng.standard_normal(N + (S,))).astype(np.complex64)
    bo = ost(u.astype(np.complex128)[:, :, :, None, :], opf(og_, T, 0, 0)[0], 0, sumR=1)[:, :, :, 0, 0]
    yf, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
    ctx.set_precision(mode)
    try:
        y, _ = db.sincRigidTransform(x, et, 1, ctx=ctx)
        back, _ = db.sincRigidTransform(u, eti, 0, sumR=1, ctx=ctx)
    finally:
        ctx.set_precision("fp32")
    print("transform rel. err. vs FP64 oracle: %s %.2e (fp32 FFT %.2e), inverse %.2e"
          % (mode, rel(y, yo), rel(yf, yo), rel(back, bo)))
    assert rel(y, yo) < TOL[mode]
    assert rel(back, bo) < TOL[mode]


@pytest.mark.parametrize("mode", ["bf16x3", "tf32x3"])
def test_encode_with_tensor_core_dft_passes(ctx, mode):
    """encode (Reconstruction/encode.m) at 256x256x176, 16 coils, one state of
    a 64-shot sampling, with the transform's strided passes on the tensor
    cores: relative error of the encoded k-space against the FP64 oracle."""
    import math
    import os
    import disorder_b200 as db
    from disorder_b200 import synth
    from oracle import encoding as oenc
    from oracle import grids as og
    from oracle.encoding import Struct as OStruct
    from oracle.grids import generateTransformGrids as ogrids
    og.WORKERS = os.cpu_count() or 1
    N, C = (256, 256, 176), 16
    rng = np.random.default_rng(78)
    x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    Sm = (rng.standard_normal(N + (C,)) + 1j * rng.standard_normal(N + (C,))).astype(np.complex64)
    H = synth.random_checkered(N[:2], 64, rng)
    ky, kz, nEc, mSt, _ = synth.sample_lists(H, 64)
    n1 = int(nEc[1])
    # one state with a motion of its own (synth.motion removes the mean over
    # the shots, which for a single shot is the whole motion)
    T = np.array([[2.3, -1.7, 3.1, np.radians(4.0), np.radians(-3.0), np.radians(2.5)]], np.float32)
    cent = [math.ceil((n + 1) / 2.0) for n in N]
    Ed = db.Struct(Tr=T, NMs=1, NSe=1, Sf=ctx.upload(Sm), grids=db.generateTransformGrids(N, N, cent),
                   ky=ky[:n1], kz=kz[:n1], nEc=nEc[:2], mSt=mSt[:n1])
    Eo = OStruct(Tr=T, NMs=1, NSe=1, Sf=Sm.astype(np.complex128), ky=ky[:n1], kz=kz[:n1], nEc=nEc[:2],
                 mSt=mSt[:n1], grids=ogrids(N, N, cent, sh=1), cent=cent)
    yo = oenc.encode(x.astype(np.complex128), Eo)
    ctx.set_precision(mode)
    try:
        y = db.encode(x, Ed, ctx=ctx)
    finally:
        ctx.set_precision("fp32")
    print("encode rel. err. vs FP64 oracle: %s %.2e" % (mode, rel(y, yo)))
    assert rel(y, yo) < TOL[mode]
