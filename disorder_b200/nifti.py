"""Real-data IO: NIfTI-1 volumes on either side of the reconstruction.

``writeNII`` / ``readNII`` follow IO/writeNII.m:12-46 and IO/readNII.m:15-37:
a complex volume is written as two files, ``<dat>_<suffix>.nii`` with the
magnitude and ``<dat>_<suffix>Ph.nii`` with the phase (writeNII.m:33-40),
and read back as magnitude * exp(i phase) (readNII.m:27-32). Arrays are
float32, column-major, reshaped to (N1, N2, N3, prod of the rest)
(writeNII.m:31-32). The spacing MS goes to pixdim (make_nii.m:85-87, with
MS(4) to pixdim(5) when given, writeNII.m:37,43) and the orientation MT to
srow_x/y/z with sform_code = 1 (writeNII.m:36,42); MT defaults to the
identity scaled by MS (writeNII.m:18-25).

The file layout is the single-file NIfTI-1 format as the reference's
toolbox (Libs/NIfTI_20140122) writes it: a 348-byte header
(save_nii_hdr.m:64-224), 4 zero bytes of extension flag (vox_offset = 352,
save_nii.m:190,233,278) and the image. Header values that the toolbox sets
and DISORDER does not touch keep the toolbox's defaults (make_nii.m:165-253):
regular = 'r', aux_file = 'none', glmax / glmin = the rounded image maximum
and minimum (save_nii.m:179-180), magic = 'n+1' (save_nii.m:196), everything
else zero. ``nii_geometry`` is writeData.m's generateNIIInformation
(IO/writeData.m:60-66).
"""

import gzip
import math
import os
import struct

import numpy as np

HDR_SIZE = 348
VOX_OFFSET = 352
DT_FLOAT32 = 16
DT_FLOAT64 = 64


def _round_half_away(v):
    """MATLAB round: halves away from zero."""
    return int(math.copysign(math.floor(abs(v) + 0.5), v))


def _matlab_dims(shape):
    """size() of an array with trailing singleton dimensions dropped (at
    least 2), as make_nii.m:48-50 sees it: [ndims, dims..., 1, ...] (8 values)."""
    s = list(shape)
    while len(s) > 2 and s[-1] == 1:
        s.pop()
    if len(s) > 7:
        raise ValueError("NIfTI only allows up to 7 dimensions")
    return [len(s)] + s + [1] * (7 - len(s))


def header_bytes(shape, pixdim, srow, glmax, glmin, datatype=DT_FLOAT32):
    """The 348-byte NIfTI-1 header (little-endian) of an image of the given
    column-major shape: pixdim (8 values), srow (3 x 4, sform_code = 1)."""
    bitpix = {DT_FLOAT32: 32, DT_FLOAT64: 64}[datatype]
    h = bytearray(HDR_SIZE)
    struct.pack_into("<i", h, 0, HDR_SIZE)                      # sizeof_hdr
    # data_type[10], db_name[18] zero; extents (32) = 0, session_error (36) = 0
    h[38] = ord("r")                                              # regular
    struct.pack_into("<8h", h, 40, *_matlab_dims(shape))          # dim
    # intent_p1..3 (56..67), intent_code (68) zero
    struct.pack_into("<hhh", h, 70, datatype, bitpix, 0)          # datatype, bitpix, slice_start
    struct.pack_into("<8f", h, 76, *[float(p) for p in pixdim])   # pixdim
    struct.pack_into("<fff", h, 108, VOX_OFFSET, 0.0, 0.0)        # vox_offset, scl_slope, scl_inter
    # slice_end, slice_code, xyzt_units, cal_max/min, slice_duration, toffset zero
    struct.pack_into("<ii", h, 140, glmax, glmin)                 # glmax, glmin
    # descrip[80] at 148 zero
    h[228:232] = b"none"                                          # aux_file[24]
    struct.pack_into("<hh", h, 252, 0, 1)                         # qform_code, sform_code
    # quatern_b..d, qoffset_x..z (256..279) zero
    struct.pack_into("<12f", h, 280, *[float(v) for v in np.asarray(srow, float).ravel()])
    # intent_name[16] at 328 zero
    h[344:348] = b"n+1\x00"                                       # magic
    return bytes(h)


def _write_one(path, img, pixdim, srow):
    a = np.asarray(img, np.float32)
    finite = a[np.isfinite(a)] if a.size else a
    mx = _round_half_away(float(finite.max())) if finite.size else 0
    mn = _round_half_away(float(finite.min())) if finite.size else 0
    with open(path, "wb") as f:
        f.write(header_bytes(a.shape, pixdim, srow, mx, mn))
        f.write(b"\x00" * (VOX_OFFSET - HDR_SIZE))
        f.write(np.asfortranarray(a).tobytes(order="F"))


def writeNII(dat, suffix, x, MS=None, MT=None):
    """IO/writeNII.m: write the arrays x[n] (host or device) as
    <dat>_<suffix[n]>.nii (and <dat>_<suffix[n]>Ph.nii for complex data).
    MS[n]: spacing (3 or 4 values, default 1), MT[n]: 4 x 4 orientation
    (default diag(MS, 1))."""
    N = len(suffix)
    if MS is None:
        MS = [[1.0, 1.0, 1.0] for _ in range(N)]
    if MT is None:
        MT = []
        for n in range(N):
            m = np.eye(4)
            for d in range(3):
                m[d, d] = MS[n][d]
            MT.append(m)
    lens = {len(suffix), len(x), len(MS), len(MT)}
    if len(lens) != 1:
        raise ValueError("Size of input cells must be the same. Currently it is: %d %d %d %d"
                         % (len(suffix), len(x), len(MS), len(MT)))
    for n in range(N):
        v = x[n].numpy() if hasattr(x[n], "numpy") else np.asarray(x[n])
        M = list(v.shape) + [1] * (12 - v.ndim)
        v = v.reshape(M[:3] + [int(np.prod(M[3:12]))], order="F")
        ms = list(MS[n])
        pixdim = [0.0, ms[0], ms[1], ms[2], ms[3] if len(ms) >= 4 else 1.0, 1.0, 1.0, 1.0]
        srow = np.asarray(MT[n], float)[:3, :]
        if np.iscomplexobj(v):
            v = v.astype(np.complex64)
            if np.any(v.imag):
                _write_one("%s_%sPh.nii" % (dat, suffix[n]), np.angle(v), pixdim, srow)
                v = np.abs(v)
        _write_one("%s_%s.nii" % (dat, suffix[n]), np.real(v), pixdim, srow)


def _read_one(path):
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rb") as f:
        raw = f.read()
    if len(raw) < HDR_SIZE or struct.unpack_from("<i", raw, 0)[0] != HDR_SIZE:
        raise ValueError("%s: not a little-endian NIfTI-1 file" % path)
    if raw[344:347] != b"n+1":
        raise ValueError("%s: not a single-file NIfTI-1 image" % path)
    dim = struct.unpack_from("<8h", raw, 40)
    datatype, _bitpix = struct.unpack_from("<hh", raw, 70)
    pixdim = struct.unpack_from("<8f", raw, 76)
    vox = int(struct.unpack_from("<f", raw, 108)[0])
    srow = np.array(struct.unpack_from("<12f", raw, 280), float).reshape(3, 4)
    dt = {DT_FLOAT32: "<f4", DT_FLOAT64: "<f8", 4: "<i2", 8: "<i4", 2: "u1", 256: "i1", 512: "<u2",
          768: "<u4"}.get(datatype)
    if dt is None:
        raise ValueError("%s: datatype %d is not supported" % (path, datatype))
    shape = tuple(int(d) for d in dim[1:1 + max(1, dim[0])])
    n = int(np.prod(shape))
    img = np.frombuffer(raw, dtype=dt, count=n, offset=vox).reshape(shape, order="F")
    return img, pixdim, srow


def readNII(dat, suff):
    """IO/readNII.m: read <dat>_<suff[n]>.nii (or .nii.gz), times
    exp(i phase) when <dat>_<suff[n]>Ph.nii(.gz) exists. Returns (x, MS, MT)
    lists: MS = pixdim(2:4), MT = [srow_x; srow_y; srow_z; 0 0 0 1]."""
    x, MS, MT = [], [], []
    for s in suff:
        files = ["%s_%s.nii" % (dat, s), "%s_%s.nii.gz" % (dat, s)]
        path = next((p for p in files if os.path.exists(p)), None)
        if path is None:
            raise FileNotFoundError("File %s does not exist" % files[0])
        img, pixdim, srow = _read_one(path)
        ph_path = "%s_%sPh.nii" % (dat, s) + (".gz" if path.endswith(".gz") else "")
        if os.path.exists(ph_path):
            ph, _, _ = _read_one(ph_path)
            img = img * np.exp(1j * ph)  # single precision for float32 files, as readNII.m:31
        x.append(np.array(img))
        MS.append(np.array(pixdim[1:4], float))
        m = np.eye(4)
        m[:3, :] = srow
        MT.append(m)
    return x, MS, MT


def nii_geometry(A):
    """IO/writeData.m:60-66 (generateNIIInformation): spacing = column norms
    of A(1:3,1:3) with a 4th entry 1, orientation = diag(-1, -1, 1, 1) A
    (the acquisition's voxel-to-world matrix to the NIfTI convention)."""
    A = np.asarray(A, float)
    MS = list(np.sqrt(np.sum(A[:3, :3] ** 2, axis=0))) + [1.0]
    MT = np.diag([-1.0, -1.0, 1.0, 1.0]) @ A
    return MS, MT


def writeData(fileName, x, T=None, A=None, suffix="Aq", MotionInfo=None):
    """The parts of IO/writeData.m:1-58 on the aligned path: the
    reconstruction x as <fileName>_<suffix>.nii (+ Ph for complex data) with
    the geometry of the voxel-to-world matrix A (generateNIIInformation;
    identity spacing when A is None), and the motion T with MotionInfo as
    <fileName>_T.mat (writeData.m:52-56; MATLAB 5 format through scipy)."""
    if A is None:
        writeNII(fileName, [suffix], [x])
    else:
        MS, MT = nii_geometry(A)
        writeNII(fileName, [suffix], [x], [MS], [MT])
    if T is not None:
        from scipy.io import savemat
        savemat("%s_T.mat" % fileName, {"T": np.asarray(T), "MotionInfo": MotionInfo if MotionInfo is not None
                                        else np.zeros((0, 0))})
