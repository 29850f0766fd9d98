"""Real-data IO (disorder_b200.nifti): the NIfTI-1 files of IO/writeNII.m and
IO/readNII.m.

The header is checked byte by byte at the offsets of the NIfTI-1 standard,
with the values the reference's toolbox writes (Libs/NIfTI_20140122:
make_nii.m:165-253 defaults, save_nii.m:179-196 glmax / glmin, vox_offset
352 and magic 'n+1', save_nii_hdr.m:64-224 field order), and the image
through its byte offset and column-major order.
"""

import gzip
import os
import shutil
import struct

import numpy as np
import pytest

from disorder_b200 import nifti


def _hdr(path):
    with open(path, "rb") as f:
        return f.read()


def test_header_and_image_layout(tmp_path):
    rng = np.random.default_rng(0)
    x = (rng.standard_normal((5, 4, 3)) * 10).astype(np.float32)
    MS = [[0.8, 0.9, 1.2]]
    dat = str(tmp_path / "rec")
    nifti.writeNII(dat, ["Aq"], [x], MS)
    raw = _hdr(dat + "_Aq.nii")
    assert len(raw) == 352 + 4 * x.size
    assert struct.unpack_from("<i", raw, 0)[0] == 348                       # sizeof_hdr
    assert raw[4:38] == b"\x00" * 34                                        # data_type, db_name, extents, session_error
    assert raw[38:40] == b"r\x00"                                           # regular, dim_info
    assert struct.unpack_from("<8h", raw, 40) == (3, 5, 4, 3, 1, 1, 1, 1)  # dim
    assert struct.unpack_from("<3f", raw, 56) == (0.0, 0.0, 0.0)            # intent_p1..3
    assert struct.unpack_from("<4h", raw, 68) == (0, 16, 32, 0)             # intent_code, datatype, bitpix, slice_start
    pd = struct.unpack_from("<8f", raw, 76)
    assert np.allclose(pd, [0, 0.8, 0.9, 1.2, 1, 1, 1, 1], atol=1e-7)
    assert struct.unpack_from("<3f", raw, 108) == (352.0, 0.0, 0.0)         # vox_offset, scl_slope, scl_inter
    gl = struct.unpack_from("<2i", raw, 140)
    assert gl == (int(np.sign(x.max()) * np.floor(abs(x.max()) + 0.5)),
                  int(np.sign(x.min()) * np.floor(abs(x.min()) + 0.5)))     # glmax, glmin
    assert raw[148:228] == b"\x00" * 80                                     # descrip
    assert raw[228:252] == b"none" + b"\x00" * 20                           # aux_file
    assert struct.unpack_from("<2h", raw, 252) == (0, 1)                    # qform_code, sform_code
    srow = np.array(struct.unpack_from("<12f", raw, 280)).reshape(3, 4)
    assert np.allclose(srow, [[0.8, 0, 0, 0], [0, 0.9, 0, 0], [0, 0, 1.2, 0]], atol=1e-7)
    assert raw[344:352] == b"n+1\x00\x00\x00\x00\x00"                       # magic, extension flag
    img = np.frombuffer(raw, "<f4", offset=352).reshape(x.shape, order="F")
    assert np.array_equal(img, x)
    y, MSr, MTr = nifti.readNII(dat, ["Aq"])
    assert np.array_equal(y[0], x) and np.allclose(MSr[0], MS[0]) and np.allclose(MTr[0][:3], srow)


def test_complex_writes_magnitude_and_phase(tmp_path):
    rng = np.random.default_rng(1)
    x = (rng.standard_normal((6, 5, 4)) + 1j * rng.standard_normal((6, 5, 4))).astype(np.complex64)
    dat = str(tmp_path / "rec")
    MT = np.array([[-0.5, 0, 0, 10], [0, -0.5, 0, 20], [0, 0, 1.0, -5], [0, 0, 0, 1]])
    nifti.writeNII(dat, ["x"], [x], [[0.5, 0.5, 1.0]], [MT])
    assert os.path.exists(dat + "_x.nii") and os.path.exists(dat + "_xPh.nii")
    mag = np.frombuffer(_hdr(dat + "_x.nii"), "<f4", offset=352).reshape(x.shape, order="F")
    ph = np.frombuffer(_hdr(dat + "_xPh.nii"), "<f4", offset=352).reshape(x.shape, order="F")
    assert np.array_equal(mag, np.abs(x)) and np.array_equal(ph, np.angle(x))
    y, MS, MTr = nifti.readNII(dat, ["x"])
    assert y[0].dtype == np.complex64
    assert np.linalg.norm(y[0] - x) / np.linalg.norm(x) < 1e-6
    assert np.allclose(MTr[0], MT)
    # a real volume writes no phase file
    nifti.writeNII(dat, ["r"], [np.abs(x)])
    assert not os.path.exists(dat + "_rPh.nii")


def test_higher_dimensions_fold_into_the_fourth(tmp_path):
    x = np.arange(4 * 5 * 6 * 2 * 3, dtype=np.float32).reshape((4, 5, 6, 2, 3), order="F")
    dat = str(tmp_path / "rec")
    nifti.writeNII(dat, ["t"], [x], [[1.0, 1.0, 2.0, 3.5]])
    raw = _hdr(dat + "_t.nii")
    assert struct.unpack_from("<8h", raw, 40) == (4, 4, 5, 6, 6, 1, 1, 1)
    assert struct.unpack_from("<f", raw, 76 + 16)[0] == 3.5                 # MS(4) -> pixdim(5)
    y, _, _ = nifti.readNII(dat, ["t"])
    assert np.array_equal(y[0], x.reshape((4, 5, 6, 6), order="F"))
    # trailing singleton dimensions are dropped, as MATLAB's size() does
    nifti.writeNII(dat, ["s"], [np.ones((4, 5, 1), np.float32)])
    assert struct.unpack_from("<8h", _hdr(dat + "_s.nii"), 40) == (2, 4, 5, 1, 1, 1, 1, 1)


def test_gzip_files_and_errors(tmp_path):
    x = np.linspace(-3, 3, 60, dtype=np.float32).reshape((3, 4, 5))
    dat = str(tmp_path / "rec")
    nifti.writeNII(dat, ["g"], [x])
    with open(dat + "_g.nii", "rb") as fi, gzip.open(dat + "_g.nii.gz", "wb") as fo:
        shutil.copyfileobj(fi, fo)
    os.remove(dat + "_g.nii")
    y, _, _ = nifti.readNII(dat, ["g"])
    assert np.array_equal(y[0], x)
    with pytest.raises(FileNotFoundError):
        nifti.readNII(dat, ["missing"])
    with pytest.raises(ValueError):
        nifti.writeNII(dat, ["a", "b"], [x])


def test_geometry_from_the_acquisition_matrix():
    A = np.array([[0, 0, 1.5, -90], [0.8, 0, 0, -100], [0, 0.8, 0, -80], [0, 0, 0, 1]])
    MS, MT = nifti.nii_geometry(A)
    assert np.allclose(MS, [0.8, 0.8, 1.5, 1.0])
    assert np.allclose(MT, [[0, 0, -1.5, 90], [-0.8, 0, 0, 100], [0, 0.8, 0, -80], [0, 0, 0, 1]])


def test_write_data_writes_image_and_motion(tmp_path):
    from scipy.io import loadmat
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((6, 5, 4)) + 1j * rng.standard_normal((6, 5, 4))).astype(np.complex64)
    T = rng.standard_normal((8, 6)).astype(np.float32)
    A = np.diag([2.0, 2.0, 3.0, 1.0])
    dat = str(tmp_path / "scan")
    nifti.writeData(dat, x, T, A)
    y, MS, MT = nifti.readNII(dat, ["Aq"])
    assert np.linalg.norm(y[0] - x) / np.linalg.norm(x) < 1e-6
    assert np.allclose(MS[0], [2.0, 2.0, 3.0]) and np.allclose(MT[0], np.diag([-2.0, -2.0, 3.0, 1.0]))
    assert np.array_equal(loadmat(dat + "_T.mat")["T"], T)
