"""Minimal NIfTI-1 single-file reader/writer in numpy (the format of the
dualgpmf command line's inputs and outputs).

Arrays are (nz, ny, nx) with x fastest on disk, as the format stores them.
``qform`` follows the format's index-to-space rule for qform_code > 0: a
rotation from the quaternion (b, c, d), the pixel sizes, qfac = sign of
pixdim[0] applied to the third axis, and the offsets.
"""
from __future__ import annotations

import gzip
import struct

import numpy as np

_DT = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64, 256: np.int8, 512: np.uint16,
       768: np.uint32}
_CODE = {np.dtype(v): k for k, v in _DT.items()}


def _open(path, mode):
    return gzip.open(path, mode) if str(path).endswith(".gz") else open(path, mode)


def quatern_to_qform(b, c, d, pixdim, qoffset, qfac=1.0):
    s = b * b + c * c + d * d
    if s >= 1.0:
        r = 1.0 / np.sqrt(s)
        b, c, d, a = b * r, c * r, d * r, 0.0
    else:
        a = np.sqrt(1.0 - s)
    R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                  [2 * (b * c + a * d), a * a + c * c - b * b - d * d, 2 * (c * d - a * b)],
                  [2 * (b * d - a * c), 2 * (c * d + a * b), a * a + d * d - b * b - c * c]])
    sc = np.array([pixdim[0] if pixdim[0] > 0 else 1.0, pixdim[1] if pixdim[1] > 0 else 1.0,
                   (pixdim[2] if pixdim[2] > 0 else 1.0) * (-1.0 if qfac < 0 else 1.0)])
    Q = np.eye(4)
    Q[:3, :3] = R * sc[None, :]
    Q[:3, 3] = qoffset
    return Q.astype(np.float32)


def write(path, data, pixdim=(1.0, 1.0, 1.0), quatern=(0.0, 0.0, 0.0), qoffset=(0.0, 0.0, 0.0), qfac=1.0,
          dtype=np.float32):
    """Write a 3D array (nz, ny, nx) as a single-file NIfTI-1 (.nii or .nii.gz) with qform_code 1."""
    a = np.ascontiguousarray(data, dtype=dtype)
    nz, ny, nx = a.shape
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8h", h, 40, 3, nx, ny, nz, 1, 1, 1, 1)
    struct.pack_into("<h", h, 70, _CODE[a.dtype])
    struct.pack_into("<h", h, 72, a.dtype.itemsize * 8)
    struct.pack_into("<8f", h, 76, -1.0 if qfac < 0 else 1.0, *pixdim, 1.0, 1.0, 1.0, 1.0)
    struct.pack_into("<f", h, 108, 352.0)
    struct.pack_into("<f", h, 112, 1.0)
    struct.pack_into("<hh", h, 252, 1, 0)
    struct.pack_into("<6f", h, 256, *quatern, *qoffset)
    h[344:348] = b"n+1\x00"
    with _open(path, "wb") as f:
        f.write(bytes(h))
        f.write(b"\x00\x00\x00\x00")
        f.write(a.tobytes())


def write_like(path, data, qform):
    """Write with a diagonal (axis-aligned, positive) qform given as a 4x4 matrix."""
    Q = np.asarray(qform, np.float64)
    if np.abs(Q[:3, :3] - np.diag(np.diag(Q[:3, :3]))).max() > 0 or np.any(np.diag(Q)[:3] <= 0):
        raise ValueError("write_like supports diagonal, positive qforms only")
    write(path, data, pixdim=tuple(np.diag(Q)[:3]), qoffset=tuple(Q[:3, 3]))


def read(path):
    """Returns (array (nz, ny, nx), qform 4x4 float32, header dict)."""
    with _open(path, "rb") as f:
        raw = f.read()
    h = raw[:348]
    endian = "<" if struct.unpack("<i", h[:4])[0] == 348 else ">"
    dim = struct.unpack(endian + "8h", h[40:56])
    dt = struct.unpack(endian + "h", h[70:72])[0]
    pix = struct.unpack(endian + "8f", h[76:108])
    vox = int(struct.unpack(endian + "f", h[108:112])[0])
    qcode = struct.unpack(endian + "h", h[252:254])[0]
    qb, qc, qd, qx, qy, qz = struct.unpack(endian + "6f", h[256:280])
    nx, ny, nz = dim[1], dim[2] if dim[0] >= 2 else 1, dim[3] if dim[0] >= 3 else 1
    dtype = np.dtype(_DT[dt]).newbyteorder(endian)
    a = np.frombuffer(raw, dtype=dtype, count=nx * ny * nz, offset=max(vox, 352)).reshape(nz, ny, nx)
    if qcode > 0:
        Q = quatern_to_qform(qb, qc, qd, pix[1:4], (qx, qy, qz), pix[0])
    else:
        Q = np.diag([pix[1], pix[2], pix[3], 1.0]).astype(np.float32)
    return a.astype(a.dtype.newbyteorder("=")), Q, dict(dim=dim, datatype=dt, pixdim=pix, qform_code=qcode)
