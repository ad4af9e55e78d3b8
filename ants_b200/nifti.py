"""Pure-numpy NIfTI-1 (.nii / .nii.gz) reader and writer for scalar images and the vector
displacement fields antsRegistration writes (5-D, intent vector, component planes).

Geometry is returned in ITK's LPS convention (origin, direction), converted from the file's RAS
sform (or pixdim alone when no sform is set).
"""
from __future__ import annotations

import gzip
import struct

import numpy as np

from .synx import Geom

_HDR = struct.Struct("<i10s18sihcb8h3f4h8f3fh2c4f2i80s24s2h6f4f4f4f16s4s")
_DT = {2: np.uint8, 4: np.int16, 8: np.int32, 16: np.float32, 64: np.float64, 256: np.int8, 512: np.uint16,
       768: np.uint32}


def _open(path, mode):
    return gzip.open(path, mode) if str(path).endswith(".gz") else open(path, mode)


def write(path, data: np.ndarray, geom: Geom, vector: bool = False, time_series: bool = False,
          time_step: float = 1.0) -> None:
    """data: scalar image in numpy order (z, y, x) / (y, x); or, with vector=True, a field in
    interleaved layout grid.shape + (dim,) (the synx/ITK buffer layout); or, with time_series=True,
    a 3-D series grid.shape + (volumes,) written as a 4-D image."""
    d = geom.dim
    if time_series:
        planes = np.moveaxis(np.asarray(data, np.float32), -1, 0)  # volume slowest in the file
        dims = [4, geom.size[0], geom.size[1], geom.size[2] if d == 3 else 1, planes.shape[0], 1, 1, 1]
        intent = 0
    elif vector:
        planes = np.moveaxis(np.asarray(data, np.float32), -1, 0)  # component slowest in the file
        dims = [5, geom.size[0], geom.size[1], geom.size[2] if d == 3 else 1, 1, d, 1, 1]
        intent = 1007
    else:
        planes = np.asarray(data, np.float32)
        dims = [d, geom.size[0], geom.size[1], geom.size[2] if d == 3 else 1, 1, 1, 1, 1]
        intent = 0
    D = np.eye(3)
    D[:d, :d] = geom.direction
    sp = list(geom.spacing) + [1.0] * (3 - d)
    org = list(geom.origin) + [0.0] * (3 - d)
    A = np.zeros((3, 4))
    A[:, :3] = D * np.array(sp)[None, :]
    A[:, 3] = org
    A[:2] *= -1.0  # LPS -> RAS
    pixdim = [1.0] + sp + [float(time_step) if time_series else 1.0] + [1.0] * 3
    hdr = _HDR.pack(348, b"", b"", 0, 0, b"r", 0, *dims, 0.0, 0.0, 0.0, intent, 16, 32, 0, *pixdim, 352.0, 1.0, 0.0,
                    0, b"\0", bytes([10]), 0.0, 0.0, 0.0, 0.0, 0, 0, b"synx", b"", 0, 1, 0.0, 0.0, 0.0,
                    A[0, 3], A[1, 3], A[2, 3], *A[0], *A[1], *A[2], b"", b"n+1\0")
    with _open(path, "wb") as fh:
        fh.write(hdr)
        fh.write(b"\0\0\0\0")
        fh.write(np.ascontiguousarray(planes, np.float32).tobytes())


def read(path, dim: int | None = None):
    """Returns (array, Geom).  Scalar images come back in numpy order (z, y, x) / (y, x); vector
    images in interleaved layout grid.shape + (components,); 4-D series as grid.shape + (volumes,)."""
    with _open(path, "rb") as fh:
        raw = fh.read()
    f = _HDR.unpack(raw[:348])
    if f[0] != 348:
        raise ValueError(f"{path}: not a little-endian NIfTI-1 file")
    dims = f[7:15]
    datatype = f[19]
    pixdim = f[22:30]
    vox_offset = int(f[30])
    srow = np.array(f[52:64], dtype=np.float64).reshape(3, 4)
    sform_code = f[45]
    nd = dims[0]
    n = [max(int(x), 1) for x in dims[1:nd + 1]] + [1] * (7 - nd)
    d = dim or (3 if n[2] > 1 else 2)
    comps = n[4] * n[3]  # vector components, or the volumes of a 4-D series
    if sform_code > 0:
        A = srow.copy()
    else:
        A = np.zeros((3, 4))
        A[:, :3] = np.diag(pixdim[1:4])
    A[:2] *= -1.0
    sp = [float(pixdim[k + 1]) for k in range(3)]
    Dm = A[:, :3] / np.array(sp)[None, :]
    geom = Geom(tuple(n[:d]), tuple(sp[:d]), tuple(A[:d, 3]), Dm[:d, :d])
    arr = np.frombuffer(raw, dtype=_DT[datatype], count=int(np.prod(n[:3])) * comps, offset=max(vox_offset, 352))
    arr = arr.astype(np.float32)
    shape = geom.shape
    if comps > 1:
        arr = np.moveaxis(arr.reshape((comps,) + shape), 0, -1).copy()
    else:
        arr = arr.reshape(shape)
    return arr, geom
