"""Reader of the output files written by hcl_write_output (Domain.write_output).

An output holds the datasets the reference writes to its HDF5 outputs
(io/config.yaml.cpp:7-265): the counters output_id, iter_output_id,
time_output_id, iter, current_time and gamma, the nodes x0..x2 (with ghosts)
and x0_ng..x2_ng (interior), and the interior fields rho, ux0..ux{ndim-1}, P,
E, T and fx0..fx{nfx-1} as arrays of shape (nx2, nx1, nx0).

File layout: the magic b"HCLRAW01", a little-endian uint64 index length, a
text index with one line per dataset ("name type offset rank extents..."),
then little-endian data at the listed byte offsets.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

MAGIC = b"HCLRAW01"
_DTYPES = {"f64": np.dtype("<f8"), "i32": np.dtype("<i4")}


def read_index(path):
    """[(name, dtype, offset, shape)] of the datasets in an output file."""
    with open(path, "rb") as f:
        head = f.read(16)
        if len(head) != 16 or head[:8] != MAGIC:
            raise ValueError(f"{path} is not an output file (magic {head[:8]!r})")
        (n,) = struct.unpack("<Q", head[8:])
        text = f.read(n).decode()
    out = []
    for line in text.splitlines():
        parts = line.split()
        rank = int(parts[3])
        out.append((parts[0], _DTYPES[parts[1]], int(parts[2]), tuple(int(v) for v in parts[4:4 + rank])))
    return out


def read_output(path) -> dict:
    """Every dataset of an output file: arrays for fields and nodes, Python
    scalars for the counters and time."""
    path = Path(path)
    data = {}
    with open(path, "rb") as f:
        for name, dtype, offset, shape in read_index(path):
            f.seek(offset)
            count = int(np.prod(shape)) if shape else 1
            a = np.fromfile(f, dtype=dtype, count=count)
            data[name] = a.reshape(shape) if shape else a[0].item()
    return data
