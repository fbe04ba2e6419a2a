"""Input formats of nextdbscan-exa (magma_input.h), host side.

  .bin  int32 n, int32 d, then float32[n*d] row-major (magma_input.h:113-125)
  .csv  one point per line, coordinates separated by spaces, parsed with atof and
        cast to float (magma_input.h:127-142, dimension count from the first line
        at :53-67)
  .h5/.hdf5  dataset "xyz" (magma_input.h:74-111) -- needs h5py, which this image
        lacks; reading one raises, as the reference does without HDF5_ON (:158-160)

The reference reads a per-rank block (get_block_size/offset, magma_input.h:33-49);
with one rank that block is the whole file, which is what read_input returns.
"""
from __future__ import annotations

import os
import struct

import numpy as np


def read_bin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        head = f.read(8)
        if len(head) < 8:
            raise ValueError(f"{path}: truncated .bin header")
        n, d = struct.unpack("<ii", head)
        if n < 0 or d <= 0:
            raise ValueError(f"{path}: bad .bin header n={n} d={d}")
        data = np.fromfile(f, dtype="<f4", count=n * d)
    if data.size != n * d:
        raise ValueError(f"{path}: expected {n * d} floats, found {data.size}")
    return data.reshape(n, d)


def write_bin(path: str, coords: np.ndarray) -> None:
    coords = np.ascontiguousarray(coords, dtype="<f4")
    if coords.ndim != 2:
        raise ValueError("coords must be n x d")
    n, d = coords.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", n, d))
        coords.tofile(f)


def read_csv(path: str) -> np.ndarray:
    rows = []
    d = 0
    with open(path, "r") as f:
        for line in f:
            parts = line.split()
            if d == 0:
                d = len(parts)
            rows.append([float(v) for v in parts[:d]])
    if not rows:
        return np.zeros((0, max(d, 1)), dtype=np.float32)
    # atof -> double -> static_cast<float> (magma_input.h:138)
    return np.asarray(rows, dtype=np.float64).astype(np.float32)


def read_input(path: str) -> np.ndarray:
    """magma_input::read_input (magma_input.h:144-167) for one rank."""
    if path.endswith(".bin"):
        return read_bin(path)
    if path.endswith(".csv"):
        return read_csv(path)
    if path.endswith(".h5") or path.endswith(".hdf5"):
        raise RuntimeError("Error: HDF5 is not supported by this executable.")
    raise ValueError(f"unsupported input type: {os.path.basename(path)}")
