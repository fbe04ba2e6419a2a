"""CPU oracle for the DBSCAN hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import
this package, and only as the checker or the timed CPU baseline, never as the
thing measured on the GPU or shipped.

  reference(...)  literal restatement of the reference's phases (ndb_oracle.c)
  grid(...)       exact grid restatement of the same outputs (ndb_oracle.c)
  cells(...)      the same outputs organised for 10^7..10^8 points (ndb_oracle.c)
  border_ids(...) the border rule with given core ids (ndb_oracle.c)
  run_ref(...)    the reference's own OpenMP implementation, built from its
                  sources into _ref/ndb_ref_harness by oracle/Makefile
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libndb_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ndb_ref_harness")
NO_CLUSTER = 2**31 - 1

_lib = None


def ref_dir() -> str | None:
    """Where the reference's sources are checked out: $NDB_REF_DIR, else the
    read-only mount this repository's build reads them from.  None when neither
    holds data_process.cpp (for instance on a GPU box, which only runs the
    prebuilt _ref/ binaries)."""
    for cand in (os.environ.get("NDB_REF_DIR"), "/root/reference"):
        if cand and os.path.isfile(os.path.join(cand, "data_process.cpp")):
            return cand
    return None


def build(ref: str | None = None, targets: tuple[str, ...] = ()) -> None:
    """Builds the C restatement and, when the reference's sources are found, the
    reference's own OpenMP build into _ref/."""
    cmd = ["make", "-s", "-C", HERE]
    ref = ref or ref_dir()
    if ref:
        cmd.append(f"REF_DIR={ref}")
    subprocess.run(cmd + list(targets), check=True)


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        lib.ndb_oracle_reference.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                             ctypes.c_int32, vp, vp, vp, vp]
        lib.ndb_oracle_reference.restype = ctypes.c_int
        lib.ndb_oracle_grid.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                        vp, vp, vp]
        lib.ndb_oracle_grid.restype = ctypes.c_int
        lib.ndb_oracle_cells.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                         ctypes.c_int32, vp, vp, vp]
        lib.ndb_oracle_cells.restype = ctypes.c_int
        lib.ndb_oracle_border_ids.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                              vp, vp, vp]
        lib.ndb_oracle_border_ids.restype = ctypes.c_int
        lib.ndb_oracle_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _pts(coords) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(coords, dtype=np.float32))
    if a.ndim != 2:
        raise ValueError("coords must be n x d")
    return a


def reference(coords, eps: float, min_pts: int, approximate: bool = False):
    """Literal restatement.  Returns (nn, cluster_index, cluster_label, meta dict)."""
    a = _pts(coords)
    n, d = a.shape
    nn = np.zeros(n, np.int32)
    ci = np.zeros(n, np.int32)
    lab = np.zeros(max(n, 1), np.int32)
    meta = np.zeros(8, np.int32)
    rc = _load().ndb_oracle_reference(a.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts), int(approximate),
                                      nn.ctypes.data, ci.ctypes.data, lab.ctypes.data, meta.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ndb_oracle_reference failed: {rc}")
    m = dict(clusters=int(meta[0]), noise=int(meta[1]), cores=int(meta[2]), n=int(meta[3]), sweeps=int(meta[4]))
    return nn, ci, lab[: m["cores"]].copy(), m


def grid(coords, eps: float, min_pts: int):
    """Grid restatement (exact, OpenMP).  Returns (nn, cluster_index, meta dict)."""
    a = _pts(coords)
    n, d = a.shape
    nn = np.zeros(n, np.int32)
    ci = np.zeros(n, np.int32)
    meta = np.zeros(8, np.int32)
    rc = _load().ndb_oracle_grid(a.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts), nn.ctypes.data,
                                 ci.ctypes.data, meta.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ndb_oracle_grid failed: {rc}")
    return nn, ci, dict(clusters=int(meta[0]), noise=int(meta[1]), cores=int(meta[2]), n=int(meta[3]))


def cells(coords, eps: float, min_pts: int, early: bool = False):
    """Cell restatement (exact, OpenMP in every phase, for 10^7..10^8 points).
    Same outputs as grid(); with early=True a point stops counting at min_pts, so
    nn is exact below min_pts and some value >= min_pts otherwise (core flags,
    cluster ids and meta stay exact).  Returns (nn, cluster_index, meta dict)."""
    a = _pts(coords)
    n, d = a.shape
    nn = np.zeros(n, np.int32)
    ci = np.zeros(n, np.int32)
    meta = np.zeros(8, np.int32)
    rc = _load().ndb_oracle_cells(a.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts), int(bool(early)),
                                  nn.ctypes.data, ci.ctypes.data, meta.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ndb_oracle_cells failed: {rc}")
    return nn, ci, dict(clusters=int(meta[0]), noise=int(meta[1]), cores=int(meta[2]), n=int(meta[3]),
                        clique_cells=bool(meta[4]))


def border_ids(coords, eps: float, min_pts: int, nn, ids):
    """The border rule with given core ids (brute force): cores keep ids[i], every
    other point takes the minimum id over the cores in range.  Returns the ids."""
    a = _pts(coords)
    n, d = a.shape
    nn = np.ascontiguousarray(np.asarray(nn, dtype=np.int32))
    ids = np.ascontiguousarray(np.asarray(ids, dtype=np.int32))
    out = np.zeros(n, np.int32)
    rc = _load().ndb_oracle_border_ids(a.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts), nn.ctypes.data,
                                       ids.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ndb_oracle_border_ids failed: {rc}")
    return out


def threads() -> int:
    return int(_load().ndb_oracle_threads())


def labels_from(ci: np.ndarray, nn: np.ndarray, min_pts: int) -> np.ndarray:
    """v_cluster_label in canonical form: the cluster id of every core, in core order."""
    return ci[nn >= min_pts].astype(np.int32)


def have_ref() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(coords, eps: float, min_pts: int, threads: int = 1, approximate: bool = False,
            workdir: str | None = None):
    """Runs the reference's own implementation on coords (written as a .bin).
    Returns (nn, cluster_index, cluster_label, info dict with the phase times)."""
    a = _pts(coords)
    if not have_ref():
        raise RuntimeError(f"{REF_BIN} is not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        inp = os.path.join(td, "in.bin")
        with open(inp, "wb") as f:
            f.write(np.array([a.shape[0], a.shape[1]], dtype="<i4").tobytes())
            a.astype("<f4").tofile(f)
        out = os.path.join(td, "out")
        r = subprocess.run([REF_BIN, "-m", str(int(min_pts)), "-e", repr(float(np.float32(eps))), "-t",
                            str(int(threads)), "-a", "1" if approximate else "0", "-o", out, inp],
                           capture_output=True, text=True, check=True)
        info = json.loads(r.stdout.strip().splitlines()[-1])
        nn = np.fromfile(out + ".nn.i32", dtype="<i4")
        ci = np.fromfile(out + ".ci.i32", dtype="<i4")
        lab = np.fromfile(out + ".label.i32", dtype="<i4")
    return nn, ci, lab, info
