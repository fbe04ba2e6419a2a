"""nextdbscan-exa_b200: the DBSCAN hot path of nextdbscan-exa on one B200 (sm_100a).

Host-side mirror of the reference's algorithm-layer API over the C ABI of
libndb_b200.so (include/ndb_b200.h):

  data_process   the class of data_process.h:45-102: same constructor arguments,
                 the two phase methods select_and_process / select_cores_and_process,
                 get_result_meta and the public result vectors v_coord_nn,
                 v_coord_cluster_index and v_cluster_label.
  start          nextdbscan::start (nextdbscan.h:50, nextdbscan.cpp:28-68): read the
                 input file, run both phases, return the result meta.
  Context        direct access to the C ABI (host or device buffers, stream, stats).

All compute runs in the CUDA library; nothing here computes a neighbour, a label
or a count.  The library must be built (build.py) -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import time
from typing import NamedTuple

import numpy as np

from . import autotune, inputs, lib, synthetic

NO_CLUSTER = lib.NDB_NO_CLUSTER
__all__ = ["Context", "Result", "data_process", "start", "autotune", "inputs", "synthetic", "lib", "NO_CLUSTER"]


class Result(NamedTuple):
    """nextdbscan::result (nextdbscan.h:43-48)."""

    clusters: int
    noise: int
    core_count: int
    n: int


def _as_points(v_coord, n_dim: int | None = None) -> np.ndarray:
    a = np.asarray(v_coord)
    if a.dtype != np.float32:
        raise TypeError("coordinates must be float32 (the reference's only coordinate type)")
    if a.ndim == 1:
        if not n_dim or a.size % n_dim:
            raise ValueError("flat coordinates need n_dim dividing their size")
        a = a.reshape(-1, n_dim)
    if a.ndim != 2:
        raise ValueError("coordinates must be n x d")
    return np.ascontiguousarray(a)


def _flags(full_count: bool, approximate: bool, exact_count: bool = False, tensor_filter: bool = False,
           device: bool = False, audit: bool = False, gram_filter: bool = False) -> int:
    return ((lib.FLAG_FULL_COUNT if full_count else 0) | (lib.FLAG_APPROXIMATE if approximate else 0)
            | (lib.FLAG_EXACT_COUNT if exact_count else 0) | (lib.FLAG_TENSOR_FILTER if tensor_filter else 0)
            | (lib.FLAG_DEVICE_PTRS if device else 0) | (lib.FLAG_FILTER_AUDIT if audit else 0)
            | (lib.FLAG_GRAM_FILTER if gram_filter else 0))


class Context:
    """One libndb_b200 context (device buffers + stream) on one CUDA device."""

    def __init__(self, device: int = 0):
        self._lib = lib.load()
        h = ctypes.c_void_p()
        lib.check(self._lib.ndb_b200_create(ctypes.byref(h), int(device)), "ndb_b200_create")
        self._h = h
        self.device = device
        self.n = 0
        self._loaded = (0, 0)

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.ndb_b200_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_stream(self, stream_ptr: int | None) -> None:
        lib.check(self._lib.ndb_b200_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)),
                  "ndb_b200_set_stream", self._h)

    # -- host buffers -----------------------------------------------------
    def classify(self, coords, eps: float, min_pts: int, *, full_count: bool = False,
                 approximate: bool = False, want_nn: bool = True) -> np.ndarray | None:
        pts = _as_points(coords)
        n, d = pts.shape
        flags = (lib.FLAG_FULL_COUNT if full_count else 0) | (lib.FLAG_APPROXIMATE if approximate else 0)
        nn = np.empty(n, dtype=np.int32) if want_nn else None
        st = self._lib.ndb_b200_classify(self._h, pts.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts),
                                         flags, nn.ctypes.data if nn is not None else None)
        lib.check(st, "ndb_b200_classify", self._h)
        self.n = n
        self._keep = pts
        return nn

    def assign_labels(self, want_labels: bool = True) -> tuple[np.ndarray | None, Result]:
        ci = np.empty(self.n, dtype=np.int32) if want_labels else None
        res = lib.NdbResult()
        st = self._lib.ndb_b200_assign_labels(self._h, ci.ctypes.data if ci is not None else None,
                                              ctypes.byref(res))
        lib.check(st, "ndb_b200_assign_labels", self._h)
        return ci, Result(res.clusters, res.noise, res.core_count, res.n)

    def run(self, coords, eps: float, min_pts: int, *, full_count: bool = False,
            approximate: bool = False, exact_count: bool = False, tensor_filter: bool = False,
            audit: bool = False, gram_filter: bool = False) -> tuple[np.ndarray, np.ndarray, Result]:
        pts = _as_points(coords)
        n, d = pts.shape
        flags = _flags(full_count, approximate, exact_count, tensor_filter, audit=audit, gram_filter=gram_filter)
        nn = np.empty(n, dtype=np.int32)
        ci = np.empty(n, dtype=np.int32)
        res = lib.NdbResult()
        st = self._lib.ndb_b200_run(self._h, pts.ctypes.data, n, d, ctypes.c_float(eps), int(min_pts), flags,
                                    nn.ctypes.data, ci.ctypes.data, ctypes.byref(res))
        lib.check(st, "ndb_b200_run", self._h)
        self.n = n
        return nn, ci, Result(res.clusters, res.noise, res.core_count, res.n)

    # -- the reference's .bin file straight to the device (pinned, chunked, overlapped) --
    def load_bin(self, path: str) -> tuple[int, int]:
        """Loads a .bin file (int32 n, int32 d, n*d float32) into the context's device
        memory through pinned chunks; returns (n, d).  See ndb_b200_load_bin."""
        n = ctypes.c_int64()
        d = ctypes.c_int32()
        st = self._lib.ndb_b200_load_bin(self._h, str(path).encode(), ctypes.byref(n), ctypes.byref(d))
        lib.check(st, "ndb_b200_load_bin", self._h)
        self.n, self._loaded = n.value, (n.value, d.value)
        return n.value, d.value

    def run_loaded(self, eps: float, min_pts: int, *, full_count: bool = False, approximate: bool = False,
                   exact_count: bool = False, tensor_filter: bool = False) -> tuple[np.ndarray, np.ndarray, Result]:
        """ndb_b200_run on the loaded job, outputs in host memory."""
        n = self._loaded[0]
        nn = np.empty(n, dtype=np.int32)
        ci = np.empty(n, dtype=np.int32)
        res = lib.NdbResult()
        st = self._lib.ndb_b200_run_loaded(self._h, ctypes.c_float(eps), int(min_pts),
                                           _flags(full_count, approximate, exact_count, tensor_filter),
                                           nn.ctypes.data, ci.ctypes.data, ctypes.byref(res))
        lib.check(st, "ndb_b200_run_loaded", self._h)
        self.n = n
        return nn, ci, Result(res.clusters, res.noise, res.core_count, res.n)

    # -- raw addresses: host (pageable or pinned) or, with device=True, device memory --
    def run_ptrs(self, coords_ptr: int, n: int, d: int, eps: float, min_pts: int, nn_ptr: int | None,
                 ci_ptr: int | None, *, device: bool, full_count: bool = False,
                 approximate: bool = False, exact_count: bool = False, tensor_filter: bool = False,
                 audit: bool = False) -> Result:
        flags = _flags(full_count, approximate, exact_count, tensor_filter, device, audit)
        res = lib.NdbResult()
        st = self._lib.ndb_b200_run(self._h, ctypes.c_void_p(coords_ptr), n, d, ctypes.c_float(eps),
                                    int(min_pts), flags, ctypes.c_void_p(nn_ptr or 0),
                                    ctypes.c_void_p(ci_ptr or 0), ctypes.byref(res))
        lib.check(st, "ndb_b200_run", self._h)
        self.n = n
        return Result(res.clusters, res.noise, res.core_count, res.n)

    # -- device buffers (addresses of device memory, e.g. torch tensors) ---
    def run_device(self, coords_ptr: int, n: int, d: int, eps: float, min_pts: int, nn_ptr: int | None,
                   ci_ptr: int | None, *, full_count: bool = False, approximate: bool = False,
                   exact_count: bool = False, tensor_filter: bool = False, audit: bool = False) -> Result:
        flags = _flags(full_count, approximate, exact_count, tensor_filter, True, audit)
        res = lib.NdbResult()
        st = self._lib.ndb_b200_run(self._h, ctypes.c_void_p(coords_ptr), n, d, ctypes.c_float(eps),
                                    int(min_pts), flags, ctypes.c_void_p(nn_ptr or 0),
                                    ctypes.c_void_p(ci_ptr or 0), ctypes.byref(res))
        lib.check(st, "ndb_b200_run", self._h)
        self.n = n
        return Result(res.clusters, res.noise, res.core_count, res.n)

    # -- many independent problems in one pipeline ----------------------------
    def run_batched(self, problems, *, full_count: bool = False, approximate: bool = False,
                    want_nn: bool = True, exact_count: bool = False, tensor_filter: bool = False,
                    gram_filter: bool = False) -> list[tuple[np.ndarray | None, np.ndarray, Result]]:
        """problems: iterable of (coords n x d, eps, min_pts).  Returns per problem
        (nn, cluster_index, Result), equal to one run() each.  Raises NdbError on
        the first failing problem's status after every other one has run."""
        problems = list(problems)
        pts = [_as_points(c) for c, _, _ in problems]
        jobs = (lib.NdbJob * len(pts))()
        outs = []
        for j, ((_, eps, m), x) in enumerate(zip(problems, pts)):
            nn = np.empty(x.shape[0], dtype=np.int32) if want_nn else None
            ci = np.empty(x.shape[0], dtype=np.int32)
            jobs[j].coords = x.ctypes.data if x.size else None
            jobs[j].n, jobs[j].d = x.shape
            jobs[j].eps, jobs[j].min_pts = float(eps), int(m)
            jobs[j].nn_out = nn.ctypes.data if nn is not None and nn.size else None
            jobs[j].cluster_index_out = ci.ctypes.data if ci.size else None
            outs.append((nn, ci))
        flags = _flags(full_count, approximate, exact_count, tensor_filter, gram_filter=gram_filter)
        st = self._lib.ndb_b200_run_batched(self._h, jobs, len(pts), flags)
        self.last_jobs = jobs
        lib.check(st, "ndb_b200_run_batched", self._h)
        return [(nn, ci, Result(jobs[j].result.clusters, jobs[j].result.noise, jobs[j].result.core_count,
                                jobs[j].result.n)) for j, (nn, ci) in enumerate(outs)]

    def run_batched_jobs(self, jobs, n_jobs: int, flags: int) -> int:
        """Raw form: jobs is a ctypes array of lib.NdbJob (addresses filled by the
        caller, host or device per flags).  Returns the status without raising."""
        return self._lib.ndb_b200_run_batched(self._h, jobs, int(n_jobs), int(flags))

    def assign_border(self, core_ids) -> np.ndarray:
        """The border pass of the last run (host buffers) again with the caller's ids
        for the core points (n int32, input order); returns every point's cluster
        index.  See ndb_b200_assign_border."""
        ids = np.ascontiguousarray(np.asarray(core_ids, dtype=np.int32))
        if ids.shape != (self.n,):
            raise ValueError("core_ids must hold one int32 per point of the last run")
        out = np.empty(self.n, dtype=np.int32)
        st = self._lib.ndb_b200_assign_border(self._h, ids.ctypes.data, out.ctypes.data)
        lib.check(st, "ndb_b200_assign_border", self._h)
        return out

    def cluster_label(self, core_count: int) -> np.ndarray:
        out = np.empty(max(core_count, 0), dtype=np.int32)
        st = self._lib.ndb_b200_cluster_label(self._h, out.ctypes.data if core_count > 0 else None, core_count)
        lib.check(st, "ndb_b200_cluster_label", self._h)
        return out

    def set_memory_limit(self, max_bytes: int) -> None:
        """Caps the context's device footprint (0 = no cap); a run past it raises
        NdbError(NDB_ERR_OUT_OF_MEMORY) and leaves the context usable."""
        lib.check(self._lib.ndb_b200_set_memory_limit(self._h, int(max_bytes)), "ndb_b200_set_memory_limit",
                  self._h)

    def set_tuning(self, tc_min_dim: int = 0, tc_min_item: int = 0, gram_filter: int = 0) -> None:
        """Count-kernel choices of this context (0 = library default); see
        ndb_tuning in include/ndb_b200.h.  Results never depend on them."""
        t = lib.NdbTuning(int(tc_min_dim), int(tc_min_item), int(gram_filter))
        lib.check(self._lib.ndb_b200_set_tuning(self._h, ctypes.byref(t)), "ndb_b200_set_tuning", self._h)

    def reset_tuning(self) -> None:
        lib.check(self._lib.ndb_b200_set_tuning(self._h, None), "ndb_b200_set_tuning", self._h)

    def tuning(self) -> dict:
        t = lib.NdbTuning()
        lib.check(self._lib.ndb_b200_get_tuning(self._h, ctypes.byref(t)), "ndb_b200_get_tuning", self._h)
        return {"tc_min_dim": t.tc_min_dim, "tc_min_item": t.tc_min_item, "gram_filter": t.gram_filter}

    def set_debug_limits(self, uf_max_steps: int = 0) -> None:
        """Bound of the device-side union-find loops (0 = the library default); a run
        that reaches it raises NdbError(NDB_ERR_DEVICE_LIMIT) and leaves the context
        usable.  For tests of that error path."""
        if uf_max_steps < 0:
            raise ValueError("uf_max_steps must be >= 0")
        lib.check(self._lib.ndb_b200_set_debug_limits(self._h, int(uf_max_steps)), "ndb_b200_set_debug_limits",
                  self._h)

    def device_bytes(self) -> int:
        """Device memory the context holds now."""
        out = ctypes.c_int64()
        lib.check(self._lib.ndb_b200_device_bytes(self._h, ctypes.byref(out)), "ndb_b200_device_bytes", self._h)
        return out.value

    def stats(self) -> dict:
        s = lib.NdbStats()
        lib.check(self._lib.ndb_b200_get_stats(self._h, ctypes.byref(s)), "ndb_b200_get_stats", self._h)
        return s.as_dict()


class data_process:  # noqa: N801 -- the reference's class name
    """Mirror of the reference class data_process (data_process.h:45-102).

    Constructor arguments as data_process.h:60-77: the coordinates (float32, flat
    n*d or n x d), m (minPts), e (eps), n_dim, n_total_coord, is_approximate.  The
    phase methods take the reference's magmaMPI argument for signature
    compatibility; one GPU is one rank, so it is ignored.

    full_count (default True) makes v_coord_nn exact for every point, like the
    reference; with False core points stop counting at m (exact core flags and
    labels, v_coord_nn >= m for cores).
    """

    def __init__(self, v_coord, m: int, e: float, n_dim: int, n_total_coord: int, is_approximate: bool,
                 *, full_count: bool = True, device: int = 0, context: Context | None = None):
        self.m = int(m)
        self.n_dim = int(n_dim)
        self.e = float(np.float32(e))
        self.e2 = float(np.float32(e) * np.float32(e))  # data_process.h:73
        self.is_approximate = bool(is_approximate)
        self.v_coord = _as_points(v_coord, self.n_dim)
        self.n_coord = self.v_coord.shape[0]
        self.n_total_coord = int(n_total_coord)
        self.allocated_bytes = self.n_coord * self.n_dim * 4
        self.full_count = full_count
        self._ctx = context if context is not None else Context(device)
        self.v_coord_id = None
        self.v_coord_nn = None
        self.v_coord_cluster_index = None
        self.v_cluster_label = None
        self._result: Result | None = None

    def select_and_process(self, mpi=None) -> None:
        """data_process.cpp:334-392: neighbour counts and core flags."""
        self.v_coord_id = np.arange(self.n_coord, dtype=np.int32)
        self.v_coord_nn = self._ctx.classify(self.v_coord, self.e, self.m, full_count=self.full_count,
                                             approximate=self.is_approximate)

    def select_cores_and_process(self, mpi=None) -> None:
        """data_process.cpp:268-332: core-connected clusters and border points."""
        ci, res = self._ctx.assign_labels()
        self.v_coord_cluster_index = ci
        self._result = res
        self.v_cluster_label = self._ctx.cluster_label(res.core_count)

    def get_result_meta(self, mpi=None) -> tuple[int, int, int, int]:
        """data_process.cpp:50-91: returns (cores, noise, clusters, n)."""
        if self._result is None:
            raise RuntimeError("select_cores_and_process has not run")
        r = self._result
        return r.core_count, r.noise, r.clusters, r.n


def start(m: int, e: float, n_thread: int, in_file: str, mpi=None, is_approximate: bool = False,
          *, verbose: bool = True, device: int = 0) -> Result:
    """nextdbscan::start (nextdbscan.cpp:28-68) on one B200.

    n_thread is accepted for signature compatibility (the reference's OpenMP thread
    count); the GPU decides its own parallelism.
    """
    t0 = time.perf_counter()
    coords = inputs.read_input(in_file)
    t1 = time.perf_counter()
    if verbose:
        print(f"Read {coords.shape[0]} aggregated points with {coords.shape[1]} dimensions. ")
    dp = data_process(coords, m, e, coords.shape[1], coords.shape[0], is_approximate, full_count=False,
                      device=device)
    ta = time.perf_counter()
    dp.select_and_process(mpi)
    tb = time.perf_counter()
    dp.select_cores_and_process(mpi)
    tc = time.perf_counter()
    cores, noise, clusters, n = dp.get_result_meta(mpi)
    t2 = time.perf_counter()
    if verbose:
        print(f"Classify Points: {int((tb - ta) * 1000)} milliseconds")
        print(f"Assign Labels: {int((tc - tb) * 1000)} milliseconds")
        print(f"Total Execution Time: {int((t2 - t0) * 1000)} milliseconds")
        print(f"Total Execution Time (without I/O): {int((t2 - t1) * 1000)} milliseconds")
    return Result(clusters, noise, cores, n)
