"""ctypes binding of libndb_b200.so (the C ABI declared in include/ndb_b200.h).

The binding fails loudly when the shared library is missing: there is no CPU
fallback anywhere on the product path.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libndb_b200.so")

NDB_NO_CLUSTER = 2**31 - 1
NDB_MAX_DIM = 16

FLAG_APPROXIMATE = 0x1
FLAG_FULL_COUNT = 0x2
FLAG_DEVICE_PTRS = 0x4
FLAG_EXACT_COUNT = 0x8
FLAG_TENSOR_FILTER = 0x10
FLAG_FILTER_AUDIT = 0x20
FLAG_GRAM_FILTER = 0x40

STATUS = {
    0: "NDB_OK",
    1: "NDB_ERR_INVALID_ARGUMENT",
    2: "NDB_ERR_UNSUPPORTED_DIM",
    3: "NDB_ERR_INVALID_EPS",
    4: "NDB_ERR_TOO_MANY_POINTS",
    5: "NDB_ERR_OUT_OF_MEMORY",
    6: "NDB_ERR_CUDA",
    7: "NDB_ERR_NO_DEVICE",
    8: "NDB_ERR_DEVICE_LIMIT",
    9: "NDB_ERR_NO_STATE",
    10: "NDB_ERR_BAD_JOB",
    11: "NDB_ERR_IO",
}

# Every symbol include/ndb_b200.h declares (tests check the library exports them).
EXPORTED = (
    "ndb_b200_create",
    "ndb_b200_destroy",
    "ndb_b200_set_stream",
    "ndb_b200_classify",
    "ndb_b200_assign_labels",
    "ndb_b200_run",
    "ndb_b200_load_bin",
    "ndb_b200_run_loaded",
    "ndb_b200_run_batched",
    "ndb_b200_cluster_label",
    "ndb_b200_assign_border",
    "ndb_b200_get_stats",
    "ndb_b200_set_memory_limit",
    "ndb_b200_device_bytes",
    "ndb_b200_set_tuning",
    "ndb_b200_get_tuning",
    "ndb_b200_set_debug_limits",
    "ndb_b200_run_noalloc",
    "ndb_b200_strerror",
    "ndb_b200_last_cuda_error",
    "ndb_b200_version",
)


class NdbResult(ctypes.Structure):
    """nextdbscan::result (nextdbscan.h:43-48)."""

    _fields_ = [("clusters", ctypes.c_int32), ("noise", ctypes.c_int32),
                ("core_count", ctypes.c_int32), ("n", ctypes.c_int32)]


class NdbJob(ctypes.Structure):
    """ndb_job: one independent problem of ndb_b200_run_batched."""

    _fields_ = [("coords", ctypes.c_void_p), ("n", ctypes.c_int64), ("d", ctypes.c_int32),
                ("eps", ctypes.c_float), ("min_pts", ctypes.c_int32), ("nn_out", ctypes.c_void_p),
                ("cluster_index_out", ctypes.c_void_p), ("result", NdbResult), ("status", ctypes.c_int32)]


class NdbTuning(ctypes.Structure):
    """ndb_tuning: count-kernel thresholds of a context (0 = library default)."""

    _fields_ = [("tc_min_dim", ctypes.c_int32), ("tc_min_item", ctypes.c_int32), ("gram_filter", ctypes.c_int32)]


class NdbStats(ctypes.Structure):
    _fields_ = [
        ("n_valid", ctypes.c_int64),
        ("n_cells", ctypes.c_int64),
        ("n_tiles", ctypes.c_int64),
        ("grid_dims", ctypes.c_int32),
        ("stencil_rows", ctypes.c_int32),
        ("same_cell_linked", ctypes.c_int32),
        ("key_bits", ctypes.c_int32),
        ("count_pairs", ctypes.c_int64),
        ("union_pairs", ctypes.c_int64),
        ("border_pairs", ctypes.c_int64),
        ("ms_grid", ctypes.c_float),
        ("ms_count", ctypes.c_float),
        ("ms_union", ctypes.c_float),
        ("ms_border", ctypes.c_float),
        ("ms_sort_kernels", ctypes.c_float),
        ("ms_count_kernel", ctypes.c_float),
        ("ms_union_kernel", ctypes.c_float),
        ("ms_border_kernel", ctypes.c_float),
        ("sort_passes", ctypes.c_int32),
        ("key_bytes", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int32),
        ("pipelines", ctypes.c_int32),
        ("count_pair_dims", ctypes.c_int64),
        ("union_pair_dims", ctypes.c_int64),
        ("border_pair_dims", ctypes.c_int64),
        ("solo_jobs", ctypes.c_int32),
        ("tensor_filter", ctypes.c_int32),
        ("band_pairs", ctypes.c_int64),
        ("tensor_items", ctypes.c_int64),
        ("filter_max_abs_err", ctypes.c_double),
        ("filter_max_err_over_bound", ctypes.c_double),
        ("filter_audited_pairs", ctypes.c_int64),
        ("filter_misclassified_pairs", ctypes.c_int64),
        ("count_fp32_ops", ctypes.c_int64),
        ("gram_filter", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class NdbError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


_lib = None
_lock = threading.Lock()


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads libndb_b200.so and declares the C signatures."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise RuntimeError(
                f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(p)
        c_void_pp = ctypes.POINTER(ctypes.c_void_p)
        i32p = ctypes.c_void_p  # host or device int32 buffers are passed as raw addresses
        lib.ndb_b200_create.argtypes = [c_void_pp, ctypes.c_int32]
        lib.ndb_b200_destroy.argtypes = [ctypes.c_void_p]
        lib.ndb_b200_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ndb_b200_classify.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                          ctypes.c_float, ctypes.c_int32, ctypes.c_uint32, i32p]
        lib.ndb_b200_assign_labels.argtypes = [ctypes.c_void_p, i32p, ctypes.POINTER(NdbResult)]
        lib.ndb_b200_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                     ctypes.c_float, ctypes.c_int32, ctypes.c_uint32, i32p, i32p,
                                     ctypes.POINTER(NdbResult)]
        lib.ndb_b200_load_bin.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int32)]
        lib.ndb_b200_run_loaded.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_int32, ctypes.c_uint32, i32p,
                                            i32p, ctypes.POINTER(NdbResult)]
        lib.ndb_b200_run_batched.argtypes = [ctypes.c_void_p, ctypes.POINTER(NdbJob), ctypes.c_int64,
                                             ctypes.c_uint32]
        lib.ndb_b200_cluster_label.argtypes = [ctypes.c_void_p, i32p, ctypes.c_int64]
        lib.ndb_b200_assign_border.argtypes = [ctypes.c_void_p, i32p, i32p]
        lib.ndb_b200_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(NdbStats)]
        lib.ndb_b200_set_memory_limit.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        lib.ndb_b200_device_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
        lib.ndb_b200_set_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(NdbTuning)]
        lib.ndb_b200_get_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(NdbTuning)]
        lib.ndb_b200_set_debug_limits.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        lib.ndb_b200_strerror.argtypes = [ctypes.c_int]
        lib.ndb_b200_strerror.restype = ctypes.c_char_p
        lib.ndb_b200_last_cuda_error.argtypes = [ctypes.c_void_p]
        lib.ndb_b200_last_cuda_error.restype = ctypes.c_char_p
        lib.ndb_b200_version.restype = ctypes.c_char_p
        for name in ("ndb_b200_create", "ndb_b200_destroy", "ndb_b200_set_stream", "ndb_b200_classify",
                     "ndb_b200_assign_labels", "ndb_b200_run", "ndb_b200_run_batched", "ndb_b200_cluster_label",
                     "ndb_b200_assign_border", "ndb_b200_load_bin", "ndb_b200_run_loaded",
                     "ndb_b200_get_stats", "ndb_b200_set_memory_limit", "ndb_b200_device_bytes",
                     "ndb_b200_set_tuning", "ndb_b200_get_tuning", "ndb_b200_set_debug_limits"):
            getattr(lib, name).restype = ctypes.c_int
        _lib = lib
        return lib


def check(status: int, where: str, ctx: int | None = None) -> None:
    if status == 0:
        return
    detail = ""
    lib = load()
    if ctx:
        detail = (lib.ndb_b200_last_cuda_error(ctx) or b"").decode()
    raise NdbError(status, where, detail)
