"""ndb_b200_run_noalloc: the entry point for callers that may not allocate device
memory (a service that reserves its GPU memory at start-up, a host that only lends
out buffers it owns).  Its scratch is a fixed array inside the library, so its
results must equal ndb_b200_run's on the same inputs, call after call, even though
every call reuses that array.

Collected last on purpose, and self-contained: it passes alone in a fresh process
and after the rest of the suite."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden, load_pkg

pytestmark = pytest.mark.gpu


def noalloc_fn(lib):
    f = lib.ndb_b200_run_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_int32, ctypes.c_uint32,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def run_both(pkg, ctx, fn, x_np, eps, m, full, tensor=False):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(x_np)).cuda()
    n, d = x.shape
    outs = {}
    for which in ("existing", "noalloc"):
        nn = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        ci = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        if which == "existing":
            r = ctx.run_device(x.data_ptr(), n, d, eps, m, nn.data_ptr(), ci.data_ptr(), full_count=full,
                               tensor_filter=tensor)
            meta = (r.clusters, r.noise, r.core_count, r.n)
        else:
            res = pkg.lib.NdbResult()
            flags = (pkg.lib.FLAG_DEVICE_PTRS | (pkg.lib.FLAG_FULL_COUNT if full else 0)
                     | (pkg.lib.FLAG_TENSOR_FILTER if tensor else 0))
            st = fn(ctypes.c_void_p(x.data_ptr()), n, d, ctypes.c_float(eps), m, flags,
                    ctypes.c_void_p(nn.data_ptr()), ctypes.c_void_p(ci.data_ptr()), ctypes.byref(res),
                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert st == 0, pkg.lib.STATUS.get(st, st)
            meta = (res.clusters, res.noise, res.core_count, res.n)
        torch.cuda.synchronize()
        outs[which] = (nn.cpu().numpy(), ci.cpu().numpy(), meta)
    return outs


def test_noalloc_matches_existing_entry_point_on_consecutive_calls():
    pkg = load_pkg()
    lib = pkg.lib.load()
    fn = noalloc_fn(lib)
    cases = [load_golden("c2_n6000"), load_golden("blobs_d8"), load_golden("c1_n4000")]
    with pkg.Context(0) as ctx:
        for g in cases:  # consecutive calls, each reusing the shared array
            for full in (True, False):
                m = int(g["min_pts"])
                o = run_both(pkg, ctx, fn, g["coords"], float(g["eps"]), m, full)
                if full:
                    np.testing.assert_array_equal(o["noalloc"][0], o["existing"][0])  # exact, like every parity test
                else:  # early exit: a core's count only says ">= min_pts", and the two count kernels stop apart
                    below = o["existing"][0] < m
                    np.testing.assert_array_equal(o["noalloc"][0][below], o["existing"][0][below])
                    assert (o["noalloc"][0][~below] >= m).all()
                np.testing.assert_array_equal(o["noalloc"][1], o["existing"][1])
                assert o["noalloc"][2] == o["existing"][2]
                if full:
                    np.testing.assert_array_equal(o["noalloc"][0], g["nn"])
                np.testing.assert_array_equal(o["noalloc"][1], g["cluster_index"])


def test_noalloc_at_its_maximum_and_beyond():
    import torch
    pkg = load_pkg()
    lib = pkg.lib.load()
    fn = noalloc_fn(lib)
    cap = 32768
    w = pkg.synthetic.config1(n=cap)
    with pkg.Context(0) as ctx:
        o = run_both(pkg, ctx, fn, w.coords, w.eps, w.min_pts, True)
        np.testing.assert_array_equal(o["noalloc"][0], o["existing"][0])
        np.testing.assert_array_equal(o["noalloc"][1], o["existing"][1])
    big = torch.zeros((cap + 1, 2), dtype=torch.float32, device="cuda")
    res = pkg.lib.NdbResult()
    st = fn(ctypes.c_void_p(big.data_ptr()), cap + 1, 2, ctypes.c_float(1.0), 4, pkg.lib.FLAG_DEVICE_PTRS, None,
            None, ctypes.byref(res), None)
    assert pkg.lib.STATUS[st] == "NDB_ERR_TOO_MANY_POINTS"


@pytest.mark.parametrize("shape", ["d16_sparse_tensor", "d3_wide_64bit_keys", "d5_sparse", "d7_sparse"])
def test_noalloc_at_its_maximum_on_the_largest_slices(shape):
    """Jobs of exactly the maximum size that fill the slices sized from bounds: one
    cell per point (cells, items, hash table and row table at their bounds), 64-bit
    keys, the 27-row stencil of four gridded dimensions, and the tensor-core count's
    item lists at d = 16."""
    pkg = load_pkg()
    lib = pkg.lib.load()
    fn = noalloc_fn(lib)
    cap = 32768
    rng = np.random.default_rng(77)
    tensor = False
    if shape == "d16_sparse_tensor":
        x, eps, m, tensor = rng.uniform(0, 100, (cap, 16)), 2.0, 4, True
    elif shape == "d3_wide_64bit_keys":
        x, eps, m = rng.uniform(0, 2000, (cap, 3)), 1.0, 2
    elif shape == "d5_sparse":
        x, eps, m = rng.uniform(0, 100, (cap, 5)), 6.0, 3
    else:
        x, eps, m = rng.uniform(0, 100, (cap, 7)), 5.0, 3
    x = x.astype(np.float32)
    with pkg.Context(0) as ctx:
        for _ in range(2):  # two calls in a row on the shared array
            o = run_both(pkg, ctx, fn, x, eps, m, True, tensor=tensor)
            s = ctx.stats()
            np.testing.assert_array_equal(o["noalloc"][0], o["existing"][0])
            np.testing.assert_array_equal(o["noalloc"][1], o["existing"][1])
            assert o["noalloc"][2] == o["existing"][2]
        if shape == "d3_wide_64bit_keys":
            assert s["key_bytes"] == 8 and s["same_cell_linked"] == 1
        if shape == "d16_sparse_tensor":
            assert s["tensor_filter"] == 1
        assert s["n_cells"] > cap // 2  # mostly one point per cell: the cell-sized slices near their bound
