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


def run_both(pkg, ctx, fn, x_np, eps, m, full):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(x_np)).cuda()
    n, d = x.shape
    outs = {}
    for which in ("existing", "noalloc"):
        nn = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        ci = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        if which == "existing":
            r = ctx.run_device(x.data_ptr(), n, d, eps, m, nn.data_ptr(), ci.data_ptr(), full_count=full)
            meta = (r.clusters, r.noise, r.core_count, r.n)
        else:
            res = pkg.lib.NdbResult()
            flags = pkg.lib.FLAG_DEVICE_PTRS | (pkg.lib.FLAG_FULL_COUNT if full else 0)
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
