"""GPU parity: the CUDA path through the C ABI against the reference's outputs
(golden fixtures), against the oracle at sizes it finishes in seconds, and
through size-independent properties at the full benchmark sizes.

Bar: bit-exact for counts, core flags and cluster ids (integer work on the
reference's exact FP32 predicate)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, golden_names, load_golden, roots_of

pytestmark = pytest.mark.gpu
NAMES = golden_names()
NO_CLUSTER = 2**31 - 1


def meta_of(res):
    return [res.clusters, res.noise, res.core_count, res.n]


@pytest.mark.parametrize("name", NAMES)
def test_golden_full_count(ctx, name):
    g = load_golden(name)
    nn, ci, res = ctx.run(g["coords"], float(g["eps"]), int(g["min_pts"]), full_count=True)
    np.testing.assert_array_equal(nn, g["nn"])
    np.testing.assert_array_equal(ci, g["cluster_index"])
    assert meta_of(res) == list(g["meta"])
    lab = ctx.cluster_label(res.core_count)
    np.testing.assert_array_equal(roots_of(lab), roots_of(g["cluster_label"]))


@pytest.mark.parametrize("name", NAMES)
def test_golden_early_exit(ctx, name):
    """Default mode: counts stop at min_pts; exact below it, core flags and labels exact."""
    g = load_golden(name)
    m = int(g["min_pts"])
    nn, ci, res = ctx.run(g["coords"], float(g["eps"]), m)
    ref = g["nn"]
    below = ref < m
    np.testing.assert_array_equal(nn[below], ref[below])
    assert (nn[~below] >= m).all()
    np.testing.assert_array_equal(ci, g["cluster_index"])
    assert meta_of(res) == list(g["meta"])


@pytest.mark.parametrize("name", NAMES)
def test_golden_approximate_flag(ctx, name):
    """-a 1: cores and noise equal the reference's approximate run; the cluster count
    is the exact one, hence within the reference's upper bound."""
    g = load_golden(name)
    nn, ci, res = ctx.run(g["coords"], float(g["eps"]), int(g["min_pts"]), approximate=True)
    am = g["approx_meta"]
    assert res.core_count == am[2] and res.noise == am[1]
    assert res.clusters <= am[0]
    np.testing.assert_array_equal(ci, g["cluster_index"])


def test_data_process_mirror(pkg):
    g = load_golden("c1_n4000")
    x = g["coords"]
    dp = pkg.data_process(x.ravel(), int(g["min_pts"]), float(g["eps"]), x.shape[1], x.shape[0], False)
    dp.select_and_process(None)
    dp.select_cores_and_process(None)
    cores, noise, clusters, n = dp.get_result_meta(None)
    assert [clusters, noise, cores, n] == list(g["meta"])
    np.testing.assert_array_equal(dp.v_coord_nn, g["nn"])
    np.testing.assert_array_equal(dp.v_coord_cluster_index, g["cluster_index"])
    np.testing.assert_array_equal(roots_of(dp.v_cluster_label), roots_of(g["cluster_label"]))


def test_start_reads_bin(pkg, tmp_path):
    g = load_golden("blobs_d3")
    p = str(tmp_path / "in.bin")
    pkg.inputs.write_bin(p, g["coords"])
    r = pkg.start(int(g["min_pts"]), float(g["eps"]), 1, p, verbose=False)
    assert [r.clusters, r.noise, r.core_count, r.n] == list(g["meta"])


def test_c1_full_against_reference_hashes(ctx, pkg):
    with open(os.path.join(GOLDEN, "c1_full.json")) as f:
        doc = json.load(f)
    w = pkg.synthetic.config1()
    assert hashlib.sha256(w.coords.astype("<f4").tobytes()).hexdigest() == doc["coords_sha256"]
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=True)
    assert hashlib.sha256(nn.astype("<i4").tobytes()).hexdigest() == doc["nn_sha256"]
    assert hashlib.sha256(ci.astype("<i4").tobytes()).hexdigest() == doc["cluster_index_sha256"]
    assert (res.clusters, res.noise, res.core_count) == (doc["clusters"], doc["noise"], doc["cores"])
    _, ci2, _ = ctx.run(w.coords, w.eps, w.min_pts)
    np.testing.assert_array_equal(ci2, ci)


ORACLE_CASES = [
    ("c2_200k", 2, 200_000, None),
    ("c3_40k", 3, 40_000, None),
    ("c5_200k", 5, 200_000, None),
]


@pytest.mark.parametrize("name,config,n,m", ORACLE_CASES)
def test_seeded_against_oracle(ctx, pkg, name, config, n, m):
    w = pkg.synthetic.make(config, n=n)
    mp = m or w.min_pts
    nn_o, ci_o, meta = oracle.grid(w.coords, w.eps, mp)
    nn, ci, res = ctx.run(w.coords, w.eps, mp, full_count=True)
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(ci, ci_o)
    assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])


@pytest.mark.parametrize("d", list(range(1, 17)))
def test_every_dimensionality_against_oracle(ctx, d):
    rng = np.random.default_rng(1000 + d)
    k = 8
    c = rng.uniform(0, 12, (k, d))
    lab = rng.integers(0, k, 6000)
    x = (c[lab] + rng.normal(0, 0.5, (6000, d))).astype(np.float32)
    x = np.concatenate([x, rng.uniform(0, 12, (500, d)).astype(np.float32)])
    eps = float(0.35 * np.sqrt(d))
    for m in (1, 4, 12):
        nn_o, ci_o, meta = oracle.grid(x, eps, m)
        nn, ci, res = ctx.run(x, eps, m, full_count=True)
        np.testing.assert_array_equal(nn, nn_o)
        np.testing.assert_array_equal(ci, ci_o)
        _, ci_e, res_e = ctx.run(x, eps, m)
        np.testing.assert_array_equal(ci_e, ci_o)
        assert res_e == res


def test_device_pointer_path(ctx, pkg):
    import torch
    g = load_golden("c2_n6000")
    x = torch.from_numpy(g["coords"]).cuda()
    n, d = x.shape
    nn = torch.empty(n, dtype=torch.int32, device="cuda")
    ci = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    res = ctx.run_device(x.data_ptr(), n, d, float(g["eps"]), int(g["min_pts"]), nn.data_ptr(), ci.data_ptr(),
                         full_count=True)
    np.testing.assert_array_equal(nn.cpu().numpy(), g["nn"])
    np.testing.assert_array_equal(ci.cpu().numpy(), g["cluster_index"])
    assert meta_of(res) == list(g["meta"])


def test_pinned_host_buffers(ctx, pkg):
    """Pinned host outputs: the count copy runs on its own stream, overlapping the
    label phase; the call returns only when both outputs are complete."""
    import torch
    w = pkg.synthetic.config2(n=200_000)
    n, d = w.coords.shape
    hx = torch.from_numpy(w.coords).pin_memory()
    nn_o, ci_o, meta = oracle.grid(w.coords, w.eps, w.min_pts)
    for rep in range(3):
        for full in (True, False):
            hnn = torch.full((n,), -7, dtype=torch.int32).pin_memory()
            hci = torch.full((n,), -7, dtype=torch.int32).pin_memory()
            res = ctx.run_ptrs(hx.data_ptr(), n, d, w.eps, w.min_pts, hnn.data_ptr(), hci.data_ptr(), device=False,
                               full_count=full)
            nn, ci = hnn.numpy(), hci.numpy()
            np.testing.assert_array_equal(ci, ci_o)
            if full:
                np.testing.assert_array_equal(nn, nn_o)
            else:
                below = nn_o < w.min_pts
                np.testing.assert_array_equal(nn[below], nn_o[below])
                assert (nn[~below] >= w.min_pts).all()
            assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])


def test_error_statuses(ctx, pkg):
    x = np.zeros((10, 17), np.float32)
    with pytest.raises(pkg.lib.NdbError, match="UNSUPPORTED_DIM"):
        ctx.run(x, 1.0, 2)
    with pytest.raises(pkg.lib.NdbError, match="INVALID_EPS"):
        ctx.run(np.zeros((10, 2), np.float32), 1e20, 2)
    with pytest.raises(pkg.lib.NdbError, match="INVALID_EPS"):
        ctx.run(np.zeros((10, 2), np.float32), float("nan"), 2)
    nn, ci, res = ctx.run(np.zeros((0, 3), np.float32), 1.0, 2)
    assert res == (0, 0, 0, 0) and nn.size == 0
    fresh = pkg.Context(0)
    with pytest.raises(pkg.lib.NdbError, match="NO_STATE"):
        fresh.assign_labels()
    fresh.close()


def test_context_reuse_grows_and_shrinks(ctx, pkg):
    a = load_golden("blobs_d2")
    b = pkg.synthetic.config1(n=50_000)
    for _ in range(2):
        nn, ci, res = ctx.run(a["coords"], float(a["eps"]), int(a["min_pts"]), full_count=True)
        np.testing.assert_array_equal(ci, a["cluster_index"])
        ctx.run(b.coords, b.eps, b.min_pts)


def partition_key(ci):
    """Canonical form of a labelling: ids renumbered by first appearance."""
    _, first, inv = np.unique(ci, return_index=True, return_inverse=True)
    order = np.argsort(np.argsort(first))
    out = order[inv]
    out[ci == NO_CLUSTER] = -1
    return out


def brute_nn(x, idx, e2):
    """Exact FP32 counts for a few points, in numpy with the reference's operation order."""
    out = []
    for i in idx:
        length = np.zeros(x.shape[0], np.float32)
        for k in range(x.shape[1]):
            t = x[:, k] - x[i, k]
            length = length + t * t
        out.append(int(np.count_nonzero(length <= e2)))
    return np.array(out)


def test_full_size_plain_3d_properties(ctx, pkg):
    """n=10M 3-D (the benchmark workload): oracle-free properties."""
    w = pkg.synthetic.config2()
    x, eps, m = w.coords, w.eps, w.min_pts
    e2 = np.float32(np.float32(eps) * np.float32(eps))
    nn_f, ci_f, res_f = ctx.run(x, eps, m, full_count=True)
    nn_e, ci_e, res_e = ctx.run(x, eps, m)
    np.testing.assert_array_equal(ci_e, ci_f)  # early exit changes nothing but saturated counts
    assert res_e == res_f
    core = nn_f >= m
    np.testing.assert_array_equal(core, nn_e >= m)
    below = nn_f < m
    np.testing.assert_array_equal(nn_e[below], nn_f[below])
    # cluster ids are core ranks of each component's smallest core
    rank = np.cumsum(core) - 1
    ids = np.unique(ci_f[ci_f != NO_CLUSTER])
    assert ids.size == res_f.clusters
    core_idx = np.nonzero(core)[0]
    np.testing.assert_array_equal(ci_f[core_idx[ids]], ids)
    assert (ci_f[core] <= rank[core]).all()
    assert res_f.noise == int(np.count_nonzero(ci_f == NO_CLUSTER))
    # exact counts of a sample of points
    rng = np.random.default_rng(5)
    idx = rng.choice(x.shape[0], 24, replace=False)
    np.testing.assert_array_equal(nn_f[idx], brute_nn(x, idx, e2))
    # input order changes ids, never the partition
    perm = rng.permutation(x.shape[0])
    _, ci_p, res_p = ctx.run(x[perm], eps, m)
    assert (res_p.clusters, res_p.noise, res_p.core_count) == (res_f.clusters, res_f.noise, res_f.core_count)
    core_p = core[perm]
    np.testing.assert_array_equal(partition_key(ci_p[core_p]), partition_key(ci_f[perm][core_p]))


def test_outputs_larger_than_l2_match_the_batched_path(ctx, pkg):
    """Above 24M points the input-order outputs are scattered in destination
    windows (several passes).  The batched entry point writes through its own
    single-pass path; on one job both must agree exactly."""
    w = pkg.synthetic.config1(n=30_000_000)
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts)
    (nn_b, ci_b, res_b), = ctx.run_batched([(w.coords, w.eps, w.min_pts)])
    np.testing.assert_array_equal(nn, nn_b)
    np.testing.assert_array_equal(ci, ci_b)
    assert res == res_b
    assert res.noise == int(np.count_nonzero(ci == NO_CLUSTER))
