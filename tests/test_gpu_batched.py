"""ndb_b200_run_batched: many independent jobs in one pipeline.  Every job's
outputs must equal what a single ndb_b200_run gives on it (and therefore the
reference's), whatever the other jobs in the batch are."""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden, roots_of

pytestmark = pytest.mark.gpu


def meta_of(res):
    return [res.clusters, res.noise, res.core_count, res.n]


def golden_problems():
    out = []
    for name in golden_names():
        g = load_golden(name)
        e = np.float32(g["eps"])
        if not np.isfinite(np.float32(e * e)):
            continue
        out.append((name, g))
    return out


@pytest.mark.parametrize("full", [True, False])
def test_golden_fixtures_as_one_batch(ctx, full):
    probs = golden_problems()
    outs = ctx.run_batched([(g["coords"], float(g["eps"]), int(g["min_pts"])) for _, g in probs],
                           full_count=full)
    for (name, g), (nn, ci, res) in zip(probs, outs):
        np.testing.assert_array_equal(ci, g["cluster_index"], err_msg=name)
        assert meta_of(res) == list(g["meta"]), name
        m = int(g["min_pts"])
        if full:
            np.testing.assert_array_equal(nn, g["nn"], err_msg=name)
        else:
            below = g["nn"] < m
            np.testing.assert_array_equal(nn[below], g["nn"][below], err_msg=name)
            assert (nn[~below] >= m).all(), name


def test_repeated_runs_give_the_same_ids(ctx):
    """The union-find runs lock-free across SMs, so its timing differs from run to
    run; the ids must not.  The golden batch and each 3-D fixture alone, many times:
    a flatten pass whose root stores another thread could overwrite gave one point
    of this batch a wrong id in about one run of a dozen."""
    probs = golden_problems()
    batch = [(g["coords"], float(g["eps"]), int(g["min_pts"])) for _, g in probs]
    for _ in range(12):
        for (name, g), (_, ci, _) in zip(probs, ctx.run_batched(batch)):
            np.testing.assert_array_equal(ci, g["cluster_index"], err_msg=name)
    for name, g in probs:
        if g["coords"].shape[1] != 3:
            continue
        for _ in range(6):
            _, ci, _ = ctx.run(g["coords"], float(g["eps"]), int(g["min_pts"]))
            np.testing.assert_array_equal(ci, g["cluster_index"], err_msg=name)


def test_batch_equals_single_runs(ctx, pkg):
    jobs = pkg.synthetic.config4(n_jobs=48, seed=11, n_min=200, n_max=6000)
    outs = ctx.run_batched([(j.coords, j.eps, j.min_pts) for j in jobs], full_count=True)
    for k, (j, (nn, ci, res)) in enumerate(zip(jobs, outs)):
        nn1, ci1, res1 = ctx.run(j.coords, j.eps, j.min_pts, full_count=True)
        np.testing.assert_array_equal(nn, nn1, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci, ci1, err_msg=f"job {k}")
        assert res == res1, k


def test_batch_against_oracle(ctx, pkg):
    jobs = pkg.synthetic.config4(n_jobs=24, seed=12, n_min=500, n_max=8000)
    outs = ctx.run_batched([(j.coords, j.eps, j.min_pts) for j in jobs])
    for k, (j, (nn, ci, res)) in enumerate(zip(jobs, outs)):
        nn_o, ci_o, meta = oracle.grid(j.coords, j.eps, j.min_pts)
        np.testing.assert_array_equal(ci, ci_o, err_msg=f"job {k}")
        below = nn_o < j.min_pts
        np.testing.assert_array_equal(nn[below], nn_o[below], err_msg=f"job {k}")
        assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"]), k


def test_batch_device_pointers(ctx, pkg):
    import torch
    jobs = pkg.synthetic.config4(n_jobs=16, seed=13, n_min=300, n_max=5000)
    dev = []
    arr = (pkg.lib.NdbJob * len(jobs))()
    for k, j in enumerate(jobs):
        x = torch.from_numpy(j.coords).cuda()
        nn = torch.full((j.n,), -5, dtype=torch.int32, device="cuda")
        ci = torch.full((j.n,), -5, dtype=torch.int32, device="cuda")
        dev.append((x, nn, ci))
        arr[k].coords, arr[k].n, arr[k].d = x.data_ptr(), j.n, j.d
        arr[k].eps, arr[k].min_pts = j.eps, j.min_pts
        arr[k].nn_out, arr[k].cluster_index_out = nn.data_ptr(), ci.data_ptr()
    torch.cuda.synchronize()
    st = ctx.run_batched_jobs(arr, len(jobs), pkg.lib.FLAG_DEVICE_PTRS | pkg.lib.FLAG_FULL_COUNT)
    assert st == 0, pkg.lib.STATUS.get(st, st)
    torch.cuda.synchronize()
    for k, (j, (x, nn, ci)) in enumerate(zip(jobs, dev)):
        nn1, ci1, res1 = ctx.run(j.coords, j.eps, j.min_pts, full_count=True)
        np.testing.assert_array_equal(nn.cpu().numpy(), nn1, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci.cpu().numpy(), ci1, err_msg=f"job {k}")
        assert arr[k].status == 0
        assert meta_of(arr[k].result) == list(res1), k


def test_bad_jobs_do_not_spoil_the_others(ctx, pkg):
    a = load_golden("c1_n4000")
    b = load_golden("blobs_d3")
    probs = [(a["coords"], float(a["eps"]), int(a["min_pts"])),
             (np.zeros((10, 17), np.float32), 1.0, 2),         # unsupported d
             (b["coords"], float(b["eps"]), int(b["min_pts"])),
             (np.zeros((10, 2), np.float32), 1e20, 2),         # eps*eps overflows
             (np.zeros((0, 3), np.float32), 1.0, 2)]           # empty
    with pytest.raises(pkg.lib.NdbError, match="UNSUPPORTED_DIM"):
        ctx.run_batched(probs)
    jobs = ctx.last_jobs
    st = [pkg.lib.STATUS[jobs[k].status] for k in range(len(probs))]
    assert st == ["NDB_OK", "NDB_ERR_UNSUPPORTED_DIM", "NDB_OK", "NDB_ERR_INVALID_EPS", "NDB_OK"]
    for k, g in ((0, a), (2, b)):
        assert meta_of(jobs[k].result) == list(g["meta"])
    assert meta_of(jobs[4].result) == [0, 0, 0, 0]


def test_jobs_the_pipeline_runs_alone(ctx, pkg):
    """A job whose grid is of the other kind than the first job's (2-D eps so small
    the same-cell-linked grid would overflow its keys), and one whose min_pts is
    above the neighbour-list cap, are run by themselves; results are unchanged."""
    rng = np.random.default_rng(21)
    wide = (rng.uniform(0, 1000, (3000, 2))).astype(np.float32)
    a = load_golden("c1_n4000")
    dense = pkg.synthetic.config1(n=6000)
    probs = [(a["coords"], float(a["eps"]), int(a["min_pts"])),
             (wide, 1e-6, 3),
             (dense.coords, 3.0, 100),
             (a["coords"], float(a["eps"]), 2)]
    outs = ctx.run_batched(probs, full_count=True)
    for k, ((x, e, m), (nn, ci, res)) in enumerate(zip(probs, outs)):
        nn1, ci1, res1 = ctx.run(x, e, m, full_count=True)
        np.testing.assert_array_equal(nn, nn1, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci, ci1, err_msg=f"job {k}")
        assert res == res1, k


def test_batched_cluster_roots_match_reference_labels(ctx):
    """The cluster ids of each job in a batch are exactly the roots of the
    reference's label array (id = core rank of the component's first core)."""
    probs = golden_problems()[:8]
    outs = ctx.run_batched([(g["coords"], float(g["eps"]), int(g["min_pts"])) for _, g in probs])
    for (name, g), (nn, ci, res) in zip(probs, outs):
        ids = np.unique(ci[ci != 2**31 - 1])
        np.testing.assert_array_equal(ids, roots_of(g["cluster_label"]), err_msg=name)


def test_batch_split_to_keep_32_bit_keys(ctx, pkg):
    """Jobs whose cells add up past 2^32 keys run as several pipelines with 32-bit
    keys; the results are still those of one run per job."""
    rng = np.random.default_rng(41)
    probs = []
    for k in range(3):  # about 1.5e9 cells each (3-D, extent 661, eps 1)
        x = rng.uniform(0, 661, (2000, 3)).astype(np.float32)
        x[:200] = (rng.normal(300, 0.4, (200, 3))).astype(np.float32)
        probs.append((x, 1.0, 4))
    a = load_golden("blobs_d3")
    probs.append((a["coords"], float(a["eps"]), int(a["min_pts"])))
    outs = ctx.run_batched(probs, full_count=True)
    s = ctx.stats()
    assert s["pipelines"] >= 2 and s["key_bits"] <= 32 and s["solo_jobs"] == 0
    for k, ((x, e, m), (nn, ci, res)) in enumerate(zip(probs, outs)):
        nn1, ci1, res1 = ctx.run(x, e, m, full_count=True)
        np.testing.assert_array_equal(nn, nn1, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci, ci1, err_msg=f"job {k}")
        assert res == res1, k
