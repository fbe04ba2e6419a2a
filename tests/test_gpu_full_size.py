"""Parity at the benchmark's full sizes against the pinned cell restatement
(oracle.cells, itself checked against the reference's fixtures, the literal
restatement and the grid restatement in tests/test_oracle.py).

  plain 3-D, 10M points          full counts and early exit, bit for bit
  8-D, 2M points                 the exact FP32 count and the tensor-core filtered
                                 count, each with full counts and early exit
  skewed 2-D, 100M points        early exit (the Zipf clusters hold about 10^6
                                 neighbours per point at their centres, so full
                                 counts are some 10^13 pair tests: no checker
                                 finishes them; core flags, counts below minPts,
                                 every cluster id and the meta are compared)
  4,096-job batch                the whole batch against one call per job, and the
                                 64 largest jobs (2-D to 16-D, up to 200k points)
                                 against the oracle

Counts compare exactly with full counts; with early exit exactly below minPts and
as core flags above it (a core's count only says ">= minPts" there)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def assert_same(nn, ci, res, o, m, early, what):
    nn_o, ci_o, meta = o
    if early:
        below = nn_o < m
        np.testing.assert_array_equal(nn[below], nn_o[below], err_msg=what)
        np.testing.assert_array_equal(nn >= m, nn_o >= m, err_msg=what)
    else:
        np.testing.assert_array_equal(nn, nn_o, err_msg=what)
    np.testing.assert_array_equal(ci, ci_o, err_msg=what)
    assert (res.clusters, res.noise, res.core_count, res.n) == \
        (meta["clusters"], meta["noise"], meta["cores"], meta["n"]), what


@pytest.mark.parametrize("early", [False, True])
def test_plain_3d_10m_against_oracle(ctx, pkg, early):
    w = pkg.synthetic.config2()
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=not early)
    o = oracle.cells(w.coords, w.eps, w.min_pts, early=early)
    assert_same(nn, ci, res, o, w.min_pts, early, f"plain-3d-10m early={early}")


@pytest.mark.parametrize("kernel", ["exact", "tensor"])
@pytest.mark.parametrize("early", [False, True])
def test_8d_2m_against_oracle(ctx, pkg, kernel, early):
    w = pkg.synthetic.config3()
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=not early, exact_count=kernel == "exact",
                          tensor_filter=kernel == "tensor")
    s = ctx.stats()
    assert bool(s["tensor_filter"]) == (kernel == "tensor")
    o = oracle.cells(w.coords, w.eps, w.min_pts, early=early)
    assert_same(nn, ci, res, o, w.min_pts, early, f"8d-2m {kernel} early={early}")


def test_skewed_2d_100m_against_oracle(ctx, pkg):
    w = pkg.synthetic.config5()
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts)
    o = oracle.cells(w.coords, w.eps, w.min_pts, early=True)
    assert_same(nn, ci, res, o, w.min_pts, True, "skew-2d-100m")


def test_batch_4096_jobs_against_single_runs_and_oracle(ctx, pkg):
    jobs = pkg.synthetic.config4()
    assert len(jobs) == 4096
    outs = ctx.run_batched([(j.coords, j.eps, j.min_pts) for j in jobs])
    assert ctx.stats()["pipelines"] >= 4
    for k, (j, (nn, ci, res)) in enumerate(zip(jobs, outs)):
        nn1, ci1, res1 = ctx.run(j.coords, j.eps, j.min_pts)
        below = nn1 < j.min_pts
        np.testing.assert_array_equal(nn[below], nn1[below], err_msg=f"job {k}")
        np.testing.assert_array_equal(nn >= j.min_pts, nn1 >= j.min_pts, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci, ci1, err_msg=f"job {k}")
        assert res == res1, k
    largest = sorted(range(len(jobs)), key=lambda k: -jobs[k].n)[:64]
    assert {jobs[k].d for k in largest} == {2, 3, 8, 16}
    for k in largest:
        j = jobs[k]
        nn, ci, res = outs[k]
        o = oracle.cells(j.coords, j.eps, j.min_pts, early=True)
        assert_same(nn, ci, res, o, j.min_pts, True, f"job {k} (n={j.n}, d={j.d})")
