"""The tensor-core filtered neighbour count (d >= 8) against the exact FP32 kernel
and the oracle.  The filter decides a pair only outside a guard band around eps^2
that bounds its own error; pairs inside it are rechecked with the reference's
arithmetic, so counts, core flags and cluster ids must be bit-identical."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def both(ctx, x, eps, m, full=True):
    nn_t, ci_t, r_t = ctx.run(x, eps, m, full_count=full, tensor_filter=True)
    s_t = ctx.stats()
    nn_e, ci_e, r_e = ctx.run(x, eps, m, full_count=full, exact_count=True)
    s_e = ctx.stats()
    return (nn_t, ci_t, r_t, s_t), (nn_e, ci_e, r_e, s_e)


def same_counts(nn_t, nn_e, m, full):
    """Full counts are exact everywhere; with early exit a core's count only says
    ">= min_pts" (the exact kernel stops at min_pts, the tile kernel after a tile)."""
    if full:
        np.testing.assert_array_equal(nn_t, nn_e)
    else:
        below = nn_e < m
        np.testing.assert_array_equal(nn_t[below], nn_e[below])
        assert (nn_t[~below] >= m).all()


@pytest.mark.parametrize("d", [8, 9, 12, 16])
@pytest.mark.parametrize("seed", [0, 1])
def test_filter_equals_exact_kernel(ctx, d, seed):
    rng = np.random.default_rng(500 + 10 * d + seed)
    k = 12
    c = rng.uniform(0, 20, (k, d))
    x = (c[rng.integers(0, k, 20000)] + rng.normal(0, 0.8, (20000, d))).astype(np.float32)
    x = np.concatenate([x, rng.uniform(0, 20, (1500, d)).astype(np.float32)])
    eps = float(0.45 * np.sqrt(d))
    for m in (2, 8, 2 * d):
        for full in (True, False):
            (nn_t, ci_t, r_t, s_t), (nn_e, ci_e, r_e, s_e) = both(ctx, x, eps, m, full)
            assert s_t["tensor_filter"] == 1 and s_e["tensor_filter"] == 0
            same_counts(nn_t, nn_e, m, full)
            np.testing.assert_array_equal(ci_t, ci_e)
            assert r_t == r_e


def test_filter_against_oracle_8d(ctx, pkg):
    w = pkg.synthetic.config3(n=40_000)
    nn_o, ci_o, meta = oracle.grid(w.coords, w.eps, w.min_pts)
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=True, tensor_filter=True)
    assert ctx.stats()["tensor_filter"] == 1
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(ci, ci_o)
    assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])


def test_pairs_exactly_at_eps_go_through_the_band(ctx):
    """An integer lattice with eps = 1: every axis neighbour is at distance exactly
    eps, so the filter cannot decide those pairs and the exact recheck must."""
    g = np.stack(np.meshgrid(*[np.arange(3)] * 8, indexing="ij"), -1).reshape(-1, 8).astype(np.float32)
    x = np.concatenate([g, g + np.float32(0.5)]).astype(np.float32)
    for m in (3, 9, 17):
        (nn_t, ci_t, r_t, s_t), (nn_e, ci_e, r_e, s_e) = both(ctx, x, 1.0, m)
        assert s_t["band_pairs"] > 0
        np.testing.assert_array_equal(nn_t, nn_e)
        np.testing.assert_array_equal(ci_t, ci_e)
        nn_o, ci_o, _ = oracle.grid(x, 1.0, m)
        np.testing.assert_array_equal(nn_t, nn_o)
        np.testing.assert_array_equal(ci_t, ci_o)


def test_far_from_origin_and_tiny_eps(ctx):
    """Coordinates around 1e6 with eps 0.05: the centring on each item keeps the
    Gram terms small; results equal the exact kernel's."""
    rng = np.random.default_rng(7)
    base = np.float32(1e6)
    x = (base + rng.normal(0, 0.02, (6000, 10))).astype(np.float32)
    x[:3000, 0] += np.float32(3.0)
    (nn_t, ci_t, r_t, s_t), (nn_e, ci_e, r_e, s_e) = both(ctx, x, 0.05, 5)
    assert s_t["tensor_filter"] == 1
    np.testing.assert_array_equal(nn_t, nn_e)
    np.testing.assert_array_equal(ci_t, ci_e)


def test_huge_coordinates_take_the_exact_kernel(ctx):
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (3000, 8)).astype(np.float32)
    x[0, 3] = np.float32(2.0 ** 70)
    nn, ci, res = ctx.run(x, 1.5, 4, full_count=True, tensor_filter=True)
    assert ctx.stats()["tensor_filter"] == 0
    nn_o, ci_o, _ = oracle.grid(x, 1.5, 4)
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(ci, ci_o)


def test_batched_tensor_filter_equals_exact(ctx, pkg):
    jobs = pkg.synthetic.config4(n_jobs=40, seed=31, n_min=300, n_max=9000, dims=(8, 16))
    probs = [(j.coords, j.eps, j.min_pts) for j in jobs]
    a = ctx.run_batched(probs, full_count=True, tensor_filter=True)
    assert ctx.stats()["tensor_filter"] == 1
    b = ctx.run_batched(probs, full_count=True, exact_count=True)
    assert ctx.stats()["tensor_filter"] == 0
    for k, ((nn1, ci1, r1), (nn2, ci2, r2)) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(nn1, nn2, err_msg=f"job {k}")
        np.testing.assert_array_equal(ci1, ci2, err_msg=f"job {k}")
        assert r1 == r2


def test_fill_heuristic_picks_a_kernel_and_results_agree(ctx, pkg):
    """Without either flag the library picks the kernel by tile fill; the three
    settings give one answer."""
    w = pkg.synthetic.config3(n=30_000)
    outs = [ctx.run(w.coords, w.eps, w.min_pts, full_count=True, **kw)
            for kw in ({}, {"exact_count": True}, {"tensor_filter": True})]
    for nn, ci, res in outs[1:]:
        np.testing.assert_array_equal(nn, outs[0][0])
        np.testing.assert_array_equal(ci, outs[0][1])


def test_tuning_and_autotuner(ctx, pkg):
    """Per-context thresholds (ndb_b200_set_tuning) move work between the two count
    kernels without changing a result; the autotuner times every candidate, checks
    they agree, and leaves the fastest on the context."""
    w = pkg.synthetic.config3(n=30_000)
    nn_o, ci_o, _ = oracle.grid(w.coords, w.eps, w.min_pts)
    try:
        r = pkg.autotune.tune_count(ctx, w.coords, w.eps, w.min_pts, full_count=True, reps=2)
        assert r["best"] in pkg.autotune.candidates(8)
        assert ctx.tuning() == r["best"]
        by = {(t["tc_min_dim"], t["tc_min_item"], t["gram_filter"]): t for t in r["table"]}
        assert by[(17, 0, 0)]["tensor_items"] == 0 and by[(17, 0, 1)]["tensor_items"] == 0
        assert by[(8, 1, 0)]["tensor_items"] > 0
        nn, ci, _ = ctx.run(w.coords, w.eps, w.min_pts, full_count=True)
        np.testing.assert_array_equal(nn, nn_o)
        np.testing.assert_array_equal(ci, ci_o)
        # early exit at d = 8: the default threshold (d >= 12) keeps the exact kernel,
        # a tuned tc_min_dim = 8 turns the filter on
        ctx.set_tuning(tc_min_dim=8, tc_min_item=1)
        _, ci, _ = ctx.run(w.coords, w.eps, w.min_pts)
        assert ctx.stats()["tensor_filter"] == 1
        np.testing.assert_array_equal(ci, ci_o)
        ctx.set_tuning(tc_min_dim=17)
        nn, ci, _ = ctx.run(w.coords, w.eps, w.min_pts, full_count=True)
        assert ctx.stats()["tensor_filter"] == 0
        np.testing.assert_array_equal(nn, nn_o)
        with pytest.raises(pkg.lib.NdbError, match="INVALID_ARGUMENT"):
            ctx.set_tuning(tc_min_dim=-1)
    finally:
        ctx.reset_tuning()
    assert ctx.tuning() == {"tc_min_dim": 0, "tc_min_item": 0, "gram_filter": 0}


@pytest.mark.parametrize("full", [True, False])
def test_filter_audit_every_pair_within_its_bound(ctx, pkg, full):
    """NDB_FLAG_FILTER_AUDIT: every pair the filter classified is measured against
    its FP64 distance and the exact FP32 predicate.  None is decided wrongly outside
    the guard band, the error stays inside the bound the band is built from, and the
    audited run gives the unaudited run's outputs."""
    w = pkg.synthetic.config3(n=60_000)
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=full, tensor_filter=True)
    nn_a, ci_a, res_a = ctx.run(w.coords, w.eps, w.min_pts, full_count=full, tensor_filter=True, audit=True)
    s = ctx.stats()
    assert s["tensor_filter"] == 1
    assert s["filter_audited_pairs"] > 0
    assert s["filter_misclassified_pairs"] == 0
    assert 0.0 < s["filter_max_abs_err"] and s["filter_max_err_over_bound"] <= 1.0
    np.testing.assert_array_equal(ci_a, ci)
    if full:
        np.testing.assert_array_equal(nn_a, nn)
    assert res_a == res
