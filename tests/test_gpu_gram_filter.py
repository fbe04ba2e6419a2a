"""The FP32 Gram-filtered count on CUDA cores (d >= 8): centred dot products decide
a pair outside a guard band that bounds their error, and the reference's own FP32
sum decides the pairs inside it.  It runs when asked for (NDB_FLAG_GRAM_FILTER, or a
context's tuning); the plain form (NDB_FLAG_EXACT_COUNT) never uses it.  Counts, core flags,
cluster ids and meta must be bit-identical to the exact kernel's and the oracle's,
including pairs exactly at eps, coordinates far from the origin, tiny eps, and
special values."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def both(ctx, x, eps, m, full=True):
    nn_g, ci_g, r_g = ctx.run(x, eps, m, full_count=full, gram_filter=True)
    s_g = ctx.stats()
    nn_e, ci_e, r_e = ctx.run(x, eps, m, full_count=full, exact_count=True)
    s_e = ctx.stats()
    return (nn_g, ci_g, r_g, s_g), (nn_e, ci_e, r_e, s_e)


def same(g, e, m, full):
    (nn_g, ci_g, r_g, s_g), (nn_e, ci_e, r_e, s_e) = g, e
    if full:
        np.testing.assert_array_equal(nn_g, nn_e)
    else:
        below = nn_e < m
        np.testing.assert_array_equal(nn_g[below], nn_e[below])
        np.testing.assert_array_equal(nn_g >= m, nn_e >= m)
    np.testing.assert_array_equal(ci_g, ci_e)
    assert r_g == r_e


@pytest.mark.parametrize("d", [8, 11, 16])
@pytest.mark.parametrize("full", [True, False])
def test_gram_equals_exact_kernel(ctx, d, full):
    rng = np.random.default_rng(900 + d)
    k = 10
    c = rng.uniform(0, 20, (k, d))
    x = (c[rng.integers(0, k, 25000)] + rng.normal(0, 0.8, (25000, d))).astype(np.float32)
    x = np.concatenate([x, rng.uniform(0, 20, (2000, d)).astype(np.float32)])
    eps = float(0.45 * np.sqrt(d))
    for m in (2, 8, 2 * d):
        g, e = both(ctx, x, eps, m, full)
        assert g[3]["gram_filter"] == 1 and e[3]["gram_filter"] == 0
        same(g, e, m, full)


def test_gram_against_oracle_8d(ctx, pkg):
    w = pkg.synthetic.config3(n=60_000)
    nn_o, ci_o, meta = oracle.cells(w.coords, w.eps, w.min_pts)
    nn, ci, res = ctx.run(w.coords, w.eps, w.min_pts, full_count=True, gram_filter=True)
    assert ctx.stats()["gram_filter"] == 1
    np.testing.assert_array_equal(nn, nn_o)
    np.testing.assert_array_equal(ci, ci_o)
    assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])


def test_gram_lattice_pairs_exactly_at_eps(ctx):
    """Every axis neighbour of the lattice sits exactly at eps: only the band's
    exact recheck can decide them."""
    g = np.stack(np.meshgrid(*[np.arange(3)] * 8, indexing="ij"), -1).reshape(-1, 8).astype(np.float32)
    x = np.concatenate([g, g + np.float32(0.5)]).astype(np.float32)
    for m in (3, 9, 17):
        gg, e = both(ctx, x, 1.0, m)
        assert gg[3]["band_pairs"] > 0
        same(gg, e, m, True)
        nn_o, ci_o, _ = oracle.grid(x, 1.0, m)
        np.testing.assert_array_equal(gg[0], nn_o)
        np.testing.assert_array_equal(gg[1], ci_o)


@pytest.mark.parametrize("scale,eps", [(1e6, 0.05), (1e-20, 3e-21), (3e4, 40.0)])
def test_gram_far_from_origin_tiny_and_wide(ctx, scale, eps):
    rng = np.random.default_rng(3)
    x = (np.float32(scale) * (1 + 0.01 * rng.normal(0, 1, (5000, 9)))).astype(np.float32)
    if scale < 1:
        x = (rng.normal(0, 1, (5000, 9)) * scale).astype(np.float32)
    for full in (True, False):
        g, e = both(ctx, x, eps, 5, full)
        same(g, e, 5, full)


def test_gram_with_special_values(ctx):
    rng = np.random.default_rng(4)
    x = rng.normal(0, 1, (4000, 8)).astype(np.float32)
    x[::50, 3] = np.nan
    x[::70, 0] = np.finfo(np.float32).max
    x[::90, 5] = -np.inf
    for m in (0, 1, 6):
        g, e = both(ctx, x, 1.7, m)
        same(g, e, m, True)
        nn_o, ci_o, _ = oracle.grid(x, 1.7, m)
        np.testing.assert_array_equal(g[0], nn_o)
        np.testing.assert_array_equal(g[1], ci_o)


def test_gram_in_batches(ctx, pkg):
    jobs = pkg.synthetic.config4(n_jobs=40, seed=31, n_min=500, n_max=9000, dims=(8, 16))
    outs = ctx.run_batched([(j.coords, j.eps, j.min_pts) for j in jobs], full_count=True, gram_filter=True)
    assert ctx.stats()["gram_filter"] == 1
    for j, (nn, ci, res) in zip(jobs, outs):
        nn_e, ci_e, r_e = ctx.run(j.coords, j.eps, j.min_pts, full_count=True, exact_count=True)
        np.testing.assert_array_equal(nn, nn_e)
        np.testing.assert_array_equal(ci, ci_e)


def test_gram_through_the_tuning(ctx):
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (6000, 10)).astype(np.float32)
    ctx.set_tuning(tc_min_dim=17, gram_filter=1)
    try:
        nn, ci, _ = ctx.run(x, 1.9, 6, full_count=True)
        assert ctx.stats()["gram_filter"] == 1
    finally:
        ctx.reset_tuning()
    nn_e, ci_e, _ = ctx.run(x, 1.9, 6, full_count=True, exact_count=True)
    np.testing.assert_array_equal(nn, nn_e)
    np.testing.assert_array_equal(ci, ci_e)
