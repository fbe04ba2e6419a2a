"""The oracle is pinned to the reference before anything is checked against it.

Every fixture under tests/golden/ holds outputs of nextdbscan-exa's own OpenMP
implementation (made by tests/golden/make_golden.py); both C restatements must
reproduce them bit for bit.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, golden_names, load_golden, roots_of

NAMES = golden_names()


def test_golden_present():
    assert len(NAMES) >= 20
    assert os.path.exists(os.path.join(GOLDEN, "c1_full.json"))


@pytest.mark.parametrize("name", NAMES)
def test_literal_restatement_matches_reference(name):
    g = load_golden(name)
    nn, ci, lab, meta = oracle.reference(g["coords"], float(g["eps"]), int(g["min_pts"]))
    np.testing.assert_array_equal(nn, g["nn"])
    np.testing.assert_array_equal(ci, g["cluster_index"])
    np.testing.assert_array_equal(roots_of(lab), roots_of(g["cluster_label"]))
    assert [meta["clusters"], meta["noise"], meta["cores"], meta["n"]] == list(g["meta"])


@pytest.mark.parametrize("name", NAMES)
def test_literal_restatement_matches_reference_approximate(name):
    """-a 1 (data_process.cpp:215-217) is schedule dependent; pinned single threaded."""
    g = load_golden(name)
    nn, ci, lab, meta = oracle.reference(g["coords"], float(g["eps"]), int(g["min_pts"]), approximate=True)
    np.testing.assert_array_equal(ci, g["approx_cluster_index"])
    np.testing.assert_array_equal(roots_of(lab), roots_of(g["approx_cluster_label"]))
    assert [meta["clusters"], meta["noise"], meta["cores"], meta["n"]] == list(g["approx_meta"])


@pytest.mark.parametrize("name", NAMES)
def test_grid_restatement_matches_reference(name):
    g = load_golden(name)
    e = np.float32(g["eps"])
    if not np.isfinite(np.float32(e * e)):
        pytest.skip("grid restatement needs a finite eps*eps")
    nn, ci, meta = oracle.grid(g["coords"], float(e), int(g["min_pts"]))
    np.testing.assert_array_equal(nn, g["nn"])
    np.testing.assert_array_equal(ci, g["cluster_index"])
    assert [meta["clusters"], meta["noise"], meta["cores"], meta["n"]] == list(g["meta"])


def test_grid_restatement_matches_reference_full_c1(pkg):
    """100,000-point 2-D workload against hashes of the reference's own outputs."""
    with open(os.path.join(GOLDEN, "c1_full.json")) as f:
        doc = json.load(f)
    w = pkg.synthetic.config1()
    assert hashlib.sha256(w.coords.astype("<f4").tobytes()).hexdigest() == doc["coords_sha256"], \
        "generator drift: synthetic.config1 no longer reproduces the fixture input"
    nn, ci, meta = oracle.grid(w.coords, w.eps, w.min_pts)
    assert hashlib.sha256(nn.astype("<i4").tobytes()).hexdigest() == doc["nn_sha256"]
    assert hashlib.sha256(ci.astype("<i4").tobytes()).hexdigest() == doc["cluster_index_sha256"]
    assert (meta["clusters"], meta["noise"], meta["cores"]) == (doc["clusters"], doc["noise"], doc["cores"])


def test_grid_matches_literal_random():
    """Extra agreement between the two restatements on unseeded shapes."""
    rng = np.random.default_rng(99)
    for d in (1, 2, 3, 6, 12):
        x = (rng.uniform(0, 8, (1200, d)) + rng.normal(0, 0.2, (1200, d))).astype(np.float32)
        for eps, m in ((0.5, 3), (1.0, 6)):
            a = oracle.reference(x, eps, m)
            b = oracle.grid(x, eps, m)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])


def test_oracle_planted_mistake_is_caught():
    """A wrong answer planted in the oracle's output is detected by the comparison."""
    g = load_golden("c1_n4000")
    nn, ci, meta = oracle.grid(g["coords"], float(g["eps"]), int(g["min_pts"]))
    bad = ci.copy()
    i = int(np.nonzero(bad != oracle.NO_CLUSTER)[0][0])
    bad[i] += 1
    assert not np.array_equal(bad, g["cluster_index"])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built here")
def test_reference_harness_reproduces_fixture():
    g = load_golden("blobs_d3")
    nn, ci, lab, info = oracle.run_ref(g["coords"], float(g["eps"]), int(g["min_pts"]), threads=2)
    np.testing.assert_array_equal(nn, g["nn"])
    np.testing.assert_array_equal(ci, g["cluster_index"])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built here")
def test_grid_restatement_matches_reference_harness_random():
    """Beyond the fixtures: the grid restatement against the reference's own build on
    seeded random shapes: every d class, clustered and lattice data (many pairs exactly
    at eps), minPts from 1 to past n."""
    rng = np.random.default_rng(2024)
    cases = []
    for d in (1, 2, 3, 4, 5, 8, 12, 16):
        n = int(rng.integers(400, 2000))
        k = int(rng.integers(2, 12))
        c = rng.uniform(0, 10, (k, d))
        x = c[rng.integers(0, k, n)] + rng.normal(0, rng.uniform(0.1, 0.6), (n, d))
        eps = float(rng.uniform(0.2, 0.9) * np.sqrt(d))
        cases.append((x.astype(np.float32), eps, int(rng.integers(1, 3 * d + 3))))
    for d in (2, 3):
        g = np.stack(np.meshgrid(*[np.arange(12)] * d, indexing="ij"), -1).reshape(-1, d)
        cases.append(((g * np.float32(0.25)).astype(np.float32), 0.25, int(2 * d)))
    cases.append((rng.normal(0, 1, (300, 3)).astype(np.float32), 0.3, 400))
    for x, eps, m in cases:
        nn_r, ci_r, _, _ = oracle.run_ref(x, eps, m, threads=2)
        nn, ci, _ = oracle.grid(x, eps, m)
        np.testing.assert_array_equal(nn, nn_r, err_msg=f"d={x.shape[1]} eps={eps} m={m}")
        np.testing.assert_array_equal(ci, ci_r, err_msg=f"d={x.shape[1]} eps={eps} m={m}")


def test_grid_matches_literal_property():
    """Property test of the checker itself: on arbitrary small inputs (duplicates,
    lattice points exactly eps apart, NaN, inf, FLT_MAX, subnormals, eps of 0 or
    negative, minPts 0 to past n) the grid restatement, which checks the GPU at large
    n, gives the literal restatement's outputs."""
    hyp = pytest.importorskip("hypothesis")
    st = pytest.importorskip("hypothesis.strategies")
    fmax = float(np.finfo(np.float32).max)
    values = st.sampled_from([0.0, 0.25, 0.5, 0.75, 1.0, -0.5, 3.0, 1e-40, float("nan"), float("inf"),
                              -float("inf"), fmax, 0.1, 0.2, 0.3])

    @hyp.settings(max_examples=300, deadline=None, derandomize=True)
    @hyp.given(d=st.integers(1, 16), n=st.integers(1, 40), data=st.data(),
               eps=st.sampled_from([0.0, 0.25, 0.5, -0.5, 0.3, 1.0, 2.5]), m=st.integers(0, 8))
    def check(d, n, data, eps, m):
        flat = data.draw(st.lists(values, min_size=n * d, max_size=n * d))
        x = np.array(flat, dtype=np.float32).reshape(n, d)
        a_nn, a_ci, _, a_meta = oracle.reference(x, eps, m)
        b_nn, b_ci, b_meta = oracle.grid(x, eps, m)
        np.testing.assert_array_equal(a_nn, b_nn)
        np.testing.assert_array_equal(a_ci, b_ci)
        assert [a_meta[k] for k in ("clusters", "noise", "cores", "n")] == \
            [b_meta[k] for k in ("clusters", "noise", "cores", "n")]

    check()


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built here")
def test_literal_matches_reference_harness_property():
    """The same adversarial inputs through the reference's own build: the literal
    restatement reproduces its counts, ids and meta (single-threaded reference runs,
    so its label sweep order is fixed)."""
    hyp = pytest.importorskip("hypothesis")
    st = pytest.importorskip("hypothesis.strategies")
    fmax = float(np.finfo(np.float32).max)
    values = st.sampled_from([0.0, 0.25, 0.5, 0.75, 1.0, -0.5, 3.0, 1e-40, float("nan"), float("inf"),
                              -float("inf"), fmax, 0.1, 0.2, 0.3])

    @hyp.settings(max_examples=60, deadline=None, derandomize=True)
    @hyp.given(d=st.integers(1, 16), n=st.integers(1, 40), data=st.data(),
               eps=st.sampled_from([0.0, 0.25, 0.5, -0.5, 0.3, 1.0, 2.5]), m=st.integers(0, 8))
    def check(d, n, data, eps, m):
        flat = data.draw(st.lists(values, min_size=n * d, max_size=n * d))
        x = np.array(flat, dtype=np.float32).reshape(n, d)
        r_nn, r_ci, _, _ = oracle.run_ref(x, eps, m, threads=1)
        a_nn, a_ci, _, _ = oracle.reference(x, eps, m)
        np.testing.assert_array_equal(a_nn, r_nn)
        np.testing.assert_array_equal(a_ci, r_ci)

    check()


# ---------------------------------------------------------------------------
# The cell restatement (oracle.cells), which checks the GPU at 10^7..10^8 points,
# is pinned the same way: the reference's fixtures and full C1 hashes, the literal
# restatement on adversarial inputs, and the grid restatement on seeded shapes.
# ---------------------------------------------------------------------------
def _assert_early(nn_e, nn_exact, m):
    """Early-exit counts: exact below min_pts, at least min_pts for every core."""
    below = nn_exact < m
    np.testing.assert_array_equal(nn_e[below], nn_exact[below])
    assert (nn_e[~below] >= m).all()


@pytest.mark.parametrize("name", NAMES)
def test_cell_restatement_matches_reference(name):
    g = load_golden(name)
    e = np.float32(g["eps"])
    if not np.isfinite(np.float32(e * e)):
        pytest.skip("cell restatement needs a finite eps*eps")
    m = int(g["min_pts"])
    for early in (False, True):
        nn, ci, meta = oracle.cells(g["coords"], float(e), m, early=early)
        if early:
            _assert_early(nn, g["nn"], m)
        else:
            np.testing.assert_array_equal(nn, g["nn"])
        np.testing.assert_array_equal(ci, g["cluster_index"])
        assert [meta["clusters"], meta["noise"], meta["cores"], meta["n"]] == list(g["meta"])


def test_cell_restatement_matches_reference_full_c1(pkg):
    with open(os.path.join(GOLDEN, "c1_full.json")) as f:
        doc = json.load(f)
    w = pkg.synthetic.config1()
    nn, ci, meta = oracle.cells(w.coords, w.eps, w.min_pts)
    assert meta["clique_cells"]
    assert hashlib.sha256(nn.astype("<i4").tobytes()).hexdigest() == doc["nn_sha256"]
    assert hashlib.sha256(ci.astype("<i4").tobytes()).hexdigest() == doc["cluster_index_sha256"]
    assert (meta["clusters"], meta["noise"], meta["cores"]) == (doc["clusters"], doc["noise"], doc["cores"])


def test_cell_matches_literal_property():
    """Adversarial small inputs (as for the grid restatement above), both count modes."""
    hyp = pytest.importorskip("hypothesis")
    st = pytest.importorskip("hypothesis.strategies")
    fmax = float(np.finfo(np.float32).max)
    values = st.sampled_from([0.0, 0.25, 0.5, 0.75, 1.0, -0.5, 3.0, 1e-40, float("nan"), float("inf"),
                              -float("inf"), fmax, 0.1, 0.2, 0.3, 0.35, 0.7, 1.05])

    @hyp.settings(max_examples=400, deadline=None, derandomize=True)
    @hyp.given(d=st.integers(1, 16), n=st.integers(1, 48), data=st.data(),
               eps=st.sampled_from([0.0, 0.25, 0.5, -0.5, 0.3, 1.0, 2.5, 0.7]), m=st.integers(0, 8))
    def check(d, n, data, eps, m):
        flat = data.draw(st.lists(values, min_size=n * d, max_size=n * d))
        x = np.array(flat, dtype=np.float32).reshape(n, d)
        a_nn, a_ci, _, a_meta = oracle.reference(x, eps, m)
        for early in (False, True):
            b_nn, b_ci, b_meta = oracle.cells(x, eps, m, early=early)
            if early:
                _assert_early(b_nn, a_nn, m)
            else:
                np.testing.assert_array_equal(a_nn, b_nn)
            np.testing.assert_array_equal(a_ci, b_ci)
            assert [a_meta[k] for k in ("clusters", "noise", "cores", "n")] == \
                [b_meta[k] for k in ("clusters", "noise", "cores", "n")]

    check()


@pytest.mark.parametrize("cfg,n", [(1, 60_000), (2, 300_000), (3, 80_000), (5, 400_000)])
def test_cell_matches_grid_on_benchmark_shapes(pkg, cfg, n):
    """The benchmark generators at reduced n: clique cells (2-D, 3-D), the
    three-dimension eps grid (8-D), dense Zipf clusters and filaments (skewed 2-D)."""
    w = pkg.synthetic.make(cfg, n=n)
    g_nn, g_ci, g_meta = oracle.grid(w.coords, w.eps, w.min_pts)
    nn, ci, meta = oracle.cells(w.coords, w.eps, w.min_pts)
    np.testing.assert_array_equal(nn, g_nn)
    np.testing.assert_array_equal(ci, g_ci)
    nn_e, ci_e, _ = oracle.cells(w.coords, w.eps, w.min_pts, early=True)
    _assert_early(nn_e, g_nn, w.min_pts)
    np.testing.assert_array_equal(ci_e, g_ci)
    assert (meta["clusters"], meta["noise"], meta["cores"]) == (g_meta["clusters"], g_meta["noise"], g_meta["cores"])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference harness not built here")
def test_cell_restatement_matches_reference_harness_random():
    """The cell restatement against the reference's own build on seeded random
    shapes of every d class and on lattices with pairs exactly at eps."""
    rng = np.random.default_rng(7)
    cases = []
    for d in (1, 2, 3, 4, 8, 16):
        n = int(rng.integers(400, 1500))
        k = int(rng.integers(2, 10))
        c = rng.uniform(0, 10, (k, d))
        x = c[rng.integers(0, k, n)] + rng.normal(0, rng.uniform(0.1, 0.6), (n, d))
        eps = float(rng.uniform(0.2, 0.9) * np.sqrt(d))
        cases.append((x.astype(np.float32), eps, int(rng.integers(1, 3 * d + 3))))
    for d in (2, 3):
        g = np.stack(np.meshgrid(*[np.arange(10)] * d, indexing="ij"), -1).reshape(-1, d)
        cases.append(((g * np.float32(0.25)).astype(np.float32), 0.25, int(2 * d)))
        cases.append(((g * np.float32(0.25)).astype(np.float32), float(np.float32(0.25) * np.sqrt(np.float32(d))), 3))
    for x, eps, m in cases:
        nn_r, ci_r, _, _ = oracle.run_ref(x, eps, m, threads=2)
        nn, ci, _ = oracle.cells(x, eps, m)
        np.testing.assert_array_equal(nn, nn_r, err_msg=f"d={x.shape[1]} eps={eps} m={m}")
        np.testing.assert_array_equal(ci, ci_r, err_msg=f"d={x.shape[1]} eps={eps} m={m}")
