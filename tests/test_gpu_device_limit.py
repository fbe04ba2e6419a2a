"""The device-side bound of the union-find loops (ndb_b200_set_debug_limits).

Every find and union loop on the GPU carries an iteration bound and reports
NDB_ERR_DEVICE_LIMIT instead of spinning (the reference's propagation loop,
data_process.cpp:183, has none).  Here the bound is lowered on purpose on a long
filament, whose hooking builds parent chains far deeper than a step, so that it
runs out; the same context, set back to the default, then returns the oracle's
ids.  Nothing waits on anything that never comes: the shortened loops simply end."""
import numpy as np
import pytest

from conftest import load_pkg


def filament(n, d, step, seed=0):
    """n points along a straight line, step apart, with a little jitter off it."""
    rng = np.random.default_rng(seed)
    x = np.zeros((n, d), np.float64)
    x[:, 0] = np.arange(n) * step
    x[:, 1:] += rng.uniform(-0.01, 0.01, (n, d - 1))
    return np.ascontiguousarray(x[rng.permutation(n)].astype(np.float32))


def test_debug_limits_argument_checks(pkg):
    lib = pkg.lib.load()
    assert lib.ndb_b200_set_debug_limits(None, 4) == 1  # NDB_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("d", [2, 5])  # cell units (same-cell-linked grid) and point units
def test_union_find_bound_runs_out_then_recovers(d):
    import oracle

    pkg = load_pkg()
    x = filament(60_000, d, 0.3)
    eps, m = 1.0, 3
    nn_o, ci_o, meta = oracle.grid(x, eps, m)
    assert meta["clusters"] == 1
    with pkg.Context(0) as ctx:
        with pytest.raises(ValueError):
            ctx.set_debug_limits(-1)
        ctx.set_debug_limits(1)
        with pytest.raises(pkg.lib.NdbError) as ei:
            ctx.run(x, eps, m, full_count=True)
        assert ei.value.status == 8  # NDB_ERR_DEVICE_LIMIT
        ctx.set_debug_limits(0)  # back to the default bound
        nn, ci, res = ctx.run(x, eps, m, full_count=True)
        np.testing.assert_array_equal(nn, nn_o)
        np.testing.assert_array_equal(ci, ci_o)
        assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])
        # the batched entry point honours the bound too
        ctx.set_debug_limits(1)
        with pytest.raises(pkg.lib.NdbError) as ei:
            ctx.run_batched([(x, eps, m)], full_count=True)
        assert ei.value.status == 8
        ctx.set_debug_limits(0)
        (_, ci_b, _), = ctx.run_batched([(x, eps, m)], full_count=True)
        np.testing.assert_array_equal(ci_b, ci_o)
