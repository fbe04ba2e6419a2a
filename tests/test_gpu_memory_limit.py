"""Allocation failure injected on the host: a context given a device-memory cap
refuses the run that would pass it with NDB_ERR_OUT_OF_MEMORY before it allocates,
stays usable, and gives the reference's results once the cap admits the job.  The
refusal is host code; no GPU fault is involved."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _job(name):
    g = load_golden(name)
    return g, (g["coords"], float(g["eps"]), int(g["min_pts"]))


def test_capped_context_refuses_then_recovers(pkg):
    g, (x, e, m) = _job("blobs_d3")
    with pkg.Context(0) as c:
        c.set_memory_limit(64 * 1024)  # below what any job of this size needs
        with pytest.raises(pkg.lib.NdbError, match="OUT_OF_MEMORY"):
            c.run(x, e, m, full_count=True)
        assert c.device_bytes() <= 64 * 1024
        c.set_memory_limit(0)
        nn, ci, res = c.run(x, e, m, full_count=True)
        np.testing.assert_array_equal(nn, g["nn"])
        np.testing.assert_array_equal(ci, g["cluster_index"])
        held = c.device_bytes()
        assert held > 0
        # the buffers are kept, so a cap at the current footprint admits the same job
        c.set_memory_limit(held)
        nn, ci, _ = c.run(x, e, m, full_count=True)
        np.testing.assert_array_equal(ci, g["cluster_index"])
        assert c.device_bytes() == held


def test_lower_cap_releases_buffers_and_pending_state(pkg):
    g, (x, e, m) = _job("c1_n4000")
    with pkg.Context(0) as c:
        c.classify(x, e, m, full_count=True)
        held = c.device_bytes()
        c.set_memory_limit(held // 2)
        assert c.device_bytes() == 0
        with pytest.raises(pkg.lib.NdbError, match="NO_STATE"):
            c.assign_labels()
        c.set_memory_limit(0)
        nn, ci, res = c.run(x, e, m, full_count=True)
        np.testing.assert_array_equal(ci, g["cluster_index"])
        assert [res.clusters, res.noise, res.core_count, res.n] == list(g["meta"])


def test_capped_batch_fails_every_job_then_recovers(pkg):
    ga, a = _job("c1_n4000")
    gb, b = _job("blobs_d8")
    with pkg.Context(0) as c:
        c.set_memory_limit(64 * 1024)
        with pytest.raises(pkg.lib.NdbError, match="OUT_OF_MEMORY"):
            c.run_batched([a, b], full_count=True)
        st = {pkg.lib.STATUS[c.last_jobs[k].status] for k in range(2)}
        assert st == {"NDB_ERR_OUT_OF_MEMORY"}
        c.set_memory_limit(0)
        outs = c.run_batched([a, b], full_count=True)
        for g, (nn, ci, _) in zip((ga, gb), outs):
            np.testing.assert_array_equal(nn, g["nn"])
            np.testing.assert_array_equal(ci, g["cluster_index"])
