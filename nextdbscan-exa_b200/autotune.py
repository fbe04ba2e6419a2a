"""Autotuner for the neighbour-count thresholds of a context (ndb_tuning).

For d >= 8 the library counts neighbours with the exact FP32 sum, the FP32 Gram
filter on CUDA cores, the tensor-core Gram filter, or a mix, with each item (up to 32
points of one cell) sent to the tensor cores by its size.  Which is faster depends on the data: how full the items are,
d, and whether counts stop early at minPts.  The tuner runs the job under each
candidate setting and times the count kernels with the library's own device
events (ndb_stats.ms_count_kernel, min over repetitions).  It requires every
candidate to give the same core flags and cluster ids (and the same counts with
full counts), then leaves the fastest setting on the context and returns the
table.  It computes nothing itself: every run is a call of the CUDA library.

The reference has one count form (data_process.cpp:395-458), so it has nothing
to tune; the thresholds only pick between kernels that give identical results.
"""
from __future__ import annotations

import numpy as np

# tc_min_dim above NDB_MAX_DIM keeps every count on the CUDA cores
EXACT_ONLY = {"tc_min_dim": 17, "tc_min_item": 0, "gram_filter": 0}
GRAM_ONLY = {"tc_min_dim": 17, "tc_min_item": 0, "gram_filter": 1}
ITEM_SIZES = (1, 8, 12, 16, 20, 24, 28, 32)


def candidates(d: int) -> list[dict]:
    """Settings worth timing at dimensionality d (none below the filters' d = 8): the
    exact sum, the FP32 Gram filter, and the tensor-core filter for items of at least
    k points (the rest on the exact sum)."""
    if d < 8:
        return []
    return [dict(EXACT_ONLY), dict(GRAM_ONLY)] + [{"tc_min_dim": d, "tc_min_item": k, "gram_filter": 0}
                                                  for k in ITEM_SIZES]


def tune_count(ctx, coords, eps: float, min_pts: int, *, full_count: bool = False, reps: int = 3) -> dict:
    """Times every candidate on this job and applies the fastest to ctx.

    Returns {"best": setting, "table": [{setting, ms_count_kernel, tensor_items}, ...]}.
    Raises AssertionError if two candidates disagree (they never should: the
    thresholds choose between exact kernels)."""
    x = np.ascontiguousarray(coords, dtype=np.float32)
    d = x.shape[1]
    table = []
    ref = None
    for cand in candidates(d):
        ctx.set_tuning(**cand)
        nn, ci, res = ctx.run(x, eps, min_pts, full_count=full_count)  # warm-up, and the results checked
        core = nn >= min_pts
        if ref is None:
            ref = (nn, core, ci, res)
        else:
            assert np.array_equal(ci, ref[2]) and np.array_equal(core, ref[1]) and res == ref[3], cand
            if full_count:
                assert np.array_equal(nn, ref[0]), cand
        times = []
        for _ in range(max(1, reps)):
            ctx.run(x, eps, min_pts, full_count=full_count)
            times.append(ctx.stats()["ms_count_kernel"])
        st = ctx.stats()
        table.append({**cand, "ms_count_kernel": min(times), "tensor_items": int(st["tensor_items"])})
    if not table:
        ctx.reset_tuning()
        return {"best": None, "table": []}
    best = min(table, key=lambda r: r["ms_count_kernel"])
    setting = {"tc_min_dim": best["tc_min_dim"], "tc_min_item": best["tc_min_item"],
               "gram_filter": best["gram_filter"]}
    ctx.set_tuning(**setting)
    return {"best": setting, "table": table}
