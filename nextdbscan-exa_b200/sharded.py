"""DBSCAN over several ranks: spatial slabs with a halo, one local run per rank, a
merge of the components that cross slab boundaries, and a border pass with the
merged ids.

The reference scales n over MPI ranks by broadcasting every chunk of points (and
of cores) to every rank and merging labels with allreduce-min
(data_process.cpp:129, 175, 232-233, 325, 387; magma_mpi.h:58-123).  Here a rank
instead receives only the points of its slab along the widest axis plus the points
within 2r of it (r bounds the per-dimension difference of any pair the FP32
predicate accepts), and runs the single-GPU library on them:

  * a point's neighbours lie within r of it, so every point of the slab and of the
    inner ring (within r of the slab) has its exact count and core flag locally;
    the outer ring (r to 2r) can only be under-counted, so a local core is always a
    true core;
  * every core-core edge with an endpoint in the slab joins two points of the slab
    or the inner ring: it is found by the slab's rank, so the union of the ranks'
    local components is the true core partition;
  * components meet across ranks only through points that several ranks hold (halo
    copies and the points near a boundary): each rank contributes (point, smallest
    index of its local component) for those, every rank merges the pairs the same
    way, and a component's id is the rank among all cores (index order) of its
    smallest core, as in the reference (data_process.cpp:141-171, :204-260);
  * a border point's cores in range are all in its slab or inner ring, so the border
    pass with the merged ids (ndb_b200_assign_border) gives the reference's minimum
    (data_process.cpp:204-209).

Ranks start from contiguous blocks of the input in index order, as the reference's
reader hands them out (magma_input.h:113-125), and get their block's outputs back.
The exchanges use torch.distributed object collectives; every rank takes the same
collective steps in the same order.  The local step is pluggable: the library on the
rank's GPU by default (gpu_local_step), the CPU oracle in tests.
"""
from __future__ import annotations

import math
from typing import Callable, NamedTuple

import numpy as np

NO_CLUSTER = 2**31 - 1
FLT_MAX = float(np.finfo(np.float32).max)
SAMPLES_PER_RANK = 4096


class LocalResult(NamedTuple):
    nn: np.ndarray                      # int32 per local point
    cluster_index: np.ndarray           # int32: equal ids for the cores of one local component
    border: Callable[[np.ndarray], np.ndarray]  # core ids (input order) -> every point's cluster index


class ShardedResult(NamedTuple):
    nn: np.ndarray
    cluster_index: np.ndarray
    clusters: int
    noise: int
    core_count: int
    n: int


def reach(eps: float) -> float:
    """r: |a_k - b_k| <= r in every dimension for every pair the FP32 predicate
    accepts (the rounded square of the rounded difference is <= e2)."""
    e2 = float(np.float32(eps) * np.float32(eps))
    return max(math.sqrt(e2), 2.0 ** -63) * (1.0 + 2.0 ** -20)


def valid_mask(x: np.ndarray) -> np.ndarray:
    """Points that take part in a grid: finite, first coordinate not FLT_MAX (the
    reference's padding marker, data_process.cpp:440); the others are in range of
    nothing."""
    if x.shape[0] == 0:
        return np.zeros(0, bool)
    return np.isfinite(x).all(axis=1) & (x[:, 0] != np.float32(FLT_MAX))


def gpu_local_step(ctx) -> Callable:
    """The library on this rank's GPU: one ndb_b200_run, then its border pass with
    the merged ids."""

    def step(x: np.ndarray, eps: float, min_pts: int, full_count: bool) -> LocalResult:
        nn, ci, _ = ctx.run(x, eps, min_pts, full_count=full_count)
        return LocalResult(nn, ci, ctx.assign_border)

    return step


class _Comm:
    def __init__(self, group):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def gather(self, obj) -> list:
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out

    def exchange(self, parts: list) -> list:
        """parts[s] goes to rank s; returns what every rank sent here."""
        allp = self.gather(parts)
        return [allp[src][self.rank] for src in range(self.world)]


def _merge_roots(pairs: np.ndarray) -> dict:
    """Union of (a, b) pairs of global indices; returns {index: smallest index of
    its merged set} for every index that occurs."""
    if pairs.size == 0:
        return {}
    keys, inv = np.unique(pairs.reshape(-1), return_inverse=True)
    a, b = inv[0::2], inv[1::2]
    lab = np.arange(keys.size)
    while True:  # min-label propagation over the pairs with pointer jumping
        old = lab.copy()
        m = np.minimum(lab[a], lab[b])
        np.minimum.at(lab, a, m)
        np.minimum.at(lab, b, m)
        lab = lab[lab]
        if np.array_equal(lab, old):
            break
    return dict(zip(keys.tolist(), keys[lab].tolist()))


def run_sharded(coords, eps: float, min_pts: int, *, local: Callable, gid_offset: int | None = None,
                group=None, full_count: bool = False) -> ShardedResult:
    """DBSCAN of the union of every rank's block of points.

    coords: this rank's block (n_r x d float32), block r of the input in index order.
    local: the local step (gpu_local_step(ctx), or a CPU stand-in in tests).
    Returns this block's nn and cluster_index (the reference's encoding, identical to
    one run over the whole input) and the global meta."""
    comm = _Comm(group)
    W, me = comm.world, comm.rank
    x = np.ascontiguousarray(np.asarray(coords, dtype=np.float32))
    n_r, d = x.shape
    sizes = comm.gather(int(n_r))
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    if gid_offset is None:
        gid_offset = int(offsets[me])
    n_total = int(offsets[-1])
    gids = gid_offset + np.arange(n_r, dtype=np.int64)
    ok = valid_mask(x)

    # slabs along the widest axis, split at sampled quantiles
    lo = x[ok].min(axis=0).astype(np.float64) if ok.any() else np.full(d, np.inf)
    hi = x[ok].max(axis=0).astype(np.float64) if ok.any() else np.full(d, -np.inf)
    boxes = comm.gather((lo, hi))
    glo = np.min([b[0] for b in boxes], axis=0)
    ghi = np.max([b[1] for b in boxes], axis=0)
    span = np.where(np.isfinite(ghi - glo), ghi - glo, -1.0)
    axis = int(np.argmax(span))
    xa = x[:, axis].astype(np.float64)
    mine = np.sort(xa[ok])
    take = np.unique(np.linspace(0, mine.size - 1, min(mine.size, SAMPLES_PER_RANK)).astype(np.int64)) \
        if mine.size else np.zeros(0, np.int64)
    samples = np.sort(np.concatenate([s for s in comm.gather(mine[take]) if s.size] or [np.zeros(0)]))
    if samples.size:
        bounds = samples[np.minimum((np.arange(1, W) * samples.size) // W, samples.size - 1)]
    else:
        bounds = np.zeros(W - 1)
    slab_lo = np.concatenate([[-np.inf], bounds])
    slab_hi = np.concatenate([bounds, [np.inf]])
    h = 2.0 * reach(eps) * (1.0 + 2.0 ** -10)  # halo width, with room for the double arithmetic

    owner = np.full(n_r, me, np.int64)  # points outside the grid stay where they are
    owner[ok] = np.searchsorted(bounds, xa[ok], side="right")
    parts = []
    for s in range(W):
        near = ok & (xa >= slab_lo[s] - h) & (xa < slab_hi[s] + h)
        sel = (owner == s) | near
        parts.append((x[sel], gids[sel], owner[sel] == s))
    got = comm.exchange(parts)
    lx = np.concatenate([g[0] for g in got]) if got else np.zeros((0, d), np.float32)
    lg = np.concatenate([g[1] for g in got]).astype(np.int64)
    lown = np.concatenate([g[2] for g in got]).astype(bool)
    order = np.argsort(lg, kind="stable")  # the local problem in global index order
    lx, lg, lown = np.ascontiguousarray(lx[order]), lg[order], lown[order]

    L = local(lx, eps, min_pts, full_count)
    core = L.nn >= min_pts
    # local components: cores with one local id; their smallest global index
    comp_min = {}
    for cid, g in zip(L.cluster_index[core].tolist(), lg[core].tolist()):
        if g < comp_min.get(cid, n_total):
            comp_min[cid] = g
    lxa = lx[:, axis].astype(np.float64)
    lok = valid_mask(lx)
    own_slab = me
    near_edge = lok & ((lxa < slab_lo[own_slab] + h) | (lxa >= slab_hi[own_slab] - h))
    shared = core & (~lown | near_edge)
    pairs = np.array([[g, comp_min[c]] for g, c in zip(lg[shared].tolist(), L.cluster_index[shared].tolist())],
                     np.int64).reshape(-1, 2)
    all_pairs = np.concatenate([p for p in comm.gather(pairs) if p.size] or [np.zeros((0, 2), np.int64)])
    root = _merge_roots(all_pairs)
    final = {c: root.get(m, m) for c, m in comp_min.items()}  # component -> smallest core index overall
    F = np.full(lg.size, -1, np.int64)
    F[core] = [final[c] for c in L.cluster_index[core].tolist()]

    # id = rank of that smallest core among all cores in index order
    own_core_gids = np.sort(lg[core & lown])
    queries = np.unique(np.concatenate([q for q in comm.gather(np.unique(F[core])) if q.size] or
                                       [np.zeros(0, np.int64)]))
    below = np.searchsorted(own_core_gids, queries, side="left").astype(np.int64)
    ranks = np.sum(comm.gather(below), axis=0) if queries.size else np.zeros(0, np.int64)
    rank_of = dict(zip(queries.tolist(), np.asarray(ranks).tolist()))
    ids = np.full(lg.size, NO_CLUSTER, np.int32)
    ids[core] = [rank_of[f] for f in F[core].tolist()]
    ci = np.asarray(L.border(ids), dtype=np.int32)

    # this rank's slab points back to the ranks whose blocks hold them
    back = np.searchsorted(offsets, lg, side="right") - 1
    ret = comm.exchange([(lg[lown & (back == s)], L.nn[lown & (back == s)], ci[lown & (back == s)])
                         for s in range(W)])
    nn_out = np.zeros(n_r, np.int32)
    ci_out = np.full(n_r, NO_CLUSTER, np.int32)
    for g, v, c in ret:
        nn_out[g - gid_offset] = v
        ci_out[g - gid_offset] = c
    meta = np.sum(comm.gather(np.array([int((core & lown).sum()), int((ci[lown] == NO_CLUSTER).sum()),
                                        int(((F == lg) & core & lown).sum())], np.int64)), axis=0)
    return ShardedResult(nn_out, ci_out, clusters=int(meta[2]), noise=int(meta[1]), core_count=int(meta[0]),
                         n=n_total)
