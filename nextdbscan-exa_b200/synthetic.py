"""Seeded synthetic workloads with the shapes, sizes and distributions of the
five benchmark configurations (no public dataset is involved).

Every generator draws from numpy's PCG64 with a fixed seed (the configuration's
index unless given), works in float64 and casts to float32, the only coordinate
type of nextdbscan-exa (magma_input.h:105-138, data_process.h:55).  Points are
shuffled so that input order carries no cluster structure.  Passing a smaller n
draws from the same generator with every count scaled by n / n_full (the same
clusters, sparser), which is how bounded CPU-baseline samples are made.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    coords: np.ndarray  # float32, n x d, C-contiguous
    eps: float
    min_pts: int

    @property
    def n(self) -> int:
        return int(self.coords.shape[0])

    @property
    def d(self) -> int:
        return int(self.coords.shape[1])


def _split(total: int, parts: int) -> np.ndarray:
    base = np.full(parts, total // parts, dtype=np.int64)
    base[: total % parts] += 1
    return base


def _finish(rng: np.random.Generator, blocks: list[np.ndarray]) -> np.ndarray:
    pts = np.concatenate(blocks, axis=0)
    pts = pts[rng.permutation(pts.shape[0])]
    return np.ascontiguousarray(pts.astype(np.float32))


def gaussian_mixture(rng: np.random.Generator, n_clustered: int, centers: np.ndarray,
                     sigmas: np.ndarray) -> np.ndarray:
    """n_clustered points split equally over the Gaussians; sigmas is (k,) or (k, d)."""
    k, d = centers.shape
    counts = _split(n_clustered, k)
    lab = np.repeat(np.arange(k), counts)
    sig = sigmas[lab][:, None] if sigmas.ndim == 1 else sigmas[lab]
    return centers[lab] + rng.standard_normal((n_clustered, d)) * sig


def config1(n: int = 100_000, seed: int = 1) -> Workload:
    """n=100,000 2-D: 95% from 20 isotropic Gaussians (centres U[0,100]^2, sigma
    U[0.5,2]), 5% uniform noise over the box; eps=0.8, minPts=5; FP64 -> FP32."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_noise = int(round(n * 0.05))
    centers = rng.uniform(0.0, 100.0, (20, 2))
    sig = rng.uniform(0.5, 2.0, 20)
    pts = gaussian_mixture(rng, n - n_noise, centers, sig)
    noise = rng.uniform(0.0, 100.0, (n_noise, 2))
    return Workload("plain-2d-100k", _finish(rng, [pts, noise]), 0.8, 5)


def config2(n: int = 10_000_000, seed: int = 2) -> Workload:
    """n=10M 3-D: 98% from 500 anisotropic Gaussians (centres U[0,1000]^3,
    per-axis sigma log-uniform [0.5,5]), 2% uniform noise; eps=1.5, minPts=10."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_noise = int(round(n * 0.02))
    centers = rng.uniform(0.0, 1000.0, (500, 3))
    sig = np.exp(rng.uniform(np.log(0.5), np.log(5.0), (500, 3)))
    pts = gaussian_mixture(rng, n - n_noise, centers, sig)
    noise = rng.uniform(0.0, 1000.0, (n_noise, 3))
    return Workload("plain-3d-10m", _finish(rng, [pts, noise]), 1.5, 10)


def config3(n: int = 2_000_000, seed: int = 3) -> Workload:
    """n=2M 8-D: 200 Gaussians (centres U[0,50]^8, sigma U[0.3,1.0]), 5% uniform
    noise; eps=1.2, minPts=8."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_noise = int(round(n * 0.05))
    centers = rng.uniform(0.0, 50.0, (200, 8))
    sig = rng.uniform(0.3, 1.0, 200)
    pts = gaussian_mixture(rng, n - n_noise, centers, sig)
    noise = rng.uniform(0.0, 50.0, (n_noise, 8))
    return Workload("tensor-filter-8d-2m", _finish(rng, [pts, noise]), 1.2, 8)


def config5(n: int = 100_000_000, seed: int = 5, n_gauss: int = 10_000, n_filaments: int = 10,
            filament_frac: float = 0.05) -> Workload:
    """n=100M 2-D skewed: cluster sizes Zipf(s=1.2) over 10,000 Gaussians (sigma
    U[0.1,3]) + 10 polyline filaments (jitter 0.2) + 1% noise in [0,10000]^2;
    eps=0.5, minPts=4.  The filaments take filament_frac of the points."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n_noise = int(round(n * 0.01))
    n_fil = int(round(n * filament_frac))
    n_gau = n - n_noise - n_fil
    w = np.arange(1, n_gauss + 1, dtype=np.float64) ** -1.2
    w /= w.sum()
    counts = rng.multinomial(n_gau, w)
    centers = rng.uniform(0.0, 10_000.0, (n_gauss, 2))
    sig = rng.uniform(0.1, 3.0, n_gauss)
    blocks = []
    lab = np.repeat(np.arange(n_gauss), counts)
    g = centers[lab] + rng.standard_normal((n_gau, 2)) * sig[lab][:, None]
    blocks.append(g)
    del lab
    per = _split(n_fil, n_filaments)
    for f in range(n_filaments):
        verts = rng.uniform(0.0, 10_000.0, (int(rng.integers(3, 9)), 2))
        seg_len = np.linalg.norm(np.diff(verts, axis=0), axis=1)
        cum = np.concatenate([[0.0], np.cumsum(seg_len)])
        t = rng.uniform(0.0, cum[-1], int(per[f]))
        seg = np.clip(np.searchsorted(cum, t, side="right") - 1, 0, len(seg_len) - 1)
        frac = (t - cum[seg]) / seg_len[seg]
        p = verts[seg] + (verts[seg + 1] - verts[seg]) * frac[:, None]
        blocks.append(p + rng.standard_normal(p.shape) * 0.2)
    blocks.append(rng.uniform(0.0, 10_000.0, (n_noise, 2)))
    return Workload("skew-2d-100m", _finish(rng, blocks), 0.5, 4)


@dataclasses.dataclass(frozen=True)
class BatchJob:
    coords: np.ndarray  # float32, n x d
    eps: float
    min_pts: int

    @property
    def n(self) -> int:
        return int(self.coords.shape[0])

    @property
    def d(self) -> int:
        return int(self.coords.shape[1])


def _eps_4nn(rng: np.random.Generator, pts: np.ndarray) -> float:
    """90th percentile, over a 1% sample (at least 10 points), of the distance from
    each sampled point to its 4th nearest neighbour in the whole job."""
    from scipy.spatial import cKDTree

    n = pts.shape[0]
    m = min(n, max(10, n // 100))
    idx = rng.choice(n, m, replace=False)
    dist, _ = cKDTree(pts).query(pts[idx], k=5)  # k=5: the point itself is the first hit
    return float(np.percentile(dist[:, 4], 90))


def _job_shape(rng: np.random.Generator, n_min: int, n_max: int, dims) -> tuple[int, int]:
    """The first two draws of a batch job: its n (log-uniform) and its d."""
    n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
    d = int(dims[rng.integers(0, len(dims))])
    return n, d


def _one_job(args) -> BatchJob:
    seq, n_min, n_max, dims = args
    rng = np.random.Generator(np.random.PCG64(seq))
    n, d = _job_shape(rng, n_min, n_max, dims)
    k = int(rng.integers(5, 51))
    n_noise = int(round(n * 0.05))
    centers = rng.uniform(0.0, 100.0, (k, d))
    sig = rng.uniform(0.5, 2.0, k)
    pts = gaussian_mixture(rng, n - n_noise, centers, sig)
    noise = rng.uniform(0.0, 100.0, (n_noise, d))
    x = _finish(rng, [pts, noise])
    return BatchJob(x, _eps_4nn(rng, x.astype(np.float64)), 2 * d)


def config4(n_jobs: int = 4096, seed: int = 4, n_min: int = 1_000, n_max: int = 200_000,
            dims: tuple = (2, 3, 8, 16), workers: int | None = None) -> list[BatchJob]:
    """4,096 independent jobs: n log-uniform in [1,000, 200,000], d uniform in
    {2,3,8,16}, each a mixture of 5-50 isotropic Gaussians (centres U[0,100]^d,
    sigma U[0.5,2]) + 5% uniform noise; eps = 90th percentile of the 4-NN distance
    over a 1% sample; minPts = 2d.  Job j draws from the j-th child of
    SeedSequence(seed), so any prefix of the batch is reproducible alone."""
    seqs = np.random.SeedSequence(seed).spawn(n_jobs)
    args = [(s, n_min, n_max, tuple(dims)) for s in seqs]
    if workers is None:
        import os
        workers = min(len(os.sched_getaffinity(0)), 32) if n_jobs >= 64 else 1
    if workers <= 1:
        return [_one_job(a) for a in args]
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(workers) as pool:  # spawn: callers may already hold a CUDA context
        return pool.map(_one_job, args, chunksize=max(1, n_jobs // (8 * workers)))


def config4_shapes(n_jobs: int = 4096, seed: int = 4, n_min: int = 1_000, n_max: int = 200_000,
                   dims: tuple = (2, 3, 8, 16)) -> list[tuple[int, int]]:
    """(n, d) of every job of config4 with the same arguments, without drawing the
    points (for sizing and extrapolation)."""
    return [_job_shape(np.random.Generator(np.random.PCG64(s)), n_min, n_max, tuple(dims))
            for s in np.random.SeedSequence(seed).spawn(n_jobs)]


CONFIGS = {1: config1, 2: config2, 3: config3, 5: config5}


def make(config: int, n: int | None = None, seed: int | None = None) -> Workload:
    fn = CONFIGS[config]
    kw = {}
    if n is not None:
        kw["n"] = n
    if seed is not None:
        kw["seed"] = seed
    return fn(**kw)
