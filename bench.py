#!/usr/bin/env python
"""Benchmark: clustered points/s of the B200 DBSCAN hot path, chosen form against
the plain GPU form.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config C]

Default (configuration 4): one step = the 4,096-job batch (n log-uniform in
[1k, 200k], d in {2, 3, 8, 16}, 151M points, seeded synthetic data with the
benchmark's distribution) through ndb_b200_run_batched, inputs resident in HBM.
The same line carries, each measured in the same run:
  plain_gpu_form        the same jobs as one ndb_b200_run call each (the plain
                        GPU form the batched form is chosen over);
  tensor_filter_8d_2m   the 8-D 2M-point workload with the exact FP32 count (the
                        plain form), the tensor-core filtered count and the
                        library's automatic choice, in both count modes, with the
                        filter's guard-band population and an audit of every pair
                        it classified against FP64 distances and the exact
                        predicate;
  plain_3d_10m          the 10M-point 3-D workload on the plain path.
--config 1|2|3|5 times that one workload alone.

N > 1 runs under torchrun, one process per GPU: independent jobs do not need a
collective, so every rank runs its own replica of the step and the value is the
points all ranks clustered / the max over ranks of the timed device time
("scaling": "weak").

--impl reference times the reference's own OpenMP implementation (built from its
sources into oracle/_ref/) on the host cores, on a bounded sample of the same
workload; only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "clustered points/sec"
UNIT = "points/s"
HBM_PEAK_FALLBACK = 6650.0  # GB/s, used only without MEASURED_PEAKS.json
SM_COUNT = 148
FP32_LANES_PER_SM = 128
BATCH_JOBS = 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=4, help="benchmark configuration (1..5; 4, the default, is the batch)")
    ap.add_argument("--n", type=int, default=None, help="override n (smaller runs for profiling)")
    ap.add_argument("--full-count", action="store_true", help="exact neighbour counts (no early exit)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="configuration 4: skip the 8-D and 3-D workloads carried in the same line")
    ap.add_argument("--cpu-sample", type=int, default=50_000, help="points in the bounded CPU sample")
    ap.add_argument("--jobs", type=int, default=BATCH_JOBS, help="jobs of the batched configuration 4")
    ap.add_argument("--count-kernel", choices=["auto", "exact", "tensor"], default="auto",
                    help="neighbour-count kernel for d >= 8: picked per item (auto), exact FP32 only, or tensor filter")
    ap.add_argument("--autotune", action="store_true",
                    help="d >= 8: pick the count-kernel thresholds on the workload before timing")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form comparisons")
    ap.add_argument("--dims", type=str, default=None,
                    help="configuration 4: keep only the jobs of these dimensionalities (comma list)")
    ap.add_argument("--max-jobs", type=int, default=None, help="configuration 4: keep at most this many jobs")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_PEAK_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._stop.clear()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 9:
                for i, nm in enumerate(names):
                    if s[5 + i].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(val: float, world: int) -> float:
    """Largest value over the ranks (timing: the slowest rank sets the job time).
    NCCL groups reduce a device tensor, gloo groups (CPU tests) a host one."""
    if world == 1:
        return val
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([val], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, local_ms: float, world: int) -> tuple[float, float]:
    """Replicas: every rank processes units_per_rank per step; the whole job's rate
    is all ranks' units over the slowest rank's device time."""
    total_ms = max_over_ranks(local_ms, world)
    return world * units_per_rank * steps / (total_ms / 1000.0), total_ms


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# reference arm: the reference's own OpenMP implementation on the host cores
# ---------------------------------------------------------------------------
def _ensure_ref():
    import oracle

    if not oracle.have_ref():
        try:
            oracle.build()
        except Exception:
            pass
    return oracle


def cpu_reference(pkg, config: int, sample_n: int, threads: int, steps: int = 1, warmup: int = 0):
    oracle = _ensure_ref()
    import inspect
    full_n = inspect.signature(getattr(pkg.synthetic, f"config{config}")).parameters["n"].default
    if full_n <= 100_000:  # the 2-D 100k workload is timed whole: a few seconds of reference work
        sample_n = full_n
    w = pkg.synthetic.make(config, n=min(sample_n, full_n))
    if oracle.have_ref():
        kind = "reference"
        times = []
        for i in range(warmup + steps):
            _, _, _, info = oracle.run_ref(w.coords, w.eps, w.min_pts, threads=threads)
            if i >= warmup:
                times.append(info["total_ms"] / 1000.0)
        cores = threads
    else:
        kind = "port"
        times = []
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            oracle.grid(w.coords, w.eps, w.min_pts)
            if i >= warmup:
                times.append(time.perf_counter() - t0)
        cores = oracle.threads()
    per_step = sum(times) / len(times)
    whole = w.n == full_n
    return {
        "value": w.n / per_step, "unit": UNIT, "cores": cores, "kind": kind,
        # O(n^2) work: time grows with n^2, so the rate falls with n
        "extrapolated_value_at_full_n": w.n / per_step * w.n / full_n, "full_n": full_n,
        "sample": ((f"the whole {w.name} workload (n={w.n}, eps={w.eps}, minPts={w.min_pts})" if whole else
                    f"{w.name} generator at n={w.n} (same eps={w.eps}, minPts={w.min_pts})") +
                   f"; {'reference OpenMP data_process (oracle/_ref)' if kind == 'reference' else 'oracle grid port'}"
                   f", {cores} threads, {per_step:.2f} s per job" +
                   ("" if whole else "; the reference is O(n^2), so its rate at the full n is lower by about "
                                     "n_full/n_sample")),
        "seconds_per_step": per_step,
        "workload": w.name,
    }


def batch_sample(pkg, n_jobs: int = 24, n_cap: int = 40_000):
    """The bounded CPU sample of the batched configuration: the first n_jobs jobs of
    the 4,096-job batch (same generator, same seed) whose n is at most n_cap."""
    jobs = pkg.synthetic.config4(n_jobs=128)
    return [j for j in jobs if j.n <= n_cap][:n_jobs]


def cpu_reference_batch(pkg, threads: int, steps: int = 1, warmup: int = 0):
    oracle = _ensure_ref()
    jobs = batch_sample(pkg)
    pts = sum(j.n for j in jobs)
    times = []
    kind = "reference" if oracle.have_ref() else "port"
    for i in range(warmup + steps):
        t = 0.0
        for j in jobs:
            if kind == "reference":
                t += oracle.run_ref(j.coords, j.eps, j.min_pts, threads=threads)[3]["total_ms"] / 1000.0
            else:
                t0 = time.perf_counter()
                oracle.grid(j.coords, j.eps, j.min_pts)
                t += time.perf_counter() - t0
        if i >= warmup:
            times.append(t)
    per_step = sum(times) / len(times)
    cores = threads if kind == "reference" else oracle.threads()
    # the reference's time per job grows with n^2: the whole batch takes
    # per_step * sum(n^2 over the batch) / sum(n^2 over the sample)
    shapes = pkg.synthetic.config4_shapes(n_jobs=BATCH_JOBS)
    full_pts = sum(n for n, _ in shapes)
    full_sq = sum(float(n) * n for n, _ in shapes)
    sample_sq = sum(float(j.n) * j.n for j in jobs)
    return {
        "value": pts / per_step, "unit": UNIT, "cores": cores, "kind": kind,
        "extrapolated_value_at_full_n": full_pts / (per_step * full_sq / sample_sq), "full_n": full_pts,
        "sample": (f"the first {len(jobs)} jobs with n <= 40,000 of the 4,096-job batch ({pts} points, "
                   f"d in {sorted({j.d for j in jobs})}); "
                   f"{'reference OpenMP data_process (oracle/_ref)' if kind == 'reference' else 'oracle grid port'}"
                   f", one job after another, {cores} threads, {per_step:.2f} s; the reference is O(n^2) per job, "
                   f"so the whole batch (mean n 37k, up to 200k) is extrapolated by the sum of n^2"),
        "seconds_per_step": per_step,
        "workload": "batched-4096-jobs",
    }


def run_reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import importlib
    pkg = importlib.import_module("nextdbscan-exa_b200")
    threads = os.cpu_count() or 1
    if args.config == 4:
        cb = cpu_reference_batch(pkg, threads, steps=args.steps, warmup=args.warmup)
    else:
        cb = cpu_reference(pkg, args.config, args.cpu_sample, threads, steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["seconds_per_step"] * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator, benchmark distribution)",
        "config": {"workload": cb["workload"], "sample": cb["sample"], "parallelism": "host OpenMP"},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                            "extrapolated_value_at_full_n", "full_n") if k in cb},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def timed(fn, steps: int, flush, stream) -> list[float]:
    """Device time (ms) of fn() per step on the library's stream, L2 flushed before
    each step (not timed)."""
    import torch
    out = []
    for _ in range(steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def kernel_times(stats: list[dict]) -> dict:
    return {
        "count_kernel": statistics.mean(s["ms_count_kernel"] for s in stats),
        "union_kernel": statistics.mean(s["ms_union_kernel"] for s in stats),
        "border_kernel": statistics.mean(s["ms_border_kernel"] for s in stats),
        "radix_sort": statistics.mean(s["ms_sort_kernels"] for s in stats),
    }


def measure_workload(pkg, ctx, w, steps: int, warmup: int, flush, stream, full: bool, ck_kw: dict, e2e: bool,
                     world: int, clk=None) -> dict:
    """One workload on the single-job path: device-resident steps, then the same
    job through the public call with pinned host buffers (e2e)."""
    import torch
    n, d = w.n, w.d
    x = torch.from_numpy(w.coords).cuda()
    nn = torch.empty(n, dtype=torch.int32, device="cuda")
    ci = torch.empty(n, dtype=torch.int32, device="cuda")
    box = {"stats": []}

    def step():
        box["res"] = ctx.run_device(x.data_ptr(), n, d, w.eps, w.min_pts, nn.data_ptr(), ci.data_ptr(),
                                    full_count=full, **ck_kw)
        box["stats"].append(ctx.stats())

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    box["stats"] = []
    if clk is not None:
        with clk:
            ms = timed(step, steps, flush, stream)
    else:
        ms = timed(step, steps, flush, stream)
    torch.cuda.synchronize()
    barrier(world)
    value, total_ms = whole_job_rate(n, steps, sum(ms), world)
    out = {"value": value, "ms_per_step": total_ms / steps, "res": box["res"], "stats": box["stats"]}
    if e2e:
        hx = torch.from_numpy(w.coords).pin_memory()
        hnn = torch.empty(n, dtype=torch.int32).pin_memory()
        hci = torch.empty(n, dtype=torch.int32).pin_memory()

        def e2e_step():
            ctx.run_ptrs(hx.data_ptr(), n, d, w.eps, w.min_pts, hnn.data_ptr(), hci.data_ptr(), device=False,
                         full_count=full, **ck_kw)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        e_ms = timed(e2e_step, steps, flush, stream)
        e_total = max_over_ranks(sum(e_ms), world)
        out["e2e"] = {"value": world * n * steps / (e_total / 1000.0), "unit": UNIT,
                      "h2d_bytes_per_step": n * d * 4, "d2h_bytes_per_step": 2 * n * 4}
    return out


def roofline_of(stats: list[dict], n: int, workload: str, clk: dict) -> dict:
    """Roofline of the dominant kernel of a measured workload."""
    hbm_peak, peak_src = peaks()
    kern = kernel_times(stats)
    s0 = stats[-1]
    dominant = max(kern, key=kern.get)
    roof = roofline(dominant, kern[dominant], s0, n, hbm_peak, peak_src, clk)
    tkey = "tensor_count_kernel" if (dominant == "count_kernel" and s0["tensor_items"]) else dominant
    roof["traffic"] = traffic_per_launch(workload, tkey, n)
    roof["traffic_source"] = "profiles/traffic_per_launch.md (ncu capture, scaled by n)" if roof["traffic"] else None
    return roof


def summary_of(stats: list[dict]) -> dict:
    s0 = stats[-1]
    return {
        "phases_ms": {k: round(statistics.mean(s[k] for s in stats), 4)
                      for k in ("ms_grid", "ms_count", "ms_union", "ms_border")},
        "kernels_ms": {k: round(v, 4) for k, v in kernel_times(stats).items()},
        "pairs": {"count": s0["count_pairs"], "union": s0["union_pairs"], "border": s0["border_pairs"]},
        "grid": {"cells": s0["n_cells"], "tiles": s0["n_tiles"], "rows": s0["stencil_rows"],
                 "same_cell_linked": s0["same_cell_linked"], "key_bits": s0["key_bits"]},
        "kernel_launches_per_step": s0["kernel_launches"],
    }


def tensor_filter_forms(pkg, ctx, steps: int, flush, stream) -> dict:
    """The 8-D 2M-point workload: the exact FP32 count (the plain form), the
    tensor-core filtered count and the library's automatic choice, in both count
    modes, each timed on device-resident inputs with identical ids checked; then one
    audited run of the filter (NDB_FLAG_FILTER_AUDIT, untimed)."""
    import numpy as np
    import torch
    w = pkg.synthetic.config3()
    n, d = w.n, w.d
    x = torch.from_numpy(w.coords).cuda()
    nn = torch.empty(n, dtype=torch.int32, device="cuda")
    ci = torch.empty(n, dtype=torch.int32, device="cuda")
    out = {"workload": w.name, "n": n, "d": d, "eps": w.eps, "min_pts": w.min_pts,
           "l2": "flushed between timed steps", "steps": steps}
    for mode, full in (("early_exit", False), ("full_counts", True)):
        forms, ref = {}, None
        for name, kw in (("exact_fp32_count", {"exact_count": True}), ("tensor_filter_count", {"tensor_filter": True}),
                         ("chosen", {})):
            def run(kw=kw):
                ctx.run_device(x.data_ptr(), n, d, w.eps, w.min_pts, nn.data_ptr(), ci.data_ptr(), full_count=full,
                               **kw)
            run()
            torch.cuda.synchronize()
            ms = timed(run, steps, flush, stream)
            s = ctx.stats()
            ids = ci.cpu().numpy()
            if ref is None:
                ref = (ids, nn.cpu().numpy())
            f = {"value": n * len(ms) / (sum(ms) / 1000.0), "unit": UNIT, "ms_per_step": sum(ms) / len(ms),
                 "count_kernel_ms": s["ms_count_kernel"], "tensor_filter": bool(s["tensor_filter"]),
                 "tensor_items": s["tensor_items"], "of_items": s["n_tiles"], "band_pairs": s["band_pairs"],
                 "count_pairs": s["count_pairs"], "identical_cluster_ids": bool(np.array_equal(ids, ref[0]))}
            if full:
                f["identical_counts"] = bool(np.array_equal(nn.cpu().numpy(), ref[1]))
            forms[name] = f
        ex, tf, ch = forms["exact_fp32_count"], forms["tensor_filter_count"], forms["chosen"]
        forms["tensor_over_exact"] = ex["ms_per_step"] / tf["ms_per_step"]
        forms["tensor_over_exact_count_kernel"] = ex["count_kernel_ms"] / tf["count_kernel_ms"]
        forms["chosen_over_plain"] = ex["ms_per_step"] / ch["ms_per_step"]
        # the audit: every pair the filter classified, against FP64 and the exact predicate
        ctx.run_device(x.data_ptr(), n, d, w.eps, w.min_pts, nn.data_ptr(), ci.data_ptr(), full_count=full,
                       tensor_filter=True, audit=True)
        torch.cuda.synchronize()
        s = ctx.stats()
        forms["filter_audit"] = {
            "pairs": s["filter_audited_pairs"], "band_pairs": s["band_pairs"],
            "band_fraction": s["band_pairs"] / max(s["filter_audited_pairs"], 1),
            "max_abs_distance_error_vs_fp64": s["filter_max_abs_err"],
            "max_error_over_guard_bound": s["filter_max_err_over_bound"],
            "misclassified_pairs": s["filter_misclassified_pairs"],
            "identical_cluster_ids": bool(np.array_equal(ci.cpu().numpy(), ref[0])),
        }
        out[mode] = forms
    return out


def run_ours(args):
    import importlib

    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pkg = importlib.import_module("nextdbscan-exa_b200")
    w = pkg.synthetic.make(args.config, n=args.n)
    n, d = w.n, w.d
    stream = torch.cuda.current_stream()
    ctx = pkg.Context(local)
    ctx.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    full = args.full_count
    ck_kw = {"exact": {"exact_count": True}, "tensor": {"tensor_filter": True}}.get(args.count_kernel, {})
    tuning = None
    if args.autotune and d >= 8 and not ck_kw:
        # untimed: the count-kernel thresholds picked on this workload, then left on the context
        r = pkg.autotune.tune_count(ctx, w.coords, w.eps, w.min_pts, full_count=full)
        tuning = {"best": r["best"],
                  "count_kernel_ms": {f"min_dim={c['tc_min_dim']},min_item={c['tc_min_item']},gram={c['gram_filter']}":
                                      round(c["ms_count_kernel"], 4) for c in r["table"]}}
    clk = ClockSampler(local)
    m = measure_workload(pkg, ctx, w, args.steps, args.warmup, flush, stream, full, ck_kw, not args.no_e2e, world,
                         clk)
    clk_sum = clk.summary()
    stats = m["stats"]
    s0 = stats[-1]
    forms = None
    if args.config == 3 and not args.no_plain and rank == 0:
        forms = tensor_filter_forms(pkg, ctx, args.steps, flush, stream)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference(pkg, args.config, args.cpu_sample, os.cpu_count() or 1)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                  "extrapolated_value_at_full_n", "full_n") if k in cb}
    res = m["res"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator with the benchmark's distribution)",
            "config": {"workload": w.name, "n": n, "d": d, "eps": w.eps, "min_pts": w.min_pts,
                       "counts": "exact" if full else "early-exit at minPts (exact core flags and labels)",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "e2e": m.get("e2e"), "roofline": roofline_of(stats, n, w.name, clk_sum), "cpu_baseline": cpu,
            "clocks": clk_sum, "gpu_launches": count_launches(s0) * args.steps, "count_forms": forms,
            "tuning": tuning,
            "tensor_filter": {"used": bool(s0["tensor_filter"]), "items": s0["tensor_items"], "of_items": s0["n_tiles"],
                              "band_pairs": s0["band_pairs"]},
            "result": {"clusters": res.clusters, "noise": res.noise, "core_count": res.core_count},
            **summary_of(stats),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ours_batch(args):
    """Configuration 4: 4,096 independent jobs per step through ndb_b200_run_batched
    (the chosen form), beside the same jobs as one ndb_b200_run call each (the
    plain GPU form)."""
    import importlib

    import numpy as np
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    pkg = importlib.import_module("nextdbscan-exa_b200")
    lib = pkg.lib
    jobs = pkg.synthetic.config4(n_jobs=args.jobs)
    if args.dims:
        keep = {int(v) for v in args.dims.split(",")}
        jobs = [j for j in jobs if j.d in keep]
    if args.max_jobs:
        jobs = jobs[:args.max_jobs]
    nj = len(jobs)
    sizes = np.array([j.n for j in jobs], np.int64)
    dims = np.array([j.d for j in jobs], np.int64)
    total = int(sizes.sum())
    foff = np.concatenate([[0], np.cumsum(sizes * dims)])
    poff = np.concatenate([[0], np.cumsum(sizes)])
    flat = np.empty(int(foff[-1]), np.float32)
    for k, j in enumerate(jobs):
        flat[foff[k]:foff[k + 1]] = j.coords.ravel()
    stream = torch.cuda.current_stream()
    ctx = pkg.Context(local)
    ctx.set_stream(stream.cuda_stream)
    x = torch.from_numpy(flat).cuda()
    nn = torch.empty(total, dtype=torch.int32, device="cuda")
    ci = torch.empty(total, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def job_table(xp, nnp, cip):
        arr = (lib.NdbJob * nj)()
        for k, j in enumerate(jobs):
            arr[k].coords = xp + 4 * int(foff[k])
            arr[k].n, arr[k].d, arr[k].eps, arr[k].min_pts = j.n, j.d, j.eps, j.min_pts
            arr[k].nn_out = nnp + 4 * int(poff[k])
            arr[k].cluster_index_out = cip + 4 * int(poff[k])
        return arr

    full = (lib.FLAG_FULL_COUNT if args.full_count else 0) | {"exact": lib.FLAG_EXACT_COUNT,
                                                              "tensor": lib.FLAG_TENSOR_FILTER}.get(args.count_kernel, 0)
    dev_jobs = job_table(x.data_ptr(), nn.data_ptr(), ci.data_ptr())
    torch.cuda.synchronize()
    stats = []

    def step():
        st = ctx.run_batched_jobs(dev_jobs, nj, lib.FLAG_DEVICE_PTRS | full)
        if st != 0:
            raise lib.NdbError(st, "ndb_b200_run_batched")
        stats.append(ctx.stats())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    stats.clear()
    with ClockSampler(local) as clk:
        step_ms = timed(step, args.steps, flush, stream)
    torch.cuda.synchronize()
    barrier(world)
    value, total_ms = whole_job_rate(total, args.steps, sum(step_ms), world)
    h_ci = ci.cpu().numpy()
    clusters = sum(int(dev_jobs[k].result.clusters) for k in range(nj))
    noise = sum(int(dev_jobs[k].result.noise) for k in range(nj))
    cores = sum(int(dev_jobs[k].result.core_count) for k in range(nj))

    # the plain GPU form: the same jobs, one ndb_b200_run call each
    plain = None
    if not args.no_plain:
        def plain_step():
            for k, j in enumerate(jobs):
                ctx.run_device(x.data_ptr() + 4 * int(foff[k]), j.n, j.d, j.eps, j.min_pts,
                               nn.data_ptr() + 4 * int(poff[k]), ci.data_ptr() + 4 * int(poff[k]),
                               full_count=bool(full & lib.FLAG_FULL_COUNT))
        plain_step()
        torch.cuda.synchronize()
        p_ms = timed(plain_step, max(1, min(args.steps, 3)), flush, stream)
        same = bool(np.array_equal(ci.cpu().numpy(), h_ci))
        pv = total * len(p_ms) / (sum(p_ms) / 1000.0)
        plain = {"value": pv, "unit": UNIT, "ms_per_step": sum(p_ms) / len(p_ms), "steps": len(p_ms),
                 "form": "one ndb_b200_run call per job, device-resident inputs",
                 "chosen_over_plain": value / world / pv, "identical_cluster_ids": same}

    e2e = None
    if not args.no_e2e:
        hx = torch.from_numpy(flat).pin_memory()
        hnn = torch.empty(total, dtype=torch.int32).pin_memory()
        hci = torch.empty(total, dtype=torch.int32).pin_memory()
        host_jobs = job_table(hx.data_ptr(), hnn.data_ptr(), hci.data_ptr())

        def e2e_step():
            st = ctx.run_batched_jobs(host_jobs, nj, full)
            if st != 0:
                raise lib.NdbError(st, "ndb_b200_run_batched")

        e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        e_ms = timed(e2e_step, args.steps, flush, stream)
        e_total = max_over_ranks(sum(e_ms), world)
        assert np.array_equal(hci.numpy(), h_ci), "host-buffer batch differs from the device-buffer batch"
        e2e = {"value": world * total * args.steps / (e_total / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": int(flat.nbytes), "d2h_bytes_per_step": 2 * total * 4}

    clk_sum = clk.summary()
    roof = roofline_of(stats, total, "batched-4096-jobs", clk_sum)
    roof["note"] = "summed over the pipelines of one batched call (one per dimensionality)"
    s0 = stats[-1]
    launches = count_launches(s0) * args.steps

    # the other chosen form and the plain path at scale, measured in the same run
    extras = {}
    if rank == 0 and not args.no_extras:
        del x, nn, ci
        torch.cuda.empty_cache()
        extras["tensor_filter_8d_2m"] = tensor_filter_forms(pkg, ctx, args.steps, flush, stream)
        w2 = pkg.synthetic.config2()
        m2 = measure_workload(pkg, ctx, w2, args.steps, args.warmup, flush, stream, False, {}, not args.no_e2e, 1)
        extras["plain_3d_10m"] = {
            "workload": w2.name, "n": w2.n, "d": w2.d, "eps": w2.eps, "min_pts": w2.min_pts,
            "value": m2["value"], "unit": UNIT, "ms_per_step": m2["ms_per_step"], "e2e": m2.get("e2e"),
            "roofline": roofline_of(m2["stats"], w2.n, w2.name, clk_sum),
            "result": {"clusters": m2["res"].clusters, "noise": m2["res"].noise, "core_count": m2["res"].core_count},
            **summary_of(m2["stats"]),
        }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_batch(pkg, os.cpu_count() or 1)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                  "extrapolated_value_at_full_n", "full_n") if k in cb}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator with the benchmark's distribution)",
            "config": {"workload": "batched-4096-jobs" if nj == BATCH_JOBS else f"batched-subset-{nj}-jobs",
                       "jobs": nj, "points": total,
                       "points_by_d": {int(d): int(sizes[dims == d].sum()) for d in np.unique(dims)},
                       "eps": "per job: 90th percentile of the 4-NN distance over a 1% sample",
                       "min_pts": "2d", "form": "ndb_b200_run_batched, device-resident inputs",
                       "counts": "exact" if args.full_count else "early-exit at minPts (exact core flags and labels)",
                       "l2": "flushed between timed steps (256 MB write); inputs 4.4 GB",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "e2e": e2e, "plain_gpu_form": plain, "roofline": roof, "cpu_baseline": cpu, "clocks": clk_sum,
            "gpu_launches": launches,
            "result": {"clusters": clusters, "noise": noise, "core_count": cores},
            "pipelines": s0["pipelines"], "solo_jobs": s0["solo_jobs"],
            "tensor_filter": {"used": bool(s0["tensor_filter"]), "items": s0["tensor_items"], "of_items": s0["n_tiles"],
                              "band_pairs": s0["band_pairs"]},
            **summary_of(stats),
            **extras,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def traffic_per_launch(workload: str, kernel: str, n: int):
    """DRAM bytes per launch of kernel on workload, from the committed ncu captures
    (profiles/traffic_per_launch.md), scaled by points; None when not captured."""
    p = os.path.join(ROOT, "profiles", "traffic_per_launch.md")
    try:
        for line in open(p):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) >= 4 and cells[0] == workload and cells[1] == kernel and cells[2].isdigit():
                return int(cells[3]) * n / int(cells[2])
    except OSError:
        pass
    return None


def count_launches(s) -> int:
    """Kernels of one step, as counted by the library at every launch site."""
    return int(s["kernel_launches"])


def roofline(kind, ms, s, n, hbm_peak, peak_src, clk):
    """Algorithmic work of one launch / its device time."""
    if kind == "radix_sort":
        kb = s["key_bytes"]
        # per pass: upsweep reads keys; downsweep reads and writes (key, id)
        per_pass = s["n_valid"] * (kb + 2 * (kb + 4))
        achieved = per_pass * s["sort_passes"] / max(s.get("pipelines") or 1, 1) / (ms / 1000.0) / 1e9
        return {"kernel": "radix_sort (all passes)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "peak_source": f"{peak_src} hbm_gbs"}
    if kind == "union_kernel":
        # union-find over random parents: 8 bytes per tested core pair (two parent
        # reads) + 12 per point (core flag, parent write, label write)
        ab = 8 * s["union_pairs"] + 12 * s["n_valid"]
        achieved = ab / (ms / 1000.0) / 1e9
        return {"kernel": "union (main kernel)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "peak_source": f"{peak_src} hbm_gbs", "work": f"{ab} algorithmic bytes"}
    pairs = {"count_kernel": s["count_pairs"], "union_kernel": s["union_pairs"],
             "border_kernel": s["border_pairs"]}[kind]
    pair_dims = {"count_kernel": s["count_pair_dims"], "union_kernel": s["union_pair_dims"],
                 "border_kernel": s["border_pair_dims"]}[kind]
    # FP32 pipe operations: the exact sum takes a separately rounded sub, mul and add per
    # dimension (no FMA credit); the Gram filter one FMA per dimension plus three
    flops = s.get("count_fp32_ops") if kind == "count_kernel" and s.get("count_fp32_ops") else pair_dims * 3
    achieved = flops / (ms / 1000.0) / 1e12
    mhz = clk.get("sm_mhz") or 1965.0
    peak = SM_COUNT * FP32_LANES_PER_SM * mhz * 1e6 / 1e12
    return {"kernel": kind, "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None,
            "peak_source": "nominal FP32 issue rate (148 SMs x 128 lanes) at the median sampled SM clock; "
                           "no FP32 figure in MEASURED_PEAKS.json",
            "work": f"{pairs} pair predicates, {flops} FP32 pipe operations"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.config == 4:
        return run_ours_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
