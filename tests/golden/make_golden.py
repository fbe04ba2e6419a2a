"""Generates tests/golden/*.npz and c1_full.json from the REFERENCE implementation.

Every fixture's expected outputs come from nextdbscan-exa's own OpenMP code path
(data_process.cpp, compiled from the reference sources by oracle/Makefile into
oracle/_ref/ndb_ref_harness), never from this repository's code.  Inputs come from
the seeded generators in nextdbscan-exa_b200/synthetic.py or are built here from a
fixed seed.

usage: python tests/golden/make_golden.py [--ref-dir /path/to/nextdbscan-exa]
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

pkg = importlib.import_module("nextdbscan-exa_b200")

FLT_MAX = np.finfo(np.float32).max


def blobs(rng, d, n=2500, k=6, box=20.0, sigma=0.7, noise=200):
    c = rng.uniform(0, box, (k, d))
    lab = rng.integers(0, k, n)
    x = (c[lab] + rng.normal(0, sigma, (n, d))).astype(np.float32)
    return np.concatenate([x, rng.uniform(0, box, (noise, d)).astype(np.float32)])


def border_tie():
    """Two dense clusters; border points within eps of cores of both clusters, and
    of a single cluster, and of none."""
    a = np.array([[x * 0.1, y * 0.1] for x in range(5) for y in range(5)], np.float32)
    b = a + np.float32(2.0)
    pts = [a, b,
           np.array([[1.0, 1.0], [0.95, 1.05]], np.float32),   # near both blocks
           np.array([[-0.5, 0.0]], np.float32),                # near block a only
           np.array([[10.0, 10.0]], np.float32)]               # noise
    return np.concatenate(pts)


def boundary_pairs():
    """Pairs whose FP32 length is exactly e2, one ulp below and one ulp above."""
    e = np.float32(0.5)
    e2 = np.float32(e * e)
    rng = np.random.default_rng(7)
    out = []
    while len(out) < 600:
        p = rng.uniform(0, 50, 2).astype(np.float32)
        dx = np.float32(rng.uniform(0, 0.5))
        dy = np.float32(np.sqrt(np.float64(e2) - np.float64(dx) ** 2))
        for delta in (-2, -1, 0, 1, 2):
            q = np.array([p[0] + dx, np.nextafter(p[1] + dy, np.float32(np.inf) if delta > 0 else
                                                  np.float32(-np.inf)) if delta else p[1] + dy], np.float32)
            for _ in range(abs(delta) - 1 if abs(delta) > 1 else 0):
                q[1] = np.nextafter(q[1], np.float32(np.inf) if delta > 0 else np.float32(-np.inf))
            out.append(p)
            out.append(q)
    return np.asarray(out, np.float32), float(e)


def specials(rng):
    x = rng.normal(0, 1, (1500, 3)).astype(np.float32)
    x[::37, 1] = np.nan
    x[5::41, 2] = np.inf
    x[11::53, 1] = -np.inf
    x[7::43, 0] = FLT_MAX
    x[9::47, 0] = -FLT_MAX
    x[13::59, 2] = FLT_MAX
    return x


def cases():
    rng = np.random.default_rng(20261203)
    out = []
    w = pkg.synthetic.config1(n=4000)
    out.append(("c1_n4000", w.coords, w.eps, w.min_pts))
    w = pkg.synthetic.config2(n=6000)
    out.append(("c2_n6000", w.coords, w.eps, 3))
    w = pkg.synthetic.config3(n=4000)
    out.append(("c3_n4000", w.coords, w.eps, w.min_pts))
    for d, eps in ((1, 0.05), (2, 0.3), (3, 0.6), (4, 0.9), (5, 1.1), (8, 1.8), (16, 3.0)):
        out.append((f"blobs_d{d}", blobs(rng, d), eps, 5))
    lat = rng.integers(0, 30, (3000, 2)).astype(np.float32)
    out.append(("lattice2d_eps1", lat, 1.0, 4))
    out.append(("lattice2d_eps_sqrt2", lat, 1.4142135, 5))
    lat3 = (rng.integers(0, 40, (3000, 3)) * 0.1).astype(np.float32)
    out.append(("lattice3d_eps0.1", lat3, 0.1, 3))
    out.append(("lattice3d_eps_diag", lat3, 0.17320508, 6))
    bp, e = boundary_pairs()
    out.append(("boundary_pairs", bp, e, 2))
    dup = np.repeat(rng.uniform(0, 10, (50, 2)).astype(np.float32), 20, axis=0)
    out.append(("duplicates_eps0", dup, 0.0, 5))
    out.append(("duplicates_negative_eps", dup, -0.5, 25))
    sp = specials(rng)
    out.append(("specials_m4", sp, 0.4, 4))
    out.append(("specials_m0", sp, 0.4, 0))
    out.append(("specials_m1", sp, 0.4, 1))
    out.append(("all_noise", rng.uniform(0, 1000, (800, 2)).astype(np.float32), 0.5, 3))
    out.append(("single_cluster", rng.normal(0, 0.05, (1000, 3)).astype(np.float32), 0.5, 5))
    out.append(("tiny_coords", (rng.normal(0, 1, (1500, 2)) * 1e-30).astype(np.float32), 3e-31, 4))
    out.append(("border_tie", border_tie(), 0.2, 5))
    out.append(("n1", np.zeros((1, 2), np.float32), 1.0, 1))
    out.append(("n2", np.array([[0, 0], [1, 0]], np.float32), 1.0, 2))
    out.append(("minpts_large", blobs(rng, 2, n=1500), 0.3, 100000))
    return out


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-dir", default=None, help="reference checkout (default: $NDB_REF_DIR or the build's mount)")
    ap.add_argument("--skip-full", action="store_true")
    args = ap.parse_args()
    oracle.build(args.ref_dir or oracle.ref_dir())
    if not oracle.have_ref():
        raise SystemExit("reference harness could not be built")
    for name, x, eps, m in cases():
        nn, ci, lab, info = oracle.run_ref(x, eps, m, threads=4)
        # approximate mode is schedule dependent in the reference; pin it single threaded
        nn_a, ci_a, lab_a, info_a = oracle.run_ref(x, eps, m, threads=1, approximate=True)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), coords=x, eps=np.float32(eps), min_pts=np.int32(m),
                            nn=nn, cluster_index=ci, cluster_label=lab,
                            meta=np.array([info["clusters"], info["noise"], info["cores"], info["n"]], np.int32),
                            approx_cluster_index=ci_a, approx_cluster_label=lab_a,
                            approx_meta=np.array([info_a["clusters"], info_a["noise"], info_a["cores"],
                                                  info_a["n"]], np.int32))
        print(f"{name}: n={x.shape[0]} d={x.shape[1]} {info}")
    if not args.skip_full:
        w = pkg.synthetic.config1()
        nn, ci, lab, info = oracle.run_ref(w.coords, w.eps, w.min_pts, threads=os.cpu_count() or 1)
        doc = {
            "workload": w.name, "n": w.n, "d": w.d, "eps": w.eps, "min_pts": w.min_pts,
            "coords_sha256": sha(w.coords.astype("<f4")),
            "nn_sha256": sha(nn.astype("<i4")), "cluster_index_sha256": sha(ci.astype("<i4")),
            "roots_sha256": sha(np.nonzero(lab == np.arange(lab.size))[0].astype("<i4")),
            "clusters": info["clusters"], "noise": info["noise"], "cores": info["cores"],
            "reference_threads": info["threads"], "reference_total_ms": info["total_ms"],
        }
        with open(os.path.join(HERE, "c1_full.json"), "w") as f:
            json.dump(doc, f, indent=1)
        print("c1_full:", doc)


if __name__ == "__main__":
    main()
