"""The C++ side of the boundary: the command line (nextdbscan-exa_b200/cli) and the
header-only data_process drop-in (include/ndb_b200_data_process.h), compiled with
g++ against libndb_b200.so the way the reference's build would use them.

On the CPU: both compile, and the error paths the reference has (no arguments, no
-m/-e, unreadable input, no device) print and exit non-zero.  On the GPU: the CLI's
label file and meta, and the drop-in's public vectors, equal the reference's
outputs in the golden fixtures."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, load_pkg

PKG_DIR = os.path.join(ROOT, "nextdbscan-exa_b200")
INCLUDE = os.path.join(ROOT, "include")

# a caller written the way nextdbscan::start drives data_process (nextdbscan.cpp:46-58)
DROPIN_MAIN = r"""
#include <cstdio>
#include <fstream>
#include <vector>
#include "ndb_b200_data_process.h"
struct one_rank {};
int main(int argc, char **argv) {
    std::ifstream is(argv[1], std::ios::binary);
    int n = 0, d = 0;
    is.read((char *)&n, 4);
    is.read((char *)&d, 4);
    std::vector<float> v_coord((size_t)n * d);
    is.read((char *)v_coord.data(), (std::streamsize)(v_coord.size() * 4));
    const int m = std::atoi(argv[2]);
    const float e = std::strtof(argv[3], nullptr);
    one_rank mpi;
    data_process dp(v_coord, m, e, d, n, false);
    dp.select_and_process(mpi);
    dp.select_cores_and_process(mpi);
    int cores = 0, noise = 0, clusters = 0, nn = 0;
    dp.get_result_meta(cores, noise, clusters, nn, mpi);
    std::printf("%d %d %d %d\n", clusters, noise, cores, nn);
    std::FILE *f = std::fopen(argv[4], "wb");
    std::fwrite(dp.v_coord_nn.data(), 4, dp.v_coord_nn.size(), f);
    std::fwrite(dp.v_coord_cluster_index.data(), 4, dp.v_coord_cluster_index.size(), f);
    std::fclose(f);
    return 0;
}
"""


def _gpp(src, out, extra=()):
    lib = load_pkg().lib.LIB_PATH
    if not os.path.exists(lib):
        load_pkg().lib.load()  # raises with the build hint
    cmd = ["g++", "-O2", "-std=c++14", "-I", INCLUDE, *extra, src, "-L", PKG_DIR, "-lndb_b200",
           f"-Wl,-rpath,{PKG_DIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.fixture(scope="module")
def binaries(tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp")
    cli = str(d / "nextdbscan-b200")
    _gpp(os.path.join(PKG_DIR, "cli", "nextdbscan_b200.cpp"), cli, ["-I", os.path.join(PKG_DIR, "cli")])
    src = d / "dropin.cpp"
    src.write_text(DROPIN_MAIN)
    dropin = str(d / "dropin")
    _gpp(str(src), dropin)
    return cli, dropin


def _write_bin(path, x):
    load_pkg().inputs.write_bin(str(path), np.ascontiguousarray(x, dtype=np.float32))


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_cli_and_dropin_compile_and_fail_like_the_reference(binaries, tmp_path):
    cli, dropin = binaries
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stdout
    r = subprocess.run([cli, "-m", "5", "x.bin"], capture_output=True, text=True)
    assert r.returncode != 0 and "specify the m and e" in r.stdout
    bad = tmp_path / "short.bin"
    bad.write_bytes(struct.pack("<ii", 10, 3) + b"\0" * 8)
    r = subprocess.run([cli, "-m", "5", "-e", "1", str(bad)], capture_output=True, text=True)
    assert r.returncode != 0
    if _cuda_available():
        return
    g = load_golden("c1_n4000")
    p = tmp_path / "c1.bin"
    _write_bin(p, g["coords"])
    for cmd in ([cli, "-m", "5", "-e", "0.8", str(p)], [dropin, str(p), "5", "0.8", str(tmp_path / "o")]):
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode != 0 and "no CUDA device" in r.stderr, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_n4000", "blobs_d3", "blobs_d8", "border_tie"])
def test_cli_labels_and_dropin_vectors_match_reference(binaries, tmp_path, name):
    cli, dropin = binaries
    g = load_golden(name)
    p = tmp_path / f"{name}.bin"
    _write_bin(p, g["coords"])
    eps, m = repr(float(np.float32(g["eps"]))), str(int(g["min_pts"]))
    out = tmp_path / "labels.txt"
    r = subprocess.run([cli, "-m", m, "-e", eps, "-f", "1", "-o", str(out), str(p)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    ci = np.loadtxt(out, dtype=np.int64).reshape(-1)
    np.testing.assert_array_equal(ci, g["cluster_index"].astype(np.int64))
    clusters, noise, cores, n = (int(v) for v in g["meta"])
    assert f"Estimated Clusters: {clusters}" in r.stdout
    assert f"Core Points: {cores}" in r.stdout and f"Noise Points: {noise}" in r.stdout
    vec = tmp_path / "vec.bin"
    r = subprocess.run([dropin, str(p), m, eps, str(vec)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert [int(v) for v in r.stdout.split()] == [clusters, noise, cores, n]
    raw = np.fromfile(vec, dtype=np.int32)
    np.testing.assert_array_equal(raw[:n], g["nn"])
    np.testing.assert_array_equal(raw[n:], g["cluster_index"])


# ---------------------------------------------------------------------------
# The reference's own caller: main.cpp and nextdbscan.cpp compiled unchanged, with
# the -DB200_ON switch added to a copy of its data_process.h (oracle/Makefile,
# target dropin), linked against libndb_b200.so.  The binary is built where the
# reference's sources are; elsewhere the prebuilt one is used.
# ---------------------------------------------------------------------------
REF_DROPIN = os.path.join(ROOT, "oracle", "_ref", "nextdbscan-dropin")


def _ref_dropin():
    import oracle

    if oracle.ref_dir():
        oracle.build(targets=("dropin",))
    if not os.path.exists(REF_DROPIN):
        pytest.skip("the reference's caller is not built here (no reference sources, no prebuilt binary)")
    return REF_DROPIN


def test_reference_caller_builds_against_the_dropin(tmp_path):
    exe = _ref_dropin()
    r = subprocess.run([exe, "-m", "5", str(tmp_path / "x.bin")], capture_output=True, text=True)
    assert r.returncode != 0 and "specify the m and e" in r.stdout  # main.cpp:80-84
    if _cuda_available():
        return
    g = load_golden("c1_n4000")
    p = tmp_path / "c1.bin"
    _write_bin(p, g["coords"])
    r = subprocess.run([exe, "-m", "5", "-e", "0.8", "-t", "1", str(p)], capture_output=True, text=True)
    assert r.returncode != 0 and "no CUDA device" in r.stderr, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1_n4000", "blobs_d3", "blobs_d8", "blobs_d16", "border_tie", "all_noise"])
def test_reference_caller_prints_the_reference_meta(tmp_path, name):
    """The reference's main.cpp through nextdbscan::start (nextdbscan.cpp:46-58) on the
    drop-in prints the clusters, core points and noise points of the reference's own
    run (main.cpp:98-106)."""
    exe = _ref_dropin()
    g = load_golden(name)
    p = tmp_path / f"{name}.bin"
    _write_bin(p, g["coords"])
    eps, m = repr(float(np.float32(g["eps"]))), str(int(g["min_pts"]))
    r = subprocess.run([exe, "-m", m, "-e", eps, "-t", "1", str(p)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    clusters, noise, cores, n = (int(v) for v in g["meta"])
    assert f"Read {n} aggregated points" in r.stdout
    assert f"Estimated Clusters: {clusters}" in r.stdout
    assert f"Core Points: {cores}" in r.stdout and f"Noise Points: {noise}" in r.stdout
