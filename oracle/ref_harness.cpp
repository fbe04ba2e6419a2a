// ref_harness.cpp -- drives the UNMODIFIED reference implementation (TEST INFRASTRUCTURE).
//
// oracle/Makefile compiles this file together with the reference's own
// data_process.cpp (OpenMP backend, -DOMP_ON=1, exactly the reference's flags:
// Makefile:11 "omp" target, with g++ in place of icc) into oracle/_ref/.  It does
// what nextdbscan::start does (nextdbscan.cpp:28-68): read the input with the
// reference reader (magma_input::read_input, magma_input.h:144-167), construct
// data_process, run select_and_process and select_cores_and_process, collect the
// meta -- and then dumps the public result vectors that start() throws away
// (data_process.h:53-59), so that tests and the CPU baseline can use them.
//
// usage: ndb_ref_harness -m minPts -e eps -t threads [-a 0|1] [-o out_prefix] input.bin|.csv
// writes <out_prefix>.nn.i32, <out_prefix>.ci.i32 (one int32 per point) and
// <out_prefix>.label.i32 (v_cluster_label, one int32 per core); prints one JSON line.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <omp.h>

// data_process.h defines h_vec, which magma_input.h needs (same order as nextdbscan.cpp:22-24).
#include "data_process.h"
#include "magma_input.h"

static void dump(const std::string &path, const std::vector<int> &v) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        std::exit(2);
    }
    if (!v.empty()) std::fwrite(v.data(), sizeof(int), v.size(), f);
    std::fclose(f);
}

int main(int argc, char **argv) {
    int m = -1, t = 1, a = 0;
    float e = -1;
    std::string out;
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s -m minPts -e eps -t threads [-a 0|1] [-o prefix] input\n", argv[0]);
        return 2;
    }
    for (int i = 1; i + 1 < argc; i += 2) {
        std::string s(argv[i]);
        if (s == "-m") m = std::atoi(argv[i + 1]);
        else if (s == "-e") e = std::strtof(argv[i + 1], nullptr); // main.cpp:71
        else if (s == "-t") t = std::atoi(argv[i + 1]);
        else if (s == "-a") a = std::atoi(argv[i + 1]);
        else if (s == "-o") out = argv[i + 1];
    }
    std::string input = argv[argc - 1];
    omp_set_num_threads(t);
    auto mpi = magmaMPI::build();

    h_vec<float> v_coord;
    int n_total = -1, n_dim = -1;
    magma_input::read_input(input, v_coord, n_total, n_dim, mpi.n_nodes, mpi.rank);
    if (n_total <= 0 || n_dim <= 0) {
        std::fprintf(stderr, "empty or unreadable input %s\n", input.c_str());
        return 2;
    }

    auto t0 = std::chrono::steady_clock::now();
    data_process dp(v_coord, m, e, n_dim, n_total, a == 1);
    dp.select_and_process(mpi);
    auto t1 = std::chrono::steady_clock::now();
    dp.select_cores_and_process(mpi);
    auto t2 = std::chrono::steady_clock::now();
    int cores = 0, noise = 0, clusters = 0, n = 0;
    dp.get_result_meta(cores, noise, clusters, n, mpi);
    auto t3 = std::chrono::steady_clock::now();

    auto ms = [](std::chrono::steady_clock::time_point x, std::chrono::steady_clock::time_point y) {
        return std::chrono::duration<double, std::milli>(y - x).count();
    };
    if (!out.empty()) {
        dump(out + ".nn.i32", dp.v_coord_nn);
        dump(out + ".ci.i32", dp.v_coord_cluster_index);
        dump(out + ".label.i32", dp.v_cluster_label);
    }
    std::printf("{\"n\": %d, \"d\": %d, \"clusters\": %d, \"noise\": %d, \"cores\": %d, "
                "\"threads\": %d, \"classify_ms\": %.3f, \"labels_ms\": %.3f, \"meta_ms\": %.3f, "
                "\"total_ms\": %.3f}\n",
                n, n_dim, clusters, noise, cores, t, ms(t0, t1), ms(t1, t2), ms(t2, t3), ms(t0, t3));
    return 0;
}
