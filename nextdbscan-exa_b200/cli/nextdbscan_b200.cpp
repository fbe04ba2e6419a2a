// nextdbscan_b200.cpp -- command-line front end with the reference's flags
// (main.cpp:57-129), running the B200 hot path through the C ABI (.bin input:
// ndb_b200_load_bin, file to device through pinned chunks) or the C++ drop-in
// (ndb_b200_data_process.h; .csv input).
//
//   nextdbscan-b200 -m minPts -e eps [-t threads] [-a 0|1] [-o labels.txt] input.bin|input.csv
//
// -o writes one cluster id per line, in input order: the per-point output the
// reference advertises but leaves unwritten (main.cpp:46, :108-123,
// data_process.cpp:90).  Noise is written as 2147483647 (NO_CLUSTER,
// data_process.h:26), cluster ids are the reference's (rank among cores of the
// component's smallest-index core).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "ndb_b200_data_process.h"
#include "ndb_input.h"

namespace {

struct one_rank {};  // stands in for magmaMPI (one GPU is one rank)

void usage() {
    std::cout << "NextDBSCAN compiled for B200 (sm_100a)" << std::endl << std::endl;
    std::cout << "Usage: [executable] -m minPoints -e epsilon -t threads [input file]" << std::endl;
    std::cout << "    -m minPoints : DBSCAN parameter, minimum number of points required to form a cluster, "
                 "postive integer, required" << std::endl;
    std::cout << "    -e epsilon   : DBSCAN parameter, maximum neighborhood search radius for cluster, positive "
                 "floating point, required" << std::endl;
    std::cout << "    -t threads   : accepted for compatibility; the GPU sets its own parallelism" << std::endl;
    std::cout << "    -a 0|1       : approximate mode flag (accepted; the B200 result is exact, a tight upper "
                 "bound)" << std::endl;
    std::cout << "    -o output    : Output file containing the cluster ids in the same order as the input"
              << std::endl;
    std::cout << "    -f 0|1       : 1 = exact neighbour counts for every point (default 0: counts stop at m)"
              << std::endl << std::endl;
    std::cout << "Supported Input Types:" << std::endl;
    std::cout << ".csv: Text file with one sample/point per line and features/dimensions separated by a space "
                 "delimiter, i.e. ' '" << std::endl;
    std::cout << ".bin: int32 n, int32 d, then n*d float32 values" << std::endl;
}

bool has_suffix(const std::string &s, const char *suf) {
    const std::string x(suf);
    return s.size() >= x.size() && s.compare(s.size() - x.size(), x.size(), x) == 0;
}

// The library's status as the reference treats hard errors: print and exit.
void check(ndb_status s, const char *where, ndb_ctx *ctx) {
    if (s == NDB_OK) return;
    std::cerr << "nextdbscan-b200: " << where << ": " << ndb_b200_strerror(s);
    if (ctx && *ndb_b200_last_cuda_error(ctx)) std::cerr << " (" << ndb_b200_last_cuda_error(ctx) << ")";
    std::cerr << std::endl;
    std::exit(EXIT_FAILURE);
}

long long ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t).count();
}

}  // namespace

int main(int argc, char **argv) {
    int m = -1, t = 1, a = 0, f = 0;
    float e = -1;
    std::string output_file;
    if (argc < 2) {
        usage();
        return EXIT_FAILURE;
    }
    for (int i = 1; i + 1 < argc; i += 2) {
        std::string s(argv[i]);
        if (s == "-m") m = std::atoi(argv[i + 1]);
        else if (s == "-e") e = std::strtof(argv[i + 1], nullptr);
        else if (s == "-t") t = std::atoi(argv[i + 1]);
        else if (s == "-a") a = std::atoi(argv[i + 1]);
        else if (s == "-o") output_file = argv[i + 1];
        else if (s == "-f") f = std::atoi(argv[i + 1]);
    }
    std::string input_file = argv[argc - 1];
    if (m == -1 || e == -1) {  // main.cpp:80-84
        std::cout << "Input Error: Please specify the m and e parameters" << std::endl << std::endl;
        usage();
        std::exit(EXIT_FAILURE);
    }
    std::cout << "Starting NextDBSCAN with file: " << input_file << " m: " << m << " e: " << e << " t: " << t
              << " a: " << a << std::endl;

    auto t0 = std::chrono::steady_clock::now();
    int cores = 0, noise = 0, clusters = 0, n = 0;
    std::vector<int> cluster_index;
    const uint32_t flags = (f == 1 ? NDB_FLAG_FULL_COUNT : 0u) | (a == 1 ? NDB_FLAG_APPROXIMATE : 0u);
    if (has_suffix(input_file, ".bin")) {
        // the binary input goes straight from the file to the device: pinned chunks,
        // each copied while the next is read (ndb_b200_load_bin)
        ndb_ctx *ctx = nullptr;
        check(ndb_b200_create(&ctx, 0), "ndb_b200_create", nullptr);
        int64_t n_total = 0;
        int32_t n_dim = 0;
        check(ndb_b200_load_bin(ctx, input_file.c_str(), &n_total, &n_dim), "ndb_b200_load_bin", ctx);
        std::cout << "Read Input Data: " << ms_since(t0) << " milliseconds" << std::endl;
        std::cout << "Read " << n_total << " aggregated points with " << n_dim << " dimensions. " << std::endl;
        auto t1 = std::chrono::steady_clock::now();
        std::vector<int> nn((size_t)n_total);
        cluster_index.resize((size_t)n_total);
        ndb_result r{};
        check(ndb_b200_run_loaded(ctx, e, m, flags, nn.data(), cluster_index.data(), &r), "ndb_b200_run_loaded", ctx);
        ndb_stats st{};
        ndb_b200_get_stats(ctx, &st);
        // phase times of the reference's printout (nextdbscan.cpp:48-57), from the device events
        std::cout << "Classify Points: " << (long long)(st.ms_grid + st.ms_count) << " milliseconds" << std::endl;
        std::cout << "Assign Labels: " << (long long)(st.ms_union + st.ms_border) << " milliseconds" << std::endl;
        cores = r.core_count;
        noise = r.noise;
        clusters = r.clusters;
        n = r.n;
        ndb_b200_destroy(ctx);
        std::cout << "Total Execution Time: " << ms_since(t0) << " milliseconds" << std::endl;
        std::cout << "Total Execution Time (without I/O): " << ms_since(t1) << " milliseconds" << std::endl;
    } else {
        std::vector<float> v_coord;
        int n_total = -1, n_dim = -1;
        if (!ndb_input::read_input(input_file, v_coord, n_total, n_dim)) return EXIT_FAILURE;
        std::cout << "Read Input Data: " << ms_since(t0) << " milliseconds" << std::endl;
        std::cout << "Read " << n_total << " aggregated points with " << n_dim << " dimensions. " << std::endl;

        auto t1 = std::chrono::steady_clock::now();
        data_process dp(v_coord, m, e, n_dim, n_total, a == 1);
        dp.full_count = f == 1;
        one_rank mpi;
        auto tc = std::chrono::steady_clock::now();
        dp.select_and_process(mpi);
        std::cout << "Classify Points: " << ms_since(tc) << " milliseconds" << std::endl;
        auto tl = std::chrono::steady_clock::now();
        dp.select_cores_and_process(mpi);
        std::cout << "Assign Labels: " << ms_since(tl) << " milliseconds" << std::endl;
        dp.get_result_meta(cores, noise, clusters, n, mpi);
        cluster_index = std::move(dp.v_coord_cluster_index);
        std::cout << "Total Execution Time: " << ms_since(t0) << " milliseconds" << std::endl;
        std::cout << "Total Execution Time (without I/O): " << ms_since(t1) << " milliseconds" << std::endl;
    }

    std::cout << std::endl;
    if (a == 0) std::cout << "Estimated Clusters: " << clusters << std::endl;
    else std::cout << "Upper-bound Approximate Clusters: " << clusters << std::endl;
    std::cout << "Core Points: " << cores << std::endl;
    std::cout << "Noise Points: " << noise << std::endl;

    if (!output_file.empty()) {
        std::cout << "Writing output to " << output_file << std::endl;
        std::ofstream os(output_file);
        if (!os) {
            std::cerr << "Error: cannot write " << output_file << std::endl;
            return EXIT_FAILURE;
        }
        std::string buf;
        buf.reserve(cluster_index.size() * 8);
        char tmp[16];
        for (int c : cluster_index) {
            int len = std::snprintf(tmp, sizeof(tmp), "%d\n", c);
            buf.append(tmp, (size_t)len);
        }
        os << buf;
        os.close();
        std::cout << "Done!" << std::endl;
    }
    return 0;
}
