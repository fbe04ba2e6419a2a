// ndb_b200_data_process.h -- header-only C++ drop-in for nextdbscan-exa's class
// data_process (data_process.h:45-102), implemented on the C ABI of
// libndb_b200.so (ndb_b200.h).
//
// Same constructor arguments, same phase methods, same public result vectors,
// so nextdbscan::start (nextdbscan.cpp:46-58) and main.cpp compile unchanged when
// the reference's data_process.h includes this header in place of its own class.  The
// methods are noexcept like the reference's; a failing status is printed to
// std::cerr and ends the process with EXIT_FAILURE, which is how the reference
// treats hard errors (magma_input.h:158-159, data_process.cpp:38-41).
//
// The magmaMPI argument of the phase methods is a template parameter: one GPU is
// one rank here, so it is only accepted, never used.
#ifndef NDB_B200_DATA_PROCESS_H
#define NDB_B200_DATA_PROCESS_H

#include <climits>
#include <cstdlib>
#include <iostream>
#include <utility>
#include <vector>

#include "ndb_b200.h"

#ifndef NDB_B200_NO_CLUSTER_DEFINED
#define NDB_B200_NO_CLUSTER_DEFINED
static const int NO_CLUSTER = INT32_MAX;  // data_process.h:26
#endif

class data_process {
private:
    int const m, n_dim;
    std::size_t const n_coord;
    std::size_t const n_total_coord;
    float const e, e2;
    bool const is_approximate;
    ndb_ctx *ctx = nullptr;
    ndb_result res{};

    static void fail(ndb_status s, const char *where, ndb_ctx *c) noexcept {
        std::cerr << "nextdbscan-b200: " << where << ": " << ndb_b200_strerror(s);
        if (c && *ndb_b200_last_cuda_error(c)) std::cerr << " (" << ndb_b200_last_cuda_error(c) << ")";
        std::cerr << std::endl;
        std::exit(EXIT_FAILURE);
    }

public:
    unsigned long long allocated_bytes;
    std::vector<float> v_coord;
    std::vector<int> v_coord_id;
    std::vector<int> v_coord_nn;
    std::vector<int> v_coord_cluster_index;
    std::vector<int> v_cluster_label;
    // exact per-point counts like the reference (false: counts stop at m, labels unchanged)
    bool full_count = true;

    explicit data_process(std::vector<float> &v_coord, int const m, float const e, int const n_dim,
                          int const n_total_coord, bool const is_approximate, int const device = 0)
        : m(m), n_dim(n_dim), n_coord(n_dim > 0 ? v_coord.size() / n_dim : 0), n_total_coord(n_total_coord),
          e(e), e2(e * e), is_approximate(is_approximate), v_coord(std::move(v_coord)) {
        allocated_bytes = n_coord * n_dim * sizeof(float);
        ndb_status s = ndb_b200_create(&ctx, device);
        if (s != NDB_OK) fail(s, "ndb_b200_create", nullptr);
    }

    data_process(const data_process &) = delete;
    data_process &operator=(const data_process &) = delete;

    ~data_process() { ndb_b200_destroy(ctx); }

    // data_process.cpp:334-392
    template <class MPI>
    void select_and_process(MPI const &) noexcept {
        v_coord_id.resize(n_coord);
        for (std::size_t i = 0; i < n_coord; ++i) v_coord_id[i] = (int)i;
        v_coord_nn.assign(n_coord, 0);
        uint32_t flags = (full_count ? NDB_FLAG_FULL_COUNT : 0u) | (is_approximate ? NDB_FLAG_APPROXIMATE : 0u);
        ndb_status s = ndb_b200_classify(ctx, v_coord.data(), (int64_t)n_coord, n_dim, e, m, flags,
                                         v_coord_nn.data());
        if (s != NDB_OK) fail(s, "select_and_process", ctx);
        allocated_bytes += n_coord * 2 * sizeof(int);
    }

    // data_process.cpp:268-332
    template <class MPI>
    void select_cores_and_process(MPI const &) noexcept {
        v_coord_cluster_index.assign(n_coord, NO_CLUSTER);
        ndb_status s = ndb_b200_assign_labels(ctx, v_coord_cluster_index.data(), &res);
        if (s != NDB_OK) fail(s, "select_cores_and_process", ctx);
        v_cluster_label.assign((std::size_t)res.core_count, 0);
        s = ndb_b200_cluster_label(ctx, v_cluster_label.data(), res.core_count);
        if (s != NDB_OK) fail(s, "select_cores_and_process", ctx);
        allocated_bytes += n_coord * sizeof(int) + v_cluster_label.size() * sizeof(int);
    }

    // data_process.cpp:50-91
    template <class MPI>
    void get_result_meta(int &cores, int &noise, int &clusters, int &n, MPI const &) noexcept {
        cores = res.core_count;
        noise = res.noise;
        clusters = res.clusters;
        n = (int)n_coord;
    }

    ndb_stats stats() const noexcept {
        ndb_stats st{};
        ndb_b200_get_stats(ctx, &st);
        return st;
    }
};

#endif  // NDB_B200_DATA_PROCESS_H
