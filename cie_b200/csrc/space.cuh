// Internal definition of ciecu_space and the BLAS-1 kernels shared by the
// solver kernels.
#pragma once

#include "common.cuh"

#include <atomic>

struct ciecu_space_s {
    cudaStream_t stream = nullptr;
    bool ownsStream = false;
    int device = 0;
    // Scratch of the grid reductions: partial sums (kMaxPartials per slot) and the
    // arrival counter.  Results land in d_result and are copied to h_result (pinned).
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    double* d_result = nullptr;
    double* h_result = nullptr;
};

namespace ciecu {

constexpr int kMaxPartials = 8192;
constexpr int kThreads = 256;

extern std::atomic<long long> g_launches;
inline void count_launch(long long k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// Grid of the deterministic dot kernels: fixed per (n, device).
inline int dot_grid(long n) {
    long blocks = (n + kThreads * 4 - 1) / (kThreads * 4);
    const long cap = static_cast<long>(sm_count()) * 4;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return static_cast<int>(blocks);
}

template <typename T>
int launch_dot(ciecu_space space, long n, const T* a, const T* b, double* d_result);

}  // namespace ciecu
