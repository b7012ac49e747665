// Building blocks of the graph set-up kernels (reordering, sparsity pattern):
// a warp-wide bitonic sort of 64-bit keys held in shared memory, and an
// exclusive prefix sum of int32 counts over the whole grid.
#pragma once

#include "common.cuh"

#include <cstdint>

namespace ciecu {

// Smallest power of two >= n (n >= 1).
__host__ __device__ inline int pow2_at_least(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Sorts keys[0, count) ascending in place; keys[count, P) are set to ~0 first
// (P = pow2_at_least(count) <= capacity).  All 32 lanes of the warp call it.
__device__ inline void warp_bitonic_sort(unsigned long long* keys, int count) {
    const int lane = threadIdx.x & 31;
    const int P = pow2_at_least(count < 1 ? 1 : count);
    for (int i = count + lane; i < P; i += 32) keys[i] = ~0ULL;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = keys[i], b = keys[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            __syncwarp();
        }
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;                            // per thread
constexpr int kScanTile = kScanThreads * kScanItems;     // per block

// Blocks the scan of n items uses in its first pass.
inline long scan_blocks(long n) { return (n + kScanTile - 1) / kScanTile; }

// Work array entries the scan of n items needs: the block sums (b entries, one
// spare) and their scan (b + 1 entries) at every level of the recursion.
inline long scan_work(long n) {
    const long b = scan_blocks(n);
    return b <= 1 ? 1 : 2 * b + 2 + scan_work(b);
}

// out[i] = in[0] + ... + in[i-1] for i <= n (out[n] = the total); `work` holds
// scan_work(n) ints.  Sums must fit in int32 (the callers check).
int exclusive_scan(const int* d_in, int* d_out, long n, int* d_work, cudaStream_t st);

}  // namespace ciecu
