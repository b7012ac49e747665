// Shared helpers of the ciecu library: status codes, the thread-local error
// message behind ciecu_last_error, launch geometry and the fixed-order
// (run-to-run deterministic) warp / block reductions used by every dot product.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <string>
#include <utility>

#include "ciecu.h"

namespace ciecu {

// 148 SMs on B200; grids of streaming kernels are sized as a multiple of this.
constexpr int kFallbackSMs = 148;

void set_error(const std::string& message);
int fail(int status, const std::string& message);
int cuda_fail(cudaError_t error, const char* what);
int sm_count();

// Stream-ordered device memory for solver set-up: a pool per device, owned by the
// library, that keeps freed blocks (up to kPoolKeepBytes) for the next
// allocation instead of returning them to the driver, so that creating and
// destroying solvers of the same size repeatedly maps no new memory.  pool_alloc
// memory is usable on `stream` in stream order (and everywhere once the stream
// has been synchronised).  pool_release waits for the device (the implicit
// synchronisation of cudaFree) and returns the blocks to the pool; it needs no
// live stream, so a solver may be destroyed after its space.
constexpr unsigned long long kPoolKeepBytes = 4ull << 30;
cudaError_t pool_alloc(void** ptr, size_t bytes, cudaStream_t stream);
template <typename T>
cudaError_t pool_alloc(T** ptr, size_t bytes, cudaStream_t stream) {
    return pool_alloc(reinterpret_cast<void**>(ptr), bytes, stream);
}
void pool_release(std::initializer_list<void*> ptrs);

#define CIECU_CUDA(call)                                              \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return ::ciecu::cuda_fail(_e, #call);  \
    } while (0)

#define CIECU_CHECK_LAUNCH(what)                                      \
    do {                                                              \
        cudaError_t _e = cudaGetLastError();                          \
        if (_e != cudaSuccess) return ::ciecu::cuda_fail(_e, what);   \
    } while (0)

#define CIECU_REQUIRE(cond, msg)                                      \
    do {                                                              \
        if (!(cond)) return ::ciecu::fail(CIECU_ERR_ARGUMENT, msg);   \
    } while (0)

#define CIECU_TRY(call)                                               \
    do {                                                              \
        int _s = (call);                                              \
        if (_s != CIECU_OK) return _s;                                \
    } while (0)

// Loads of matrix values and indices: read once per pass over a matrix larger than
// L2, so they are marked evict-first and leave the cache to the gathered vector.
template <typename T>
__device__ __forceinline__ T stream_ld(const T* p) {
    return __ldcs(p);
}

// Nanoseconds of the GPU's global timer: a bound on a wait in wall-clock time,
// independent of the SM clock and of the SM the thread runs on.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- reductions ------------------------------------------------------------

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int offset = 16; offset > 0; offset >>= 1) v += __shfl_xor_sync(0xffffffffu, v, offset);
    return v;
}

// Sum over the block in a fixed order.  Every thread receives the result.
// scratch must hold 32 values; the call contains two __syncthreads().
template <typename T, int THREADS>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T total = lane < WARPS ? scratch[lane] : T(0);
    total = warp_sum(total);
    __syncthreads();
    return total;
}

// The last block to finish a grid-wide reduction (detected with a counter that
// it resets) sums the per-block partials in block order, so the result does not
// depend on which block arrived last.  Returns true in the last block, where
// `out[k]` (k < K) holds the k-th grid-wide sum in every thread.
template <int K, int THREADS>
__device__ __forceinline__ bool grid_reduce_last(const double (&mine)[K], double* partials,
                                                 unsigned* counter, double (&out)[K]) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double sums[K];
#pragma unroll
    for (int k = 0; k < K; ++k) sums[k] = block_sum<double, THREADS>(mine[k], s_red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[k * gridDim.x + blockIdx.x] = sums[k];
        __threadfence();
        const unsigned ticket = atomicAdd(counter, 1u);
        s_last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double acc = 0.0;
        // volatile: partials were written by other blocks during this kernel.
        const volatile double* p = partials + k * gridDim.x;
        for (unsigned b = threadIdx.x; b < gridDim.x; b += THREADS) acc += p[b];
        out[k] = block_sum<double, THREADS>(acc, s_red);
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// out = inScale*out + outScale*sum with the special cases of the reference
// operators (linalg/packages/solvers/src/CSROperator.cpp:78-110), including the
// (-1, -1) combination that yields sum - out.
template <typename T>
__device__ __forceinline__ T combine(T inScale, T old, T outScale, T sum) {
    if (inScale == T(1)) {
        if (outScale == T(1)) return old + sum;
        if (outScale == T(-1)) return old - sum;
        return old + outScale * sum;
    }
    if (inScale == T(0)) {
        if (outScale == T(1)) return sum;
        if (outScale == T(-1)) return -sum;
        return outScale * sum;
    }
    if (inScale == T(-1)) {
        if (outScale == T(1) || outScale == T(-1)) return sum - old;
        return outScale * sum - old;
    }
    if (outScale == T(1)) return inScale * old + sum;
    if (outScale == T(-1)) return inScale * old - sum;
    return inScale * old + outScale * sum;
}

// Largest grid of `kernel` whose blocks are all resident at once (one wave),
// capped by the blocks the work needs; cached per kernel.
int resident_blocks(const void* kernel, int threads, size_t smem);

template <typename K>
inline int fit_grid(K* kernel, int threads, long needBlocks, size_t smem = 0) {
    const long cap = static_cast<long>(resident_blocks(reinterpret_cast<const void*>(kernel), threads, smem));
    long g = needBlocks < cap ? needBlocks : cap;
    return static_cast<int>(g < 1 ? 1 : g);
}

inline int grid_for(long n, int threads, int perSM = 8) {
    long blocks = (n + threads - 1) / threads;
    const long cap = static_cast<long>(sm_count()) * perSM;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return static_cast<int>(blocks);
}

}  // namespace ciecu
