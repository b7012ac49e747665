// CSR SpMV device engine shared by the operator kernels and the fused solver
// kernels.  Two schedules:
//
//  * vector_rows<VS>: VS lanes per row (VS = 2..32; the sub-group-per-row scheme
//    of SYCLCSROperator.cpp:55-86).  Lane j of a row handles entries j, j + VS,
//    ...; a warp load instruction covers VS consecutive entries of each of its
//    32/VS rows, each lane keeps UNROLL loads in flight, and the lanes of a row
//    reduce with shuffles.
//  * stream_rows: rows are grouped host-side into row blocks of at most TILE
//    entries.  A CTA stages its block's column indices, values and the gathered
//    x[col] into shared memory, then one thread per row accumulates the row in
//    CSR order with FMA -- the summation order of CSROperator.cpp:49-56, so row
//    sums match the reference's FMA-contracted build bit for bit.  Rows longer
//    than TILE form single-row blocks that the whole CTA reduces cooperatively.
//
// Epilogues are structs with pre(row) -> Pre and post(row, Pre, sum): pre() is
// issued before the row's loads so that operands the epilogue needs (p[r],
// b[r], D^-1[r], ...) are in flight with them instead of adding a dependent
// memory latency after the reduction; post() runs exactly once per row, so fused
// epilogues (scaled update, solver dot products) need no second pass.
//
// Column indices: CI = int (absolute) or short (offset from the row, the 16-bit
// encoding of the mixed-precision inner matrix).
#pragma once

#include "common.cuh"

#include <cstdint>
#include <type_traits>
#include <vector>

struct ciecu_csr_s;

namespace ciecu {

constexpr int kStreamThreads = 256;
constexpr int kStreamTile = 2048;       // entries per row block
constexpr int kStreamMaxRows = 1024;    // rows per row block
constexpr int kVectorThreads = 256;

template <typename V, typename CI = int>
struct CsrArgs {
    const int* __restrict__ rowptr;
    const CI* __restrict__ col;
    const V* __restrict__ val;
    int nrows;
    long nnz;
    const int* __restrict__ blocks;  // row-block boundaries (nblocks + 1)
    int nblocks;
    const uint16_t* __restrict__ mask;  // optional (masked operator)
    uint16_t threshold;
    bool aligned16;  // col and val base pointers are 16-byte aligned
};

struct NoPre {};

template <typename V>
struct Vec4;
template <>
struct Vec4<double> {
    static __device__ __forceinline__ void load(const double* p, double (&v)[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};
template <>
struct Vec4<float> {
    static __device__ __forceinline__ void load(const float* p, float (&v)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
};

template <typename CI>
struct Col4;
template <>
struct Col4<int> {
    static __device__ __forceinline__ void load(const int* p, int row, int (&c)[4]) {
        const int4 a = __ldg(reinterpret_cast<const int4*>(p));
        c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
        (void)row;
    }
    static __device__ __forceinline__ int one(const int* p, int row) {
        (void)row;
        return stream_ld(p);
    }
};
template <>
struct Col4<short> {
    static __device__ __forceinline__ void load(const short* p, int row, int (&c)[4]) {
        const uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
        c[0] = row + static_cast<short>(a.x & 0xffffu);
        c[1] = row + static_cast<short>(a.x >> 16);
        c[2] = row + static_cast<short>(a.y & 0xffffu);
        c[3] = row + static_cast<short>(a.y >> 16);
    }
    static __device__ __forceinline__ int one(const short* p, int row) { return row + stream_ld(p); }
};

template <bool MASKED, typename T, typename V, typename CI>
__device__ __forceinline__ T gather(const CsrArgs<V, CI>& A, const T* __restrict__ x, int c) {
    if constexpr (MASKED) {
        return A.mask[c] < A.threshold ? __ldg(x + c) : T(0);
    } else {
        return __ldg(x + c);
    }
}

// Stages entries [e0, e1) of the row block: s_val[k] = val[e0+k], s_x[k] = x[col[e0+k]].
template <typename T, typename V, int THREADS, bool MASKED>
__device__ __forceinline__ void stage_block(const CsrArgs<V, int>& A, const T* __restrict__ x, int e0, int e1,
                                            V* s_val, T* s_x) {
    const int tid = threadIdx.x;
    if (A.aligned16) {
        int a0 = (e0 + 3) & ~3;
        if (a0 > e1) a0 = e1;
        const int groups = (e1 - a0) >> 2;
        const int a1 = a0 + (groups << 2);
        // head and tail: at most 3 entries each
        if (tid < a0 - e0) {
            const int k = e0 + tid;
            s_val[tid] = A.val[k];
            s_x[tid] = gather<MASKED>(A, x, A.col[k]);
        }
        if (tid < e1 - a1) {
            const int k = a1 + tid;
            s_val[k - e0] = A.val[k];
            s_x[k - e0] = gather<MASKED>(A, x, A.col[k]);
        }
        const int base = a0 - e0;
#pragma unroll 2
        for (int g = tid; g < groups; g += THREADS) {
            int c[4];
            Col4<int>::load(A.col + a0 + 4 * g, 0, c);
            V v[4];
            Vec4<V>::load(A.val + a0 + 4 * g, v);
            const int k = base + 4 * g;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                s_x[k + u] = gather<MASKED>(A, x, c[u]);
                s_val[k + u] = v[u];
            }
        }
    } else {
        for (int k = e0 + tid; k < e1; k += THREADS) {
            s_val[k - e0] = A.val[k];
            s_x[k - e0] = gather<MASKED>(A, x, A.col[k]);
        }
    }
}

// Row sums of every row block assigned to this CTA (persistent loop over blocks).
template <typename T, typename V, int THREADS, int TILE, bool MASKED, typename Op>
__device__ __forceinline__ void stream_rows(const CsrArgs<V, int>& A, const T* __restrict__ x, Op& op) {
    __shared__ __align__(16) V s_val[TILE];
    __shared__ __align__(16) T s_x[TILE];
    __shared__ T s_red[32];
    for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
        const int r0 = A.blocks[b], r1 = A.blocks[b + 1];
        const int e0 = A.rowptr[r0], e1 = A.rowptr[r1];
        if (e1 - e0 <= TILE) {
            stage_block<T, V, THREADS, MASKED>(A, x, e0, e1, s_val, s_x);
            __syncthreads();
            for (int r = r0 + threadIdx.x; r < r1; r += THREADS) {
                const auto pre = op.pre(r);
                const int k0 = A.rowptr[r] - e0, k1 = A.rowptr[r + 1] - e0;
                T sum = T(0);
                if (!MASKED || A.mask[r] < A.threshold)
                    for (int k = k0; k < k1; ++k) sum = fma(static_cast<T>(s_val[k]), s_x[k], sum);
                op.post(r, pre, sum);
            }
            __syncthreads();
        } else {
            // one long row: the whole CTA reduces it (fixed order)
            const auto pre = op.pre(r0);
            T sum = T(0);
            const bool active = !MASKED || A.mask[r0] < A.threshold;
            if (active)
                for (int k = e0 + threadIdx.x; k < e1; k += THREADS)
                    sum = fma(static_cast<T>(A.val[k]), gather<MASKED>(A, x, A.col[k]), sum);
            sum = block_sum<T, THREADS>(sum, s_red);
            if (threadIdx.x == 0) op.post(r0, pre, sum);
            __syncthreads();
        }
    }
}

// VS lanes per row.  Loop bounds are uniform per warp so the shuffles always see
// all 32 lanes.  Each lane issues the loads of UNROLL strided entries (a warp
// instruction covers VS consecutive entries of 32/VS rows) before the FMA chain.
template <typename T, typename V, typename CI, int VS, int THREADS, bool MASKED, typename Op>
__device__ __forceinline__ void vector_rows(const CsrArgs<V, CI>& A, const T* __restrict__ x, Op& op) {
    constexpr int ROWS_PER_WARP = 32 / VS;
    constexpr int UNROLL = VS <= 4 ? 8 : 4;
    const int lane = threadIdx.x & 31;
    const int sub = lane % VS;
    const long warpGlobal = (static_cast<long>(blockIdx.x) * THREADS + threadIdx.x) >> 5;
    const long warps = (static_cast<long>(gridDim.x) * THREADS) >> 5;
    const long rowGroups = (A.nrows + ROWS_PER_WARP - 1) / ROWS_PER_WARP;
    for (long g = warpGlobal; g < rowGroups; g += warps) {
        const long rowL = g * ROWS_PER_WARP + lane / VS;
        const bool valid = rowL < A.nrows;
        const int r = valid ? static_cast<int>(rowL) : 0;
        typename Op::Pre pre{};
        if (valid && sub == 0) pre = op.pre(r);
        T sum = T(0);
        if (valid && (!MASKED || A.mask[r] < A.threshold)) {
            const int k1 = A.rowptr[r + 1];
            for (int k = A.rowptr[r] + sub; k < k1; k += UNROLL * VS) {
                V v[UNROLL];
                int c[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) {
                    const int kk = k + u * VS;
                    const bool in = kk < k1;
                    v[u] = in ? stream_ld(A.val + kk) : V(0);
                    c[u] = in ? Col4<CI>::one(A.col + kk, r) : -1;
                }
                T xv[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) xv[u] = c[u] >= 0 ? gather<MASKED>(A, x, c[u]) : T(0);
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) sum = fma(static_cast<T>(v[u]), xv[u], sum);
            }
        }
#pragma unroll
        for (int offset = VS / 2; offset > 0; offset >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, offset, VS);
        if (valid && sub == 0) op.post(r, pre, sum);
    }
}

// Row pass with the schedule fixed at compile time: KERNEL = 1 (stream) or VS.
template <int KERNEL, typename T, typename V, bool MASKED, typename CI = int, typename Op>
__device__ __forceinline__ void csr_rows(const CsrArgs<V, CI>& A, const T* __restrict__ x, Op& op) {
    if constexpr (KERNEL == 1) {
        static_assert(std::is_same<CI, int>::value, "the stream schedule reads int32 columns");
        stream_rows<T, V, kStreamThreads, kStreamTile, MASKED>(A, x, op);
    } else {
        vector_rows<T, V, CI, KERNEL, kVectorThreads, MASKED>(A, x, op);
    }
}

template <int KERNEL>
constexpr int csr_threads() {
    return KERNEL == 1 ? kStreamThreads : kVectorThreads;
}

// Calls f(std::integral_constant<int, KERNEL>) for the runtime schedule id.
template <typename F>
int with_schedule(int kernel, F&& f) {
    switch (kernel) {
        case 2: return f(std::integral_constant<int, 2>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        default: return f(std::integral_constant<int, 1>{});
    }
}

}  // namespace ciecu

struct ciecu_csr_s {
    ciecu_space space = nullptr;
    int rows = 0, cols = 0;
    long nnz = 0;
    const int* rowptr = nullptr;
    const int* col = nullptr;
    const void* val = nullptr;
    int valueType = CIECU_F64;
    int kernel = 0;  // 0 = not yet tuned
    bool aligned16 = false;
    int* d_blocks = nullptr;
    int nblocks = 0;
    int maxRow = 0;
    double avgRow = 0.0;
    int diaState = 0;             // 0 not analysed, 1 DIA offsets found, 2 not a few-diagonal matrix
    std::vector<int> diaOffsets;  // ascending diagonal offsets (dia.cuh)

    template <typename V>
    ciecu::CsrArgs<V> args(const uint16_t* mask = nullptr, uint16_t threshold = 0) const {
        return ciecu::CsrArgs<V>{rowptr, col, static_cast<const V*>(val), rows, nnz, d_blocks, nblocks,
                                 mask, threshold, aligned16};
    }
};

namespace ciecu {
// Grid of a CSR row pass for the matrix's chosen schedule (persistent).
int csr_grid(const ciecu_csr_s* csr, int kernel);
int ensure_tuned(ciecu_csr_s* csr);
}  // namespace ciecu
