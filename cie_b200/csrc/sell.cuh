// SELL-32: sliced ELLPACK with slices of 32 consecutive rows, one thread per row.
// Entry j of row r lives at sliceStart[r / 32] + 32 j + r % 32, so the 32 lanes of
// a warp read 32 consecutive values (and column indices) with one fully coalesced
// load per entry position -- no row pointers, no shuffles.  Each slice is padded
// to its longest row; sliceLen < 0 marks a slice whose rows differ in length, and
// only there is the per-row length read, so padding entries are never touched.
// Built on the device from a CSR matrix (mixed.cu); the inner operator of the
// mixed-precision solver.
#pragma once

#include "common.cuh"

namespace ciecu {

template <typename V, typename CI>
struct SellArgs {
    int nrows;
    const int* __restrict__ sliceLen;               // padded length, negative: ragged slice
    const long long* __restrict__ sliceStart;       // first entry of each slice
    const unsigned short* __restrict__ rowLen;      // per-row length (ragged slices only)
    const V* __restrict__ val;
    const CI* __restrict__ col;                      // int: absolute column, short: offset from the row
};

template <typename CI>
__device__ __forceinline__ int sell_col(const CI* p, int row);
template <>
__device__ __forceinline__ int sell_col<int>(const int* p, int) {
    return __ldg(p);
}
template <>
__device__ __forceinline__ int sell_col<short>(const short* p, int row) {
    return row + __ldg(p);
}

// Row sums with the pre/post epilogue interface of spmv.cuh.  The grid-stride loop
// moves whole warps (blockDim and the grid are multiples of 32), so a warp always
// covers 32 consecutive rows of one slice.
template <int U, typename T, typename V, typename CI, typename Op>
__device__ __forceinline__ void sell_rows(const SellArgs<V, CI>& A, const T* __restrict__ x, Op& op) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long rl = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; rl < A.nrows; rl += stride) {
        const int r = static_cast<int>(rl);
        const auto pre = op.pre(r);
        const int s = r >> 5;
        int len = __ldg(A.sliceLen + s);
        if (len < 0) len = __ldg(A.rowLen + r);
        const long long base = __ldg(A.sliceStart + s) + (r & 31);
        T sum = T(0);
        for (int j = 0; j < len; j += U) {
            V v[U];
            int c[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool in = j + u < len;
                const long long idx = base + 32LL * (j + u);
                v[u] = in ? __ldg(A.val + idx) : V(0);
                c[u] = in ? sell_col<CI>(A.col + idx, r) : -1;
            }
            T xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : T(0);
#pragma unroll
            for (int u = 0; u < U; ++u) sum = fma(static_cast<T>(v[u]), xv[u], sum);
        }
        op.post(r, pre, sum);
    }
}

}  // namespace ciecu
