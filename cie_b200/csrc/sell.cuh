// SELL-32x4: sliced ELLPACK with slices of 32 consecutive rows, one thread per
// row, entries interleaved in groups of four.  Entry j of row r lives at
//     sliceStart[r / 32] + 128 * (j / 4) + 4 * (r % 32) + j % 4,
// so a lane reads four values with one 16-byte load (four 16-bit column offsets
// with one 8-byte load) and the 32 lanes of a warp read 512 contiguous bytes --
// no row pointers, no shuffles, four entries per load instruction.  Each slice
// is padded to its longest row (rounded up to a group); sliceLen < 0 marks a
// slice whose rows differ in length, and only there is the per-row length read.
// Entries past a row's length are masked, never gathered.  Built on the device
// from a CSR matrix (mixed.cu); the inner operator of the mixed-precision solver.
#pragma once

#include "common.cuh"

namespace ciecu {

template <typename V, typename CI>
struct SellArgs {
    int nrows;
    const int* __restrict__ sliceLen;               // longest row of the slice, negative: ragged slice
    const long long* __restrict__ sliceStart;       // first entry of each slice
    const unsigned short* __restrict__ rowLen;      // per-row length (ragged slices only)
    const V* __restrict__ val;
    const CI* __restrict__ col;                      // int: absolute column, short: offset from the row
};

template <typename V>
struct Group4;
template <>
struct Group4<float> {
    static __device__ __forceinline__ void load(const float* p, float (&v)[4]) {
        const float4 a = stream_ld(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
};
template <>
struct Group4<double> {
    static __device__ __forceinline__ void load(const double* p, double (&v)[4]) {
        const double2 a = stream_ld(reinterpret_cast<const double2*>(p));
        const double2 b = stream_ld(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
};

template <typename CI>
struct GroupCols;
template <>
struct GroupCols<short> {
    static __device__ __forceinline__ void load(const short* p, int row, int (&c)[4]) {
        const uint2 a = stream_ld(reinterpret_cast<const uint2*>(p));
        c[0] = row + static_cast<short>(a.x & 0xffffu);
        c[1] = row + static_cast<short>(a.x >> 16);
        c[2] = row + static_cast<short>(a.y & 0xffffu);
        c[3] = row + static_cast<short>(a.y >> 16);
    }
};
template <>
struct GroupCols<int> {
    static __device__ __forceinline__ void load(const int* p, int, int (&c)[4]) {
        const int4 a = stream_ld(reinterpret_cast<const int4*>(p));
        c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
    }
};

// x[c] read through the read-only path: the operand of a plain SpMV.
template <typename T>
struct LoadGather {
    const T* __restrict__ x;
    __device__ __forceinline__ T operator()(int c) const { return __ldg(x + c); }
};

// Row sums with the pre/post epilogue interface of spmv.cuh, the operand entry of
// column c given by gather(c).  The grid-stride loop moves whole warps (blockDim
// and the grid are multiples of 32), so a warp always covers 32 consecutive rows
// of one slice.  U groups (4U entries) per lane are in flight before the FMA chain.
template <int U, typename T, typename V, typename CI, typename Op, typename TGather>
__device__ __forceinline__ void sell_rows_gather(const SellArgs<V, CI>& A, const TGather& gather, Op& op) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long rl = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; rl < A.nrows; rl += stride) {
        const int r = static_cast<int>(rl);
        const auto pre = op.pre(r);
        const int s = r >> 5;
        int len = __ldg(A.sliceLen + s);
        if (len < 0) len = __ldg(A.rowLen + r);
        const long long base = __ldg(A.sliceStart + s) + 4 * (r & 31);
        const int groups = (len + 3) >> 2;
        T sum = T(0);
        for (int g = 0; g < groups; g += U) {
            V v[U][4];
            int c[U][4];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (g + u < groups) {
                    const long long idx = base + 128LL * (g + u);
                    Group4<V>::load(A.val + idx, v[u]);
                    GroupCols<CI>::load(A.col + idx, r, c[u]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        v[u][e] = V(0);
                        c[u][e] = 0;
                    }
                }
            }
            T xv[U][4];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < 4; ++e) xv[u][e] = 4 * (g + u) + e < len ? gather(c[u][e]) : T(0);
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < 4; ++e) sum = fma(static_cast<T>(v[u][e]), xv[u][e], sum);
        }
        op.post(r, pre, sum);
    }
}

template <int U, typename T, typename V, typename CI, typename Op>
__device__ __forceinline__ void sell_rows(const SellArgs<V, CI>& A, const T* __restrict__ x, Op& op) {
    sell_rows_gather<U, T, V, CI>(A, LoadGather<T>{x}, op);
}

}  // namespace ciecu
