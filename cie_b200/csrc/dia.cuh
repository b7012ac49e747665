// Diagonal (DIA) storage of a CSR matrix whose nonzeros lie on few diagonals:
// the Q1 stiffness matrices of structured grids (9 diagonals in 2D, 27 in 3D,
// lexicographic node order).  Entry (r, c) with c - r = off[d] is stored at
// val[d * ld + r]; entries of a diagonal that are not in the CSR pattern are
// zero.  No column indices are stored, so a row pass reads 8 (FP64) or 4 (FP32)
// bytes per stored entry instead of 12 or 6, and the gathers x[r + off[d]] of
// consecutive rows are consecutive addresses.
//
// Row sums run over the diagonals in ascending offset order, i.e. in the
// column order of the CSR row, one FMA per diagonal.  For finite x a padded zero
// adds nothing, so the sums equal the sequential CSR-order FMA sums of
// CSROperator.cpp:49-56 up to the sign of zero.  When x holds an Inf or NaN at
// a column a padded zero points to, 0 * Inf gives NaN in that row where the CSR
// sum, which never touches that column, stays finite.
//
// The CSR view stays the source of truth: the offsets are found once per CSR
// handle (the pattern is fixed for its lifetime, as the row-block schedule
// already assumes), and solvers refill the values from the CSR arrays.
#pragma once

#include <cstdlib>

#include "spmv.cuh"
#include "sell.cuh"

#include <vector>

namespace ciecu {

constexpr int kMaxDiagonals = 32;

template <typename V>
struct DiaArgs {
    int nrows;
    int ndiag;
    long ld;  // stride between diagonals (rows rounded up to a multiple of 32)
    const V* __restrict__ val;
    int off[kMaxDiagonals];  // ascending
};

// Calls step(d) for every diagonal: fully unrolled when the count ND is known at
// compile time (27 and 9, the 3D and 2D Q1 stencils: every load of a row in
// flight at once), else over the runtime count.
template <int ND, typename V, typename F>
__device__ __forceinline__ void for_diagonals(const DiaArgs<V>& A, F&& step) {
    if constexpr (ND > 0) {
#pragma unroll
        for (int d = 0; d < ND; ++d) step(d);
    } else {
#pragma unroll 9
        for (int d = 0; d < A.ndiag; ++d) step(d);
    }
}

// One thread per row (grid-stride); epilogue interface of the CSR engines.
template <int ND, typename T, typename V, typename Op>
__device__ __forceinline__ void dia_rows(const DiaArgs<V>& A, const T* __restrict__ x, Op& op) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long rl = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; rl < A.nrows; rl += stride) {
        const int r = static_cast<int>(rl);
        const auto pre = op.pre(r);
        T sum = T(0);
        for_diagonals<ND>(A, [&](int d) {
            const int c = r + A.off[d];
            const V v = stream_ld(A.val + static_cast<long>(d) * A.ld + r);
            const T xv = static_cast<unsigned>(c) < static_cast<unsigned>(A.nrows) ? __ldg(x + c) : T(0);
            sum = fma(static_cast<T>(v), xv, sum);
        });
        op.post(r, pre, sum);
    }
}

// Four consecutive rows per thread with 16-byte loads of each diagonal (FP32:
// a warp reads 512 contiguous bytes per diagonal instead of 128).  Rows past
// nrows (up to ld, zero-filled) are computed and dropped; the gathers stay
// inside [0, nrows).  The operand entry of column c is gather(c); the epilogue
// takes the four rows at once (op.pre4(r, pre), op.post4(r, pre, sum)) and skips
// rows past nrows itself.
template <int ND, typename Op, typename TGather>
__device__ __forceinline__ void dia_rows4_gather(const DiaArgs<float>& A, const TGather& gather, Op& op) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x * 4;
    for (long r0 = (static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) * 4; r0 < A.nrows; r0 += stride) {
        const int r = static_cast<int>(r0);
        typename Op::Pre pre[4];
        op.pre4(r, pre);
        float sum[4] = {0.f, 0.f, 0.f, 0.f};
        for_diagonals<ND>(A, [&](int d) {
            const float4 v = __ldcs(reinterpret_cast<const float4*>(A.val + static_cast<long>(d) * A.ld + r));
            const int c = r + A.off[d];
            float xv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
                xv[i] = static_cast<unsigned>(c + i) < static_cast<unsigned>(A.nrows) ? gather(c + i) : 0.f;
            sum[0] = fmaf(v.x, xv[0], sum[0]);
            sum[1] = fmaf(v.y, xv[1], sum[1]);
            sum[2] = fmaf(v.z, xv[2], sum[2]);
            sum[3] = fmaf(v.w, xv[3], sum[3]);
        });
        op.post4(r, pre, sum);
    }
}

// Row-by-row pre/post of an epilogue of the CSR interface, as the four-row
// epilogue (pre4 / post4 for rows r .. r + 3) that the four-row passes call.
template <typename Op>
struct RowsOf4 {
    using Pre = typename Op::Pre;
    Op& op;
    int nrows;
    __device__ __forceinline__ void pre4(int r, Pre (&pre)[4]) const {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (r + i < nrows) pre[i] = op.pre(r + i);
    }
    __device__ __forceinline__ void post4(int r, Pre (&pre)[4], const float (&sum)[4]) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (r + i < nrows) op.post(r + i, pre[i], sum[i]);
    }
};

template <int ND, typename Op>
__device__ __forceinline__ void dia_rows4(const DiaArgs<float>& A, const float* __restrict__ x, Op& op) {
    RowsOf4<Op> rows{op, A.nrows};
    dia_rows4_gather<ND>(A, LoadGather<float>{x}, rows);
}

// dia_rows4 for stencils whose sorted offsets come in consecutive triples
// (o - 1, o, o + 1), the Q1 stencils: for each triple the thread loads the six
// operand entries x[r + o - 1 .. r + o + 4] of its four rows once, where
// dia_rows4 loads twelve.  Triples ascending and the three diagonals of a triple
// in order keep every row sum in the column order of dia_rows4, bit for bit.
template <int ND, typename Op, typename TGather>
__device__ __forceinline__ void dia_rows4_triples_gather(const DiaArgs<float>& A, const TGather& gather, Op& op) {
    constexpr int NT = ND / 3;
    const int nt = NT > 0 ? NT : A.ndiag / 3;
    const long stride = static_cast<long>(gridDim.x) * blockDim.x * 4;
    for (long r0 = (static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) * 4; r0 < A.nrows; r0 += stride) {
        const int r = static_cast<int>(r0);
        typename Op::Pre pre[4];
        op.pre4(r, pre);
        float sum[4] = {0.f, 0.f, 0.f, 0.f};
        auto triple = [&](int t) {
            const int c = r + A.off[3 * t + 1] - 1;
            float xv[6];
#pragma unroll
            for (int j = 0; j < 6; ++j)
                xv[j] = static_cast<unsigned>(c + j) < static_cast<unsigned>(A.nrows) ? gather(c + j) : 0.f;
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const float4 v = __ldcs(reinterpret_cast<const float4*>(A.val + static_cast<long>(3 * t + e) * A.ld + r));
                sum[0] = fmaf(v.x, xv[e], sum[0]);
                sum[1] = fmaf(v.y, xv[e + 1], sum[1]);
                sum[2] = fmaf(v.z, xv[e + 2], sum[2]);
                sum[3] = fmaf(v.w, xv[e + 3], sum[3]);
            }
        };
        if constexpr (NT > 0) {
#pragma unroll
            for (int t = 0; t < NT; ++t) triple(t);
        } else {
            for (int t = 0; t < nt; ++t) triple(t);
        }
        op.post4(r, pre, sum);
    }
}

// dia_rows4_triples_gather for an operand that is costly to gather (formed from
// several vectors): per triple a lane needs the six operand entries starting at
// column c = r + o - 1, i.e. offsets s .. s + 5 (s = c mod 4, the same in every
// lane) of the three aligned 4-column blocks b, b + 1, b + 2 with 4b = c - s.
// Block b + 1 of lane l is block b of lane l + 1, and block b + 2 that of lane
// l + 2, so each lane forms ONE block (gather.block(b): the four operand values
// of columns 4b .. 4b + 3 from 16-byte loads) and takes the others from its
// neighbours by warp shuffles; the last lanes of the warp form theirs directly.
// A warp takes this path when all of its 32 lanes hold rows (R + 128 <= nrows)
// and every block it touches lies inside [0, nrows); otherwise it gathers entry
// by entry through gather(c) as dia_rows4_triples_gather does.  Values and sums
// are the same either way.  blockDim.x must be a multiple of 32.
template <int ND, typename Op, typename TGather>
__device__ __forceinline__ void dia_rows4_triples_window(const DiaArgs<float>& A, const TGather& gather, Op& op) {
    constexpr int NT = ND / 3;
    const int nt = NT > 0 ? NT : A.ndiag / 3;
    const int lane = threadIdx.x & 31;
    const long stride = static_cast<long>(gridDim.x) * blockDim.x * 4;
    const long warpBase = (static_cast<long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31)) * 4;
    for (long R = warpBase; R < A.nrows; R += stride) {
        const bool fullWarp = R + 128 <= A.nrows;  // the same in every lane
        const int r = static_cast<int>(R) + 4 * lane;
        if (!fullWarp && r >= A.nrows) continue;  // this warp takes the entry-by-entry path only
        typename Op::Pre pre[4];
        op.pre4(r, pre);
        float sum[4] = {0.f, 0.f, 0.f, 0.f};
        auto triple = [&](int t) {
            const int o = A.off[3 * t + 1];
            const int s = (o - 1) & 3;
            const long first = R + o - 1 - s;  // first column of lane 0's blocks
            float xv[6];
            if (fullWarp && first >= 0 && first + 4 * 31 + 11 < A.nrows) {
                const int b = static_cast<int>((r + o - 1 - s) >> 2);
                const float4 p0 = gather.block(b);
                float4 p1;
                p1.x = __shfl_down_sync(0xffffffffu, p0.x, 1);
                p1.y = __shfl_down_sync(0xffffffffu, p0.y, 1);
                p1.z = __shfl_down_sync(0xffffffffu, p0.z, 1);
                p1.w = __shfl_down_sync(0xffffffffu, p0.w, 1);
                if (lane == 31) p1 = gather.block(b + 1);
                if (s == 3) {
                    float p2 = __shfl_down_sync(0xffffffffu, p0.x, 2);
                    const float from31 = __shfl_down_sync(0xffffffffu, p1.x, 1);
                    if (lane == 30) p2 = from31;
                    if (lane == 31) p2 = gather.block(b + 2).x;
                    xv[0] = p0.w; xv[1] = p1.x; xv[2] = p1.y; xv[3] = p1.z; xv[4] = p1.w; xv[5] = p2;
                } else if (s == 2) {
                    xv[0] = p0.z; xv[1] = p0.w; xv[2] = p1.x; xv[3] = p1.y; xv[4] = p1.z; xv[5] = p1.w;
                } else if (s == 1) {
                    xv[0] = p0.y; xv[1] = p0.z; xv[2] = p0.w; xv[3] = p1.x; xv[4] = p1.y; xv[5] = p1.z;
                } else {
                    xv[0] = p0.x; xv[1] = p0.y; xv[2] = p0.z; xv[3] = p0.w; xv[4] = p1.x; xv[5] = p1.y;
                }
            } else {
                const int c = r + o - 1;
#pragma unroll
                for (int j = 0; j < 6; ++j)
                    xv[j] = static_cast<unsigned>(c + j) < static_cast<unsigned>(A.nrows) ? gather(c + j) : 0.f;
            }
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const float4 v = __ldcs(reinterpret_cast<const float4*>(A.val + static_cast<long>(3 * t + e) * A.ld + r));
                sum[0] = fmaf(v.x, xv[e], sum[0]);
                sum[1] = fmaf(v.y, xv[e + 1], sum[1]);
                sum[2] = fmaf(v.z, xv[e + 2], sum[2]);
                sum[3] = fmaf(v.w, xv[e + 3], sum[3]);
            }
        };
        if constexpr (NT > 0) {
#pragma unroll
            for (int t = 0; t < NT; ++t) triple(t);
        } else {
            for (int t = 0; t < nt; ++t) triple(t);
        }
        op.post4(r, pre, sum);
    }
}

template <int ND, typename Op>
__device__ __forceinline__ void dia_rows4_triples(const DiaArgs<float>& A, const float* __restrict__ x, Op& op) {
    RowsOf4<Op> rows{op, A.nrows};
    dia_rows4_triples_gather<ND>(A, LoadGather<float>{x}, rows);
}

// CIECU_DIA_TRIPLES=0 keeps the plain four-row pass for triple stencils (for
// comparison).
inline bool dia_triples_enabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("CIECU_DIA_TRIPLES");
        return !(v && v[0] == '0');
    }();
    return enabled;
}

// Whether the sorted offsets come in consecutive triples (o - 1, o, o + 1).
template <typename V>
bool dia_has_triples(const DiaArgs<V>& d) {
    if (d.ndiag == 0 || d.ndiag % 3 != 0) return false;
    for (int t = 0; t < d.ndiag / 3; ++t)
        if (d.off[3 * t] + 1 != d.off[3 * t + 1] || d.off[3 * t + 1] + 1 != d.off[3 * t + 2]) return false;
    return true;
}

// Calls f(std::integral_constant<int, ND>) with ND = 27, 9 or 0 (runtime count).
template <typename F>
int with_diagonals(int ndiag, F&& f) {
    switch (ndiag) {
        case 27: return f(std::integral_constant<int, 27>{});
        case 9: return f(std::integral_constant<int, 9>{});
        default: return f(std::integral_constant<int, 0>{});
    }
}

// Distinct diagonal offsets of a square CSR matrix, ascending, cached in the
// handle.  Empty when there are more than kMaxDiagonals or when DIA storage would
// hold less than 60 % nonzeros.
int dia_offsets(ciecu_csr_s* csr, const std::vector<int>** out);

// Diagonal stride for n rows.
inline long dia_ld(long n) { return ((n + 31) / 32) * 32; }

// Shape of the DIA copy of csr (values pointer left null).
template <typename V>
DiaArgs<V> dia_shape(const ciecu_csr_s* csr, const std::vector<int>& offsets) {
    DiaArgs<V> a{};
    a.nrows = csr->rows;
    a.ndiag = static_cast<int>(offsets.size());
    a.ld = dia_ld(csr->rows);
    a.val = nullptr;
    for (int d = 0; d < a.ndiag; ++d) a.off[d] = offsets[static_cast<size_t>(d)];
    return a;
}

// Writes the CSR values of csr into the DIA array `out` of shape `a` (entries of
// the pattern only; the caller zero-fills `out` once).  With sdiag, entry (r, c)
// is scaled by sdiag[r] * sdiag[c] (the symmetric Jacobi scaling of the mixed
// solver's inner matrix) before the conversion to V.
int dia_fill_f64(const ciecu_csr_s* csr, const DiaArgs<double>& a, double* out, cudaStream_t st);
int dia_fill_f32(const ciecu_csr_s* csr, const DiaArgs<float>& a, float* out, const double* sdiag, cudaStream_t st);

// CIECU_DIA_SYMMETRIC=0 makes the FP64 PCG read every diagonal of a bitwise
// symmetric DIA copy (for comparison); by default it reads only the upper half.
inline bool dia_symmetric_enabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("CIECU_DIA_SYMMETRIC");
        return !(v && v[0] == '0');
    }();
    return enabled;
}

// Whether the DIA copy `full` (offsets symmetric about 0) is bitwise symmetric:
// entry (r, r + o) equals entry (r + o, r) for every stored pair.
template <typename V>
int dia_symmetric(const DiaArgs<V>& full, cudaStream_t st, unsigned* d_flag, bool* symmetric);

// The upper half of a full copy with offsets symmetric about 0, as a view into
// it: the ndiag / 2 + 1 diagonals from the main one on are contiguous there.
template <typename V>
DiaArgs<V> dia_upper_view(const DiaArgs<V>& full) {
    DiaArgs<V> u{};
    u.nrows = full.nrows;
    u.ld = full.ld;
    u.ndiag = full.ndiag / 2 + 1;
    for (int d = 0; d < u.ndiag; ++d) u.off[d] = full.off[full.ndiag / 2 + d];
    u.val = full.val + static_cast<long>(full.ndiag / 2) * full.ld;
    return u;
}

// One thread per row over the upper half U of a bitwise symmetric matrix
// (diagonal d of U holds A[r][r + off[d]], off[0] = 0, ascending): the lower term
// A[r][r - off[d]] = A[r - off[d]][r] is read back from diagonal d at row
// r - off[d], data streamed about off[d] rows earlier (an L2 hit), so only the
// upper half crosses HBM.  Lower terms from the farthest diagonal in, the main
// diagonal, the upper ones: the column order of dia_rows on the full copy, so the
// row sums are the same.
template <int NU, typename T, typename V, typename Op>
__device__ __forceinline__ void dia_rows_sym(const DiaArgs<V>& U, const T* __restrict__ x, Op& op) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    const int nu = NU > 0 ? NU : U.ndiag;
    for (long rl = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; rl < U.nrows; rl += stride) {
        const int r = static_cast<int>(rl);
        const auto pre = op.pre(r);
        T sum = T(0);
#pragma unroll 7
        for (int d = nu - 1; d >= 1; --d) {
            const int c = r - U.off[d];
            const bool in = c >= 0;
            const V v = in ? __ldg(U.val + static_cast<long>(d) * U.ld + c) : V(0);
            const T xv = in ? __ldg(x + c) : T(0);
            sum = fma(static_cast<T>(v), xv, sum);
        }
        for_diagonals<NU>(U, [&](int d) {
            const int c = r + U.off[d];
            const V v = stream_ld(U.val + static_cast<long>(d) * U.ld + r);
            const T xv = static_cast<unsigned>(c) < static_cast<unsigned>(U.nrows) ? __ldg(x + c) : T(0);
            sum = fma(static_cast<T>(v), xv, sum);
        });
        op.post(r, pre, sum);
    }
}

}  // namespace ciecu
