// Multi-right-hand-side Jacobi-PCG (SpMM-CG): k <= 32 independent conjugate-
// gradient solves against ONE matrix, each following ConjugateGradients_impl.hpp:
// 49-201 with its own alpha, beta and stopping test, while every iteration reads
// the matrix once for all k.  No reference counterpart as one object (the
// reference would run k solver objects, one per right-hand side).
//
// Vectors are row-major n x k blocks (entry (i, c) at i*k + c).  A CTA stages a
// row block's (value, column) pairs in shared memory; a group of KP lanes (KP =
// the power of two >= k) owns a row, reads each pair as a shared-memory
// broadcast, and lane c gathers P[j][c] -- k consecutive doubles, one coalesced
// access per matrix entry for the group.  Each row sum runs over the entries in
// CSR order.
// Dot products are per column, reduced in a fixed order (per-block column sums,
// then the last block sums the blocks in block order).
//
// One iteration = three kernels (K1 SpMM + p_c^T q_c, K2 update + dots +
// decision, K3 direction) in the device-side graph loop of the other solvers;
// a column that has converged is left unchanged by K2/K3.
#include "dia.cuh"
#include "graph.cuh"
#include "pcg.cuh"
#include "ciecu_multi.h"

#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <type_traits>
#include <string>
#include <vector>

namespace ciecu {
namespace {

constexpr int kT = 256;
constexpr int kWarps = kT / 32;

struct ColumnScalars {
    double rz, pq, alpha, beta, rr, r0, absres, relres;
    long long iter;
    int done;       // 0 running, 1 converged, 2 iteration limit, 3 breakdown
    int errorKind;  // 1: r^T z <= 0 at start, 2: p^T A p <= 0
    long long errorIter;
    // FP32-refined form: reliable-update state of the column
    double maxrx, maxrr;  // largest FP32 residual norm since the last x / r replacement
    double rzPending;     // r^T z of the FP32 recursion when a replacement is due
    long long refinements;
    int pending;  // a replacement is due at the end of this iteration
    int updateX;  // ... and it folds the FP32 solution into the FP64 one
    int restart;  // an FP32 breakdown: no step, direction restarted after the replacement
    int breakdowns;
};

struct MultiGlobal {
    unsigned finished;
    unsigned anyPending;  // FP32-refined form: some column requested a replacement
    long long chunkIter, chunkLimit, maxIter;
    double absTol, relTol;
    double delta;  // FP32-refined form: replacement trigger
    long long replacements;  // FP32-refined form: residual recomputations (launches of T)
};

// FP32 breakdowns (p^T A p <= 0 in single precision) a column may recover from
// by a replacement with a restarted direction before it reports the breakdown.
constexpr int kMaxColumnBreakdowns = 64;

template <bool COND>
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle cond, unsigned value) {
    if constexpr (COND) cudaGraphSetConditional(cond, value);
}

// Per-column sums of NV values over the grid.  Every thread holds the values of
// its column (lane % KP); the CTA holding the last block gets the totals of
// column c in thread c (c < k) and returns true.  partials: NV x grid x 32.
template <int KP, int NV>
__device__ __forceinline__ bool column_reduce_last(const double (&mine)[NV], int k, double* partials,
                                                   unsigned* counter, double (&out)[NV]) {
    __shared__ double s_red[NV][kT];
    __shared__ bool s_last;
#pragma unroll
    for (int v = 0; v < NV; ++v) s_red[v][threadIdx.x] = mine[v];
    __syncthreads();
    if (threadIdx.x < k) {
        const int c = threadIdx.x;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double acc = 0.0;
            for (int t = c; t < kT; t += KP) acc += s_red[v][t];  // fixed order: warps, then slots
            partials[(static_cast<long>(v) * gridDim.x + blockIdx.x) * 32 + c] = acc;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    // column c = lane, blocks split over the warps, then the warps' sums in order
    const int c = threadIdx.x & 31, part = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double acc = 0.0;
        const volatile double* p = partials + static_cast<long>(v) * gridDim.x * 32;
        if (c < k)
            for (unsigned b = part; b < gridDim.x; b += kWarps) acc += p[static_cast<long>(b) * 32 + c];
        __syncthreads();
        s_red[v][threadIdx.x] = acc;
        __syncthreads();
        if (threadIdx.x < k) {
            double tot = 0.0;
            for (int w = 0; w < kWarps; ++w) tot += s_red[v][w * 32 + threadIdx.x];
            out[v] = tot;
        }
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// Row sums of A times the n x k block X; calls op(row, c, sum) for each row and
// active column.  The CTA takes the row blocks of the CSR handle (at most
// kStreamTile entries each) in turn, interleaved over the grid so that all CTAs
// advance through the rows together and the gathered X rows stay in L2; it
// stages a block's values and column indices in shared memory with coalesced
// loads, then every lane of a row group reads (a_ij, j) as a shared-memory
// broadcast and gathers X[j][c]: one load and one FMA per entry and lane, the
// entries of a row summed in CSR order.  A row longer than the tile (a block of
// its own) is read straight from global memory.
struct __align__(16) Entry {
    double a;
    int col;
    int pad;
};

// One 16-byte shared-memory read of an entry.
__device__ __forceinline__ void load_entry(const Entry* e, double& a, int& col) {
    const double2 raw = *reinterpret_cast<const double2*>(e);
    a = raw.x;
    col = static_cast<int>(__double_as_longlong(raw.y) & 0xffffffffLL);
}

// FULL: k == KP, so every lane is active and the row stride of X is the
// compile-time KP (the gather address is a shift and an add).  V: stored value
// type (staged as a double, exactly), T: vector and accumulation type.
template <int KP, bool FULL, typename V, typename T, typename Op>
__device__ __forceinline__ void multi_rows(const CsrArgs<V>& A, int k, const T* __restrict__ X, Op& op) {
    __shared__ Entry s_e[kStreamTile];  // one 16-byte broadcast read per entry
    constexpr int RPW = 32 / KP;
    constexpr int UNROLL = 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    const bool active = FULL || c < k;
    const long ld = FULL ? KP : k;
    const T* __restrict__ xc = X + c;
    for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
        const int r0 = A.blocks[b], r1 = A.blocks[b + 1];
        const int e0 = A.rowptr[r0], e1 = A.rowptr[r1];
        const bool staged = e1 - e0 <= kStreamTile;
        if (staged) {
            for (int j = threadIdx.x; j < e1 - e0; j += kT)
                s_e[j] = Entry{static_cast<double>(stream_ld(A.val + e0 + j)), stream_ld(A.col + e0 + j), 0};
            __syncthreads();
        }
        for (int rbase = r0 + warp * RPW; rbase < r1; rbase += kWarps * RPW) {
            const int row = rbase + slot;
            if (row >= r1) continue;
            const int k0 = A.rowptr[row] - e0, k1 = A.rowptr[row + 1] - e0;
            T acc = 0;
            if (staged) {
                int j = k0;
                for (; j + UNROLL <= k1; j += UNROLL) {
                    T av[UNROLL], pv[UNROLL];
#pragma unroll
                    for (int u = 0; u < UNROLL; ++u) {
                        double a;
                        int col;
                        load_entry(s_e + j + u, a, col);
                        av[u] = static_cast<T>(a);
                        pv[u] = active ? __ldg(xc + static_cast<long>(col) * ld) : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < UNROLL; ++u) acc = fma(av[u], pv[u], acc);
                }
                for (; j < k1; ++j) {
                    double a;
                    int col;
                    load_entry(s_e + j, a, col);
                    acc = fma(static_cast<T>(a), active ? __ldg(xc + static_cast<long>(col) * ld) : T(0), acc);
                }
            } else {
                for (int j = e0 + k0; j < e0 + k1; ++j)
                    acc = fma(static_cast<T>(A.val[j]), active ? __ldg(xc + static_cast<long>(A.col[j]) * ld) : T(0),
                              acc);
            }
            if (active) op(row, c, acc);
        }
        if (staged) __syncthreads();
    }
}

// The same row sums over the DIA copy of a few-diagonal matrix (dia.cuh): lane c
// of a row's group reads the diagonal value (one broadcast load for the group)
// and X[row + off[d]][c] (k consecutive doubles, coalesced).  No staging, no
// column indices; the diagonals run in ascending order, i.e. in the CSR column
// order, so the sums equal those of multi_rows.
template <int KP, bool FULL, typename V, typename T, typename Op>
__device__ __forceinline__ void multi_dia_rows(const DiaArgs<V>& D, int k, const T* __restrict__ X, Op& op) {
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    const bool active = FULL || c < k;
    const long ld = FULL ? KP : k;
    const T* __restrict__ xc = X + c;
    const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
    for (long row = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; row < D.nrows; row += stride) {
        T acc = 0;
#pragma unroll 9
        for (int d = 0; d < D.ndiag; ++d) {
            const long col = row + D.off[d];
            const T a = static_cast<T>(stream_ld(D.val + static_cast<long>(d) * D.ld + row));
            const T xv =
                active && static_cast<unsigned long>(col) < static_cast<unsigned long>(D.nrows) ? __ldg(xc + col * ld)
                                                                                                 : T(0);
            acc = fma(a, xv, acc);
        }
        if (active) op(row, c, acc);
    }
}

struct ResidualOp {  // R = B - A X
    const double* __restrict__ b;
    double* __restrict__ r;
    int k;
    __device__ __forceinline__ void operator()(long row, int c, double sum) const {
        r[row * k + c] = b[row * k + c] - sum;
    }
};

template <int KP, bool FULL>
__global__ void __launch_bounds__(kT) multi_residual_kernel(CsrArgs<double> A, int k, const double* __restrict__ X,
                                                            const double* __restrict__ B, double* __restrict__ R) {
    ResidualOp op{B, R, k};
    multi_rows<KP, FULL>(A, k, X, op);
}

template <int KP, bool FULL>
__global__ void __launch_bounds__(kT) multi_residual_dia_kernel(DiaArgs<double> D, int k,
                                                                const double* __restrict__ X,
                                                                const double* __restrict__ B, double* __restrict__ R) {
    ResidualOp op{B, R, k};
    multi_dia_rows<KP, FULL>(D, k, X, op);
}

// Initial set-up per column: z = D^-1 r, p = z, rr, rz and the initial test.
template <int KP>
__global__ void __launch_bounds__(kT) multi_init_kernel(long n, int k, const double* __restrict__ R,
                                                        const double* __restrict__ dinv, double* __restrict__ P,
                                                        ColumnScalars* S, MultiGlobal* g, double* partials,
                                                        unsigned* counter) {
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    double rr = 0.0, rz = 0.0;
    const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
    if (c < k)
#pragma unroll 4
        for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
            const double ri = R[i * k + c];
            const double zi = ri * dinv[i];
            P[i * k + c] = zi;
            rr = fma(ri, ri, rr);
            rz = fma(ri, zi, rz);
        }
    double mine[2] = {rr, rz}, tot[2];
    if (column_reduce_last<KP, 2>(mine, k, partials, counter, tot) && threadIdx.x < k) {
        ColumnScalars& s = S[threadIdx.x];
        s.rr = tot[0];
        s.r0 = sqrt(tot[0]);
        s.absres = s.r0;
        s.relres = 1.0;
        s.iter = 0;
        s.done = 0;
        s.errorKind = 0;
        s.errorIter = 0;
        if (float_less(s.absres, g->absTol) || float_less(s.relres, g->relTol)) {
            s.done = 1;
        } else {
            s.rz = tot[1];
            if (!(0.0 < s.rz)) {
                s.done = 3;
                s.errorKind = 1;
            } else if (g->maxIter <= 0) {
                s.done = 2;
            }
        }
        if (s.done) atomicAdd(&g->finished, 1u);
    }
}

struct PqOp {
    const double* __restrict__ p;
    double* __restrict__ q;
    int k;
    double acc;
    __device__ __forceinline__ void operator()(long row, int c, double sum) {
        q[row * k + c] = sum;
        acc = fma(p[row * k + c], sum, acc);
    }
};

// K1: Q = A P and p_c^T q_c; alpha per column.
template <int KP, bool FULL, bool COND>
__global__ void __launch_bounds__(kT) multi_spmv_kernel(CsrArgs<double> A, int k, const double* __restrict__ P,
                                                        double* __restrict__ Q, ColumnScalars* S, MultiGlobal* g,
                                                        double* partials, unsigned* counter,
                                                        cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp op{P, Q, k, 0.0};
    multi_rows<KP, FULL>(A, k, P, op);
    double mine[1] = {op.acc}, tot[1];
    if (column_reduce_last<KP, 1>(mine, k, partials, counter, tot) && threadIdx.x < k) {
        ColumnScalars& s = S[threadIdx.x];
        if (!s.done) {
            s.pq = tot[0];
            if (!(0.0 < tot[0])) {
                s.done = 3;
                s.errorKind = 2;
                s.errorIter = s.iter;
                atomicAdd(&g->finished, 1u);
            } else {
                s.alpha = s.rz / tot[0];
            }
        }
    }
}

template <int KP, bool FULL, bool COND>
__global__ void __launch_bounds__(kT) multi_spmv_dia_kernel(DiaArgs<double> D, int k, const double* __restrict__ P,
                                                            double* __restrict__ Q, ColumnScalars* S, MultiGlobal* g,
                                                            double* partials, unsigned* counter,
                                                            cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp op{P, Q, k, 0.0};
    multi_dia_rows<KP, FULL>(D, k, P, op);
    double mine[1] = {op.acc}, tot[1];
    if (column_reduce_last<KP, 1>(mine, k, partials, counter, tot) && threadIdx.x < k) {
        ColumnScalars& s = S[threadIdx.x];
        if (!s.done) {
            s.pq = tot[0];
            if (!(0.0 < tot[0])) {
                s.done = 3;
                s.errorKind = 2;
                s.errorIter = s.iter;
                atomicAdd(&g->finished, 1u);
            } else {
                s.alpha = s.rz / tot[0];
            }
        }
    }
}

// K2: X += alpha P; R -= alpha Q; rr, rz; beta and the stopping test per column.
template <int KP>
__global__ void __launch_bounds__(kT) multi_update_kernel(long n, int k, double* __restrict__ X,
                                                          double* __restrict__ R, const double* __restrict__ P,
                                                          const double* __restrict__ Q,
                                                          const double* __restrict__ dinv, ColumnScalars* S,
                                                          MultiGlobal* g, double* partials, unsigned* counter) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) return;
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    double rr = 0.0, rz = 0.0;
    if (c < k && !S[c].done) {
        const double alpha = S[c].alpha, malpha = -alpha;
        const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
#pragma unroll 4
        for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
            const long e = i * k + c;
            X[e] = fma(alpha, P[e], X[e]);
            const double ri = fma(malpha, Q[e], R[e]);
            R[e] = ri;
            rr = fma(ri, ri, rr);
            rz = fma(ri, ri * dinv[i], rz);
        }
    }
    double mine[2] = {rr, rz}, tot[2];
    if (column_reduce_last<KP, 2>(mine, k, partials, counter, tot) && threadIdx.x < k) {
        ColumnScalars& s = S[threadIdx.x];
        if (!s.done) {
            s.rr = tot[0];
            s.beta = tot[1] / s.rz;
            s.rz = tot[1];
            s.absres = sqrt(tot[0]);
            s.relres = s.absres / s.r0;
            if (float_less(s.absres, g->absTol) || float_less(s.relres, g->relTol)) {
                s.done = 1;
            } else {
                s.iter += 1;
                if (s.iter >= g->maxIter) s.done = 2;
            }
            if (s.done) atomicAdd(&g->finished, 1u);
        }
    }
}

// K3: P = beta P + D^-1 R per running column; ends the loop when all are done.
template <int KP, bool COND>
__global__ void __launch_bounds__(kT) multi_direction_kernel(long n, int k, double* __restrict__ P,
                                                             const double* __restrict__ R,
                                                             const double* __restrict__ dinv,
                                                             const ColumnScalars* S, MultiGlobal* g,
                                                             cudaGraphConditionalHandle cond) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g->chunkIter += 1;
        const bool more = *reinterpret_cast<volatile unsigned*>(&g->finished) < static_cast<unsigned>(k);
        set_loop<COND>(cond, (more && g->chunkIter < g->chunkLimit) ? 1u : 0u);
    }
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    if (c >= k || S[c].done) return;
    const double beta = S[c].beta;
    const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
#pragma unroll 4
    for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
        const long e = i * k + c;
        P[e] = __dadd_rn(__dmul_rn(P[e], beta), __dmul_rn(R[e], dinv[i]));
    }
}

// ---- FP32-refined form: FP32 inner iterations, FP64 reliable updates ---------
//
// Per column the iteration of the mixed-precision solver: K1 Q32 = A32 P32 and
// p^T q (FP64 sums); K2 X32 += alpha P32, R32 -= alpha Q32, the FP32 recursion's
// r^T r and r^T z in FP64 and the replacement decision (the FP32 residual norm
// fell below delta times its maximum since the last replacement, or below the
// stopping tolerance, or the iteration limit); when any column asks, F folds
// X32 into the FP64 solution and T recomputes R = B - A64 X64 in FP64 for those
// columns, stores float(R) and applies the FP64 stopping test; K3 P32 = D^-1 R32
// + beta P32.  Columns that are done are left unchanged.

struct PqOp32 {
    const float* __restrict__ p;
    float* __restrict__ q;
    int k;
    double acc;
    __device__ __forceinline__ void operator()(long row, int c, float sum) {
        q[row * k + c] = sum;
        acc = fma(static_cast<double>(p[row * k + c]), static_cast<double>(sum), acc);
    }
};

__device__ __forceinline__ void column_pq(ColumnScalars& s, double pq, MultiGlobal* g) {
    if (s.done) return;
    s.pq = pq;
    if (!(0.0 < pq)) {  // FP32 breakdown: no step, replacement with a restarted direction
        s.alpha = 0.0;
        s.restart = 1;
        s.breakdowns += 1;
        if (s.breakdowns > kMaxColumnBreakdowns) {
            s.done = 3;
            s.errorKind = 2;
            s.errorIter = s.iter;
            atomicAdd(&g->finished, 1u);
        }
    } else {
        s.alpha = s.rz / pq;
    }
}

template <int KP, bool FULL, bool COND>
__global__ void __launch_bounds__(kT) multi_spmv32_kernel(CsrArgs<float> A, int k, const float* __restrict__ P,
                                                          float* __restrict__ Q, ColumnScalars* S, MultiGlobal* g,
                                                          double* partials, unsigned* counter,
                                                          cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp32 op{P, Q, k, 0.0};
    multi_rows<KP, FULL>(A, k, P, op);
    double mine[1] = {op.acc}, tot[1];
    if (column_reduce_last<KP, 1>(mine, k, partials, counter, tot) && threadIdx.x < k)
        column_pq(S[threadIdx.x], tot[0], g);
}

template <int KP, bool FULL, bool COND>
__global__ void __launch_bounds__(kT) multi_spmv32_dia_kernel(DiaArgs<float> D, int k, const float* __restrict__ P,
                                                              float* __restrict__ Q, ColumnScalars* S,
                                                              MultiGlobal* g, double* partials, unsigned* counter,
                                                              cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp32 op{P, Q, k, 0.0};
    multi_dia_rows<KP, FULL>(D, k, P, op);
    double mine[1] = {op.acc}, tot[1];
    if (column_reduce_last<KP, 1>(mine, k, partials, counter, tot) && threadIdx.x < k)
        column_pq(S[threadIdx.x], tot[0], g);
}

// K2 of the refined form.  IF: the handle of the replacement (set when any column
// asks for one).
template <int KP, bool COND>
__global__ void __launch_bounds__(kT) multi_update32_kernel(long n, int k, float* __restrict__ X,
                                                            float* __restrict__ R, const float* __restrict__ P,
                                                            const float* __restrict__ Q,
                                                            const float* __restrict__ dinv, ColumnScalars* S,
                                                            MultiGlobal* g, double* partials, unsigned* counter,
                                                            cudaGraphConditionalHandle replace) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= static_cast<unsigned>(k)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(replace, 0);
        return;
    }
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    double rr = 0.0, rz = 0.0;
    if (c < k && !S[c].done) {
        const bool step = !S[c].restart;
        const float alpha = static_cast<float>(S[c].alpha), malpha = -alpha;
        const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
#pragma unroll 4
        for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
            const long e = i * k + c;
            float ri = R[e];
            if (step) {
                X[e] = fmaf(alpha, P[e], X[e]);
                ri = fmaf(malpha, Q[e], ri);
                R[e] = ri;
            }
            rr = fma(static_cast<double>(ri), static_cast<double>(ri), rr);
            rz = fma(static_cast<double>(ri), static_cast<double>(ri * dinv[i]), rz);
        }
    }
    double mine[2] = {rr, rz}, tot[2];
    __shared__ unsigned s_any;
    if (threadIdx.x == 0) s_any = 0u;
    const bool last = column_reduce_last<KP, 2>(mine, k, partials, counter, tot);
    if (!last) return;
    __syncthreads();
    // The replacement recomputes B - A X for all columns in one FP64 SpMM, so it is
    // taken by every running column at once, and only when it is due for the batch:
    // when some column must stop or restart (FP32 residual below the tolerance,
    // iteration limit, FP32 breakdown), or when at least half of the running
    // columns have seen their FP32 residual drop by delta.  A column whose drop
    // came early keeps iterating until then (reliable updates bound the drift by
    // the drop, not by the iteration).
    __shared__ unsigned s_running, s_wanting;
    if (threadIdx.x == 0) s_running = s_wanting = 0u;
    __syncthreads();
    bool running = false, updateX = false;
    if (threadIdx.x < k) {
        ColumnScalars& s = S[threadIdx.x];
        running = !s.done;
        if (running) {
            const double rnorm = sqrt(tot[0]);
            s.iter += 1;
            if (rnorm > s.maxrx) s.maxrx = rnorm;
            if (rnorm > s.maxrr) s.maxrr = rnorm;
            updateX = rnorm < g->delta * s.maxrx;
            const bool want = updateX || rnorm < g->delta * s.maxrr;
            const bool must = rnorm < g->relTol * s.r0 || rnorm < g->absTol || s.iter >= g->maxIter || s.restart;
            atomicAdd(&s_running, 1u);
            if (want) atomicAdd(&s_wanting, 1u);
            if (must) atomicOr(&s_any, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && 2u * s_wanting >= s_running && s_wanting > 0u) s_any = 1u;
    __syncthreads();
    if (threadIdx.x < k && running) {
        ColumnScalars& s = S[threadIdx.x];
        if (s_any) {
            s.pending = 1;
            s.updateX = updateX ? 1 : 0;
            s.rzPending = tot[1];
        } else {
            s.beta = tot[1] / s.rz;
            s.rz = tot[1];
        }
    }
    if (threadIdx.x == 0) {
        g->anyPending = s_any;
        set_loop<COND>(replace, s_any);
    }
}

// F: X64 += X32, X32 = 0 for the columns with a replacement due.
template <int KP>
__global__ void __launch_bounds__(kT) multi_fold32_kernel(long n, int k, double* __restrict__ X64,
                                                          float* __restrict__ X32, const ColumnScalars* S,
                                                          const MultiGlobal* g) {
    if (!*reinterpret_cast<const volatile unsigned*>(&g->anyPending)) return;
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    if (c >= k || !S[c].pending) return;
    const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
#pragma unroll 4
    for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
        const long e = i * k + c;
        X64[e] += static_cast<double>(X32[e]);
        X32[e] = 0.0f;
    }
}

// T (and the set-up, INIT): R = B - A64 X64 in FP64 for the columns with a
// replacement due (every column at the set-up); R32 = float(R), ||R|| in FP64,
// r32^T z32; the FP64 stopping test and the direction's beta.
struct TrueResidualOp {
    const double* __restrict__ b;
    const float* __restrict__ dinv;
    float* __restrict__ r32;
    const ColumnScalars* S;
    int k;
    bool init;
    double rr, rz;
    __device__ __forceinline__ void operator()(long row, int c, double sum) {
        if (!init && !S[c].pending) return;
        const double ri = b[row * k + c] - sum;
        const float rf = static_cast<float>(ri);
        r32[row * k + c] = rf;
        rr = fma(ri, ri, rr);
        rz = fma(static_cast<double>(rf), static_cast<double>(rf * dinv[row]), rz);
    }
};

template <bool INIT>
__device__ __forceinline__ void column_replace(ColumnScalars& s, const double (&tot)[2], MultiGlobal* g) {
    const double rnorm = sqrt(tot[0]);
    if (INIT) {
        s = ColumnScalars{};
        s.r0 = rnorm;
        s.absres = rnorm;
        s.relres = 1.0;
        s.maxrx = s.maxrr = rnorm;
        s.beta = 0.0;
        s.rz = tot[1];
        if (float_less(s.absres, g->absTol) || float_less(s.relres, g->relTol)) {
            s.done = 1;
        } else if (!(0.0 < tot[1])) {
            s.done = 3;
            s.errorKind = 1;
        } else if (g->maxIter <= 0) {
            s.done = 2;
        }
        if (s.done) atomicAdd(&g->finished, 1u);
        return;
    }
    if (s.done || !s.pending) return;
    s.pending = 0;
    s.refinements += 1;
    s.rr = tot[0];
    s.absres = rnorm;
    s.relres = rnorm / s.r0;
    if (float_less(s.absres, g->absTol) || float_less(s.relres, g->relTol)) {
        s.done = 1;
    } else if (s.iter >= g->maxIter) {
        s.done = 2;
    } else if (!(0.0 < tot[1])) {
        s.done = 3;
        s.errorKind = 1;
        s.errorIter = s.iter;
    } else {
        s.maxrr = rnorm;
        if (s.updateX) s.maxrx = rnorm;
        s.beta = s.restart ? 0.0 : tot[1] / s.rz;  // after an FP32 breakdown: p = z
        s.rz = tot[1];
    }
    s.restart = 0;
    if (s.done) atomicAdd(&g->finished, 1u);
}

template <int KP, bool FULL, bool INIT>
__global__ void __launch_bounds__(kT) multi_true_residual_kernel(CsrArgs<double> A, int k,
                                                                 const double* __restrict__ X,
                                                                 const double* __restrict__ B,
                                                                 const float* __restrict__ dinv,
                                                                 float* __restrict__ R32, ColumnScalars* S,
                                                                 MultiGlobal* g, double* partials,
                                                                 unsigned* counter) {
    if (!INIT && !*reinterpret_cast<volatile unsigned*>(&g->anyPending)) return;
    TrueResidualOp op{B, dinv, R32, S, k, INIT, 0.0, 0.0};
    multi_rows<KP, FULL>(A, k, X, op);
    double mine[2] = {op.rr, op.rz}, tot[2];
    if (column_reduce_last<KP, 2>(mine, k, partials, counter, tot)) {
        if (threadIdx.x < k) column_replace<INIT>(S[threadIdx.x], tot, g);
        __syncthreads();
        if (threadIdx.x == 0) {
            g->anyPending = 0u;
            if (!INIT) g->replacements += 1;
        }
    }
}

template <int KP, bool FULL, bool INIT>
__global__ void __launch_bounds__(kT) multi_true_residual_dia_kernel(DiaArgs<double> D, int k,
                                                                     const double* __restrict__ X,
                                                                     const double* __restrict__ B,
                                                                     const float* __restrict__ dinv,
                                                                     float* __restrict__ R32, ColumnScalars* S,
                                                                     MultiGlobal* g, double* partials,
                                                                     unsigned* counter) {
    if (!INIT && !*reinterpret_cast<volatile unsigned*>(&g->anyPending)) return;
    TrueResidualOp op{B, dinv, R32, S, k, INIT, 0.0, 0.0};
    multi_dia_rows<KP, FULL>(D, k, X, op);
    double mine[2] = {op.rr, op.rz}, tot[2];
    if (column_reduce_last<KP, 2>(mine, k, partials, counter, tot)) {
        if (threadIdx.x < k) column_replace<INIT>(S[threadIdx.x], tot, g);
        __syncthreads();
        if (threadIdx.x == 0) {
            g->anyPending = 0u;
            if (!INIT) g->replacements += 1;
        }
    }
}

// K3 of the refined form: P32 = D^-1 R32 + beta P32 per running column; ends the
// loop when all are done.
template <int KP, bool COND>
__global__ void __launch_bounds__(kT) multi_direction32_kernel(long n, int k, float* __restrict__ P,
                                                               const float* __restrict__ R,
                                                               const float* __restrict__ dinv,
                                                               const ColumnScalars* S, MultiGlobal* g,
                                                               cudaGraphConditionalHandle cond) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g->chunkIter += 1;
        const bool more = *reinterpret_cast<volatile unsigned*>(&g->finished) < static_cast<unsigned>(k);
        set_loop<COND>(cond, (more && g->chunkIter < g->chunkLimit) ? 1u : 0u);
    }
    constexpr int RPW = 32 / KP;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / KP, c = lane % KP;
    if (c >= k || S[c].done) return;
    const float beta = static_cast<float>(S[c].beta);
    const long stride = static_cast<long>(gridDim.x) * kWarps * RPW;
    if (beta == 0.0f) {  // a new direction: the old one may not be finite after a breakdown
#pragma unroll 4
        for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride)
            P[i * k + c] = R[i * k + c] * dinv[i];
        return;
    }
#pragma unroll 4
    for (long i = (static_cast<long>(blockIdx.x) * kWarps + warp) * RPW + slot; i < n; i += stride) {
        const long e = i * k + c;
        P[e] = fmaf(beta, P[e], R[e] * dinv[i]);
    }
}

// ---- k = 32: four columns per lane ---------------------------------------------
//
// With 32 right-hand sides a lane of the row-per-warp engines above issues one
// 4- or 8-byte gather and one FMA per entry, so the SpMM is bound by instruction
// issue, not by memory.  Here a lane keeps four consecutive columns (one 16-byte
// load for FP32, two for FP64): eight lanes cover a row's 32 columns and a warp
// works on four rows at once, so each gather instruction moves four times the
// bytes and the matrix value is loaded once per eight lanes.  The entries of a
// row are summed in the same order as above (CSR order / ascending diagonals),
// so the sums are the same.

template <typename T>
struct Quad;
template <>
struct Quad<float> {
    static __device__ __forceinline__ void load(const float* p, float (&v)[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    static __device__ __forceinline__ void load_plain(const float* p, float (&v)[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    static __device__ __forceinline__ void store(float* p, const float (&v)[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <>
struct Quad<double> {
    static __device__ __forceinline__ void load(const double* p, double (&v)[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    static __device__ __forceinline__ void load_plain(const double* p, double (&v)[4]) {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    static __device__ __forceinline__ void store(double* p, const double (&v)[4]) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
};

constexpr int kQuadLanes = 8;                 // lanes per row
constexpr int kQuadRows = 32 / kQuadLanes;    // rows per warp

// CSR rows of the row blocks (staged as in multi_rows); op.quad(row, c0, acc)
// receives columns c0 .. c0 + 3 of the row.
template <typename V, typename T, typename Op>
__device__ __forceinline__ void quad_rows(const CsrArgs<V>& A, const T* __restrict__ X, Op& op) {
    __shared__ Entry s_e[kStreamTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / kQuadLanes, c0 = (lane % kQuadLanes) * 4;
    const T* __restrict__ xc = X + c0;
    for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
        const int r0 = A.blocks[b], r1 = A.blocks[b + 1];
        const int e0 = A.rowptr[r0], e1 = A.rowptr[r1];
        const bool staged = e1 - e0 <= kStreamTile;
        if (staged) {
            for (int j = threadIdx.x; j < e1 - e0; j += kT)
                s_e[j] = Entry{static_cast<double>(stream_ld(A.val + e0 + j)), stream_ld(A.col + e0 + j), 0};
            __syncthreads();
        }
        for (int rbase = r0 + warp * kQuadRows; rbase < r1; rbase += kWarps * kQuadRows) {
            const int row = rbase + slot;
            if (row >= r1) continue;
            const int k0 = A.rowptr[row] - e0, k1 = A.rowptr[row + 1] - e0;
            T acc[4] = {T(0), T(0), T(0), T(0)};
            if (staged) {
                int j = k0;
                for (; j + 2 <= k1; j += 2) {
                    double a0, a1;
                    int col0, col1;
                    load_entry(s_e + j, a0, col0);
                    load_entry(s_e + j + 1, a1, col1);
                    T x0[4], x1[4];
                    Quad<T>::load(xc + static_cast<long>(col0) * 32, x0);
                    Quad<T>::load(xc + static_cast<long>(col1) * 32, x1);
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] = fma(static_cast<T>(a0), x0[u], acc[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] = fma(static_cast<T>(a1), x1[u], acc[u]);
                }
                if (j < k1) {
                    double a;
                    int col;
                    load_entry(s_e + j, a, col);
                    T xv[4];
                    Quad<T>::load(xc + static_cast<long>(col) * 32, xv);
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] = fma(static_cast<T>(a), xv[u], acc[u]);
                }
            } else {
                for (int j = e0 + k0; j < e0 + k1; ++j) {
                    T xv[4];
                    Quad<T>::load(xc + static_cast<long>(A.col[j]) * 32, xv);
                    const T a = static_cast<T>(A.val[j]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] = fma(a, xv[u], acc[u]);
                }
            }
            op.quad(row, c0, acc);
        }
        if (staged) __syncthreads();
    }
}

// DIA rows (diagonals in ascending order = the CSR column order).
template <typename V, typename T, typename Op>
__device__ __forceinline__ void quad_rows(const DiaArgs<V>& D, const T* __restrict__ X, Op& op) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / kQuadLanes, c0 = (lane % kQuadLanes) * 4;
    const T* __restrict__ xc = X + c0;
    const long stride = static_cast<long>(gridDim.x) * kWarps * kQuadRows;
    for (long row = (static_cast<long>(blockIdx.x) * kWarps + warp) * kQuadRows + slot; row < D.nrows;
         row += stride) {
        T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 3
        for (int d = 0; d < D.ndiag; ++d) {
            const long col = row + D.off[d];
            const T a = static_cast<T>(stream_ld(D.val + static_cast<long>(d) * D.ld + row));
            if (static_cast<unsigned long>(col) < static_cast<unsigned long>(D.nrows)) {
                T xv[4];
                Quad<T>::load(xc + col * 32, xv);
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(a, xv[u], acc[u]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] = fma(a, T(0), acc[u]);
            }
        }
        op.quad(row, c0, acc);
    }
}

// The DIA pass for stencils whose sorted offsets come in consecutive triples
// (o - 1, o, o + 1) -- the 27- and 9-diagonal Q1 stencils: a lane keeps its four
// columns of FOUR consecutive rows (a warp sixteen rows), and for every triple
// loads the six operand rows r + o - 1 .. r + o + 4 once, where the one-row
// layout above loads twelve (each of the four rows' three neighbours).  The
// diagonal values of the four rows are one 16-byte (FP32) or two (FP64) loads,
// the same address for the eight lanes of a row group.  Triples in ascending
// order and the three diagonals of a triple in order keep every row sum in the
// CSR column order (out-of-range operand rows are zeros, as above), so the sums
// are those of quad_rows.
template <typename V, typename T, typename Op>
__device__ __forceinline__ void quad_rows_dia3(const DiaArgs<V>& D, const T* __restrict__ X, Op& op) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = lane / kQuadLanes, c0 = (lane % kQuadLanes) * 4;
    const T* __restrict__ xc = X + c0;
    const int n = D.nrows;
    const int triples = D.ndiag / 3;
    const long stride = static_cast<long>(gridDim.x) * kWarps * 16;
    for (long r0l = (static_cast<long>(blockIdx.x) * kWarps + warp) * 16 + 4 * slot; r0l < n; r0l += stride) {
        const int r0 = static_cast<int>(r0l);
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[i][u] = T(0);
#pragma unroll 1
        for (int t = 0; t < triples; ++t) {
            const int o = D.off[3 * t + 1];
            T xr[6][4];
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                const int c = r0 + o - 1 + j;
                if (static_cast<unsigned>(c) < static_cast<unsigned>(n)) {
                    Quad<T>::load(xc + static_cast<long>(c) * 32, xr[j]);
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u) xr[j][u] = T(0);
                }
            }
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                V v[4];
                Quad<V>::load(D.val + static_cast<long>(3 * t + e) * D.ld + r0, v);
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[i][u] = fma(static_cast<T>(v[i]), xr[i + e][u], acc[i][u]);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (r0 + i < n) op.quad(r0 + i, c0, acc[i]);
    }
}

// The DIA pass of the k = 32 kernels: triples when the stencil has them.
template <bool TRIPLES, typename V, typename T, typename Op>
__device__ __forceinline__ void quad_rows_dia(const DiaArgs<V>& D, const T* __restrict__ X, Op& op) {
    if constexpr (TRIPLES)
        quad_rows_dia3(D, X, op);
    else
        quad_rows(D, X, op);
}

template <bool TRIPLES, typename V, typename T, typename Op>
__device__ __forceinline__ void quad_pass(const CsrArgs<V>& A, const T* __restrict__ X, Op& op) {
    quad_rows(A, X, op);
}
template <bool TRIPLES, typename V, typename T, typename Op>
__device__ __forceinline__ void quad_pass(const DiaArgs<V>& D, const T* __restrict__ X, Op& op) {
    quad_rows_dia<TRIPLES>(D, X, op);
}

// Per-column totals of four-column partial sums (thread: columns c0 .. c0+3 of
// its rows): summed over the warp's four row slots, then lane c takes column c,
// and the column reduction of the row-per-warp kernels finishes the job.
template <int NV>
__device__ __forceinline__ bool quad_reduce_last(double (&part)[NV][4], double* partials, unsigned* counter,
                                                 double (&out)[NV]) {
    const int lane = threadIdx.x & 31;
    double mine[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            double x = part[v][u];
            x += __shfl_xor_sync(0xffffffffu, x, 8);
            x += __shfl_xor_sync(0xffffffffu, x, 16);
            t[u] = __shfl_sync(0xffffffffu, x, lane >> 2);  // lane (slot 0, group lane / 4)
        }
        const int u = lane & 3;
        mine[v] = u == 0 ? t[0] : u == 1 ? t[1] : u == 2 ? t[2] : t[3];
    }
    return column_reduce_last<32, NV>(mine, 32, partials, counter, out);
}

template <typename T>
struct PqQuad {
    const T* __restrict__ p;
    T* __restrict__ q;
    double acc[1][4];
    __device__ __forceinline__ void quad(long row, int c0, const T (&sum)[4]) {
        Quad<T>::store(q + row * 32 + c0, sum);
        T pv[4];
        Quad<T>::load_plain(p + row * 32 + c0, pv);
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[0][u] = fma(static_cast<double>(pv[u]), static_cast<double>(sum[u]), acc[0][u]);
    }
};

struct ResidualQuad {  // R = B - A X
    const double* __restrict__ b;
    double* __restrict__ r;
    __device__ __forceinline__ void quad(long row, int c0, const double (&sum)[4]) {
        double bv[4], rv[4];
        Quad<double>::load_plain(b + row * 32 + c0, bv);
#pragma unroll
        for (int u = 0; u < 4; ++u) rv[u] = bv[u] - sum[u];
        Quad<double>::store(r + row * 32 + c0, rv);
    }
};

struct TrueResidualQuad {
    const double* __restrict__ b;
    const float* __restrict__ dinv;
    float* __restrict__ r32;
    const ColumnScalars* S;
    bool init;
    double acc[2][4];
    __device__ __forceinline__ void quad(long row, int c0, const double (&sum)[4]) {
        double bv[4];
        Quad<double>::load_plain(b + row * 32 + c0, bv);
        const float d = dinv[row];
        float rf[4];
        float old[4];
        Quad<float>::load_plain(r32 + row * 32 + c0, old);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool take = init || S[c0 + u].pending;
            const double ri = bv[u] - sum[u];
            rf[u] = take ? static_cast<float>(ri) : old[u];
            if (take) {
                acc[0][u] = fma(ri, ri, acc[0][u]);
                acc[1][u] = fma(static_cast<double>(rf[u]), static_cast<double>(rf[u] * d), acc[1][u]);
            }
        }
        Quad<float>::store(r32 + row * 32 + c0, rf);
    }
};

// K1 for k = 32 over either format; FP64 (the plain form) or FP32 (the refined
// form, whose breakdowns restart).
template <typename MA, typename T, bool COND, bool TRIPLES>
__device__ __forceinline__ void multi_spmv_quad(MA A, const T* __restrict__ P, T* __restrict__ Q, ColumnScalars* S,
                                                MultiGlobal* g, double* partials, unsigned* counter,
                                                cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile unsigned*>(&g->finished) >= 32u) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqQuad<T> op{P, Q, {{0.0, 0.0, 0.0, 0.0}}};
    quad_pass<TRIPLES>(A, P, op);
    double tot[1];
    if (quad_reduce_last<1>(op.acc, partials, counter, tot) && threadIdx.x < 32) {
        ColumnScalars& s = S[threadIdx.x];
        if (std::is_same<T, float>::value) {
            column_pq(s, tot[0], g);
        } else if (!s.done) {
            s.pq = tot[0];
            if (!(0.0 < tot[0])) {
                s.done = 3;
                s.errorKind = 2;
                s.errorIter = s.iter;
                atomicAdd(&g->finished, 1u);
            } else {
                s.alpha = s.rz / tot[0];
            }
        }
    }
}

template <typename MA, typename T, bool COND, bool TRIPLES = false>
__global__ void __launch_bounds__(kT) multi_spmv_quad_kernel(MA A, const T* __restrict__ P, T* __restrict__ Q,
                                                             ColumnScalars* S, MultiGlobal* g, double* partials,
                                                             unsigned* counter, cudaGraphConditionalHandle cond) {
    multi_spmv_quad<MA, T, COND, TRIPLES>(A, P, Q, S, g, partials, counter, cond);
}

// The FP32 triple pass of the refined form with up to 85 registers (three CTAs
// per SM): at the compiler's own 64 the 32-RHS FP32 solve at 128^3 measured
// 475 against 438 ms.
template <bool COND>
__global__ void __launch_bounds__(kT, 3) multi_spmv_quad3_f32_kernel(DiaArgs<float> A, const float* __restrict__ P,
                                                                     float* __restrict__ Q, ColumnScalars* S,
                                                                     MultiGlobal* g, double* partials,
                                                                     unsigned* counter,
                                                                     cudaGraphConditionalHandle cond) {
    multi_spmv_quad<DiaArgs<float>, float, COND, true>(A, P, Q, S, g, partials, counter, cond);
}

template <typename MA, bool TRIPLES = false>
__global__ void __launch_bounds__(kT) multi_residual_quad_kernel(MA A, const double* __restrict__ X,
                                                                 const double* __restrict__ B, double* __restrict__ R) {
    ResidualQuad op{B, R};
    quad_pass<TRIPLES>(A, X, op);
}

template <typename MA, bool INIT, bool TRIPLES = false>
__global__ void __launch_bounds__(kT) multi_true_residual_quad_kernel(MA A, const double* __restrict__ X,
                                                                      const double* __restrict__ B,
                                                                      const float* __restrict__ dinv,
                                                                      float* __restrict__ R32, ColumnScalars* S,
                                                                      MultiGlobal* g, double* partials,
                                                                      unsigned* counter) {
    if (!INIT && !*reinterpret_cast<volatile unsigned*>(&g->anyPending)) return;
    TrueResidualQuad op{B, dinv, R32, S, INIT, {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}}};
    quad_pass<TRIPLES>(A, X, op);
    double tot[2];
    if (quad_reduce_last<2>(op.acc, partials, counter, tot)) {
        if (threadIdx.x < 32) column_replace<INIT>(S[threadIdx.x], tot, g);
        __syncthreads();
        if (threadIdx.x == 0) {
            g->anyPending = 0u;
            if (!INIT) g->replacements += 1;
        }
    }
}

__global__ void multi_to_f32_kernel(long n, const double* __restrict__ a, float* __restrict__ b) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        b[i] = static_cast<float>(a[i]);
}

__global__ void multi_output_kernel(long count, double inScale, double outScale, const double* __restrict__ x,
                                    double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
        const double xi = x[i];
        double o = out[i];
        if (inScale == 1.0) {
            o = outScale == 1.0 ? o + xi : (outScale == -1.0 ? o - xi : o + outScale * xi);
        } else if (inScale == 0.0) {
            o = xi * outScale;
        } else {
            o *= inScale;
            o = outScale == 1.0 ? o + xi : (outScale == -1.0 ? o - xi : o + outScale * xi);
        }
        out[i] = o;
    }
}

template <typename F>
int with_group(int kp, F&& f) {
    switch (kp) {
        case 1: return f(std::integral_constant<int, 1>{});
        case 2: return f(std::integral_constant<int, 2>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 16: return f(std::integral_constant<int, 16>{});
        default: return f(std::integral_constant<int, 32>{});
    }
}

}  // namespace
}  // namespace ciecu

struct ciecu_multi_s {
    ciecu_csr_s* A = nullptr;
    const double* dinv = nullptr;
    ciecu_statistics settings{};
    long n = 0;
    int k = 0, kp = 1;
    double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
    ciecu::ColumnScalars* d_s = nullptr;
    ciecu::MultiGlobal* d_g = nullptr;
    ciecu::MultiGlobal* h_g = nullptr;
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool deviceLoop = false;
    int chunk = 16;
    int grid = 1;   // SpMM kernels (register-limited occupancy)
    int gridV = 1;  // vector kernels
    // DIA copy of a few-diagonal matrix, refilled from the CSR values at every
    // solve; used when it timed faster at the first solve.
    bool diaChecked = false;
    bool useDia = false;
    int gridD = 1;
    double* diaBuf = nullptr;
    ciecu::DiaArgs<double> dia{};
    // FP32-refined form (refineDelta > 0): FP32 copies of the matrix (in the
    // format of the FP64 solve) and of D^-1, FP32 blocks, its own graph
    double refineDelta = 0.0;
    float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr, *dinv32 = nullptr;
    float* val32 = nullptr;  // CSR values
    float* dia32 = nullptr;  // DIA copy
    ciecu::DiaArgs<float> diaF{};
    int grid32 = 1, grid32D = 1;
    cudaGraphExec_t graph32 = nullptr;
    bool deviceLoop32 = false;
    cudaStream_t side = nullptr;  // captures the IF body of the replacement
    const double* graphB = nullptr;  // right-hand sides the refined graph reads
    std::vector<ciecu::ColumnScalars> last;  // column state of the last solve
    // k = 32: the four-columns-per-lane SpMM kernels (grids per format and precision)
    bool quad = false;
    int gridQ = 1, gridQD = 1, gridQ32 = 1, gridQ32D = 1;
    bool triples = false;  // the DIA offsets come in consecutive triples: the reuse pass (quad_rows_dia3)
    int formatPin = -1;    // -1: SpMM format by timing, 0: CSR, 1: the DIA copy (ciecu_multi_set_format)
    int gridQD3 = 1, gridQ32D3 = 1;
};

namespace ciecu {
namespace {

// CIECU_MULTI_QUAD=0 keeps the row-per-warp SpMM for k = 32 (for comparison).
bool quad_enabled() {
    static const bool enabled = [] {
        const char* v = std::getenv("CIECU_MULTI_QUAD");
        return !(v && v[0] == '0');
    }();
    return enabled;
}

template <bool COND>
int launch_multi_iteration(ciecu_multi_s* M, cudaStream_t st, cudaGraphConditionalHandle cond) {
    CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        if (M->quad && M->useDia && M->triples)
            multi_spmv_quad_kernel<DiaArgs<double>, double, COND, true><<<M->gridQD3, kT, 0, st>>>(
                M->dia, M->p, M->q, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->quad && M->useDia)
            multi_spmv_quad_kernel<DiaArgs<double>, double, COND><<<M->gridQD, kT, 0, st>>>(
                M->dia, M->p, M->q, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->quad)
            multi_spmv_quad_kernel<CsrArgs<double>, double, COND><<<M->gridQ, kT, 0, st>>>(
                M->A->args<double>(), M->p, M->q, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->useDia && M->k == KP)
            multi_spmv_dia_kernel<KP, true, COND><<<M->gridD, kT, 0, st>>>(M->dia, M->k, M->p, M->q, M->d_s, M->d_g,
                                                                           M->d_partials, M->d_counter, cond);
        else if (M->useDia)
            multi_spmv_dia_kernel<KP, false, COND><<<M->gridD, kT, 0, st>>>(M->dia, M->k, M->p, M->q, M->d_s,
                                                                            M->d_g, M->d_partials, M->d_counter,
                                                                            cond);
        else if (M->k == KP)
            multi_spmv_kernel<KP, true, COND><<<M->grid, kT, 0, st>>>(M->A->args<double>(), M->k, M->p, M->q, M->d_s,
                                                                      M->d_g, M->d_partials, M->d_counter, cond);
        else
            multi_spmv_kernel<KP, false, COND><<<M->grid, kT, 0, st>>>(M->A->args<double>(), M->k, M->p, M->q,
                                                                       M->d_s, M->d_g, M->d_partials, M->d_counter,
                                                                       cond);
        multi_update_kernel<KP><<<M->gridV, kT, 0, st>>>(M->n, M->k, M->x, M->r, M->p, M->q, M->dinv, M->d_s,
                                                         M->d_g, M->d_partials, M->d_counter);
        multi_direction_kernel<KP, COND><<<M->gridV, kT, 0, st>>>(M->n, M->k, M->p, M->r, M->dinv, M->d_s, M->d_g,
                                                                 cond);
        return CIECU_OK;
    }));
    CIECU_CHECK_LAUNCH("multi-rhs pcg iteration");
    return CIECU_OK;
}

// R = B - A X with the SpMM of the chosen format.
int launch_multi_residual(ciecu_multi_s* M, cudaStream_t st, bool dia, const double* B) {
    return with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        if (M->quad && dia && M->triples)
            multi_residual_quad_kernel<DiaArgs<double>, true><<<M->gridQD3, kT, 0, st>>>(M->dia, M->x, B, M->r);
        else if (M->quad && dia)
            multi_residual_quad_kernel<DiaArgs<double>><<<M->gridQD, kT, 0, st>>>(M->dia, M->x, B, M->r);
        else if (M->quad)
            multi_residual_quad_kernel<CsrArgs<double>><<<M->gridQ, kT, 0, st>>>(M->A->args<double>(), M->x, B, M->r);
        else if (dia && M->k == KP)
            multi_residual_dia_kernel<KP, true><<<M->gridD, kT, 0, st>>>(M->dia, M->k, M->x, B, M->r);
        else if (dia)
            multi_residual_dia_kernel<KP, false><<<M->gridD, kT, 0, st>>>(M->dia, M->k, M->x, B, M->r);
        else if (M->k == KP)
            multi_residual_kernel<KP, true><<<M->grid, kT, 0, st>>>(M->A->args<double>(), M->k, M->x, B, M->r);
        else
            multi_residual_kernel<KP, false><<<M->grid, kT, 0, st>>>(M->A->args<double>(), M->k, M->x, B, M->r);
        count_launch();
        return CIECU_OK;
    });
}

// At the first solve: build the DIA copy when the matrix has few diagonals and
// keep it if its SpMM (timed on the residual kernel, best of three) is faster.
// Later solves refill its values from the CSR arrays.
int prepare_dia(ciecu_multi_s* M, cudaStream_t st, const double* B) {
    if (!M->diaChecked) {
        M->diaChecked = true;
        const std::vector<int>* offsets = nullptr;
        CIECU_TRY(dia_offsets(M->A, &offsets));
        if (offsets->empty() || M->formatPin == 0) return CIECU_OK;
        DiaArgs<double> a = dia_shape<double>(M->A, *offsets);
        const size_t bytes = sizeof(double) * static_cast<size_t>(a.ndiag) * static_cast<size_t>(a.ld);
        if (cudaMalloc(&M->diaBuf, bytes) != cudaSuccess) {
            cudaGetLastError();  // no room for the copy: the CSR SpMM stays
            M->diaBuf = nullptr;
            return CIECU_OK;
        }
        CIECU_CUDA(cudaMemsetAsync(M->diaBuf, 0, bytes, st));
        a.val = M->diaBuf;
        M->dia = a;
        M->triples = dia_has_triples(a);
        const long needed = (M->n + static_cast<long>(kWarps) * (32 / M->kp) - 1) /
                            (static_cast<long>(kWarps) * (32 / M->kp));
        with_group(M->kp, [&](auto kk) -> int {
            constexpr int KP = decltype(kk)::value;
            M->gridD = std::min(
                resident_blocks(reinterpret_cast<const void*>(multi_spmv_dia_kernel<KP, true, true>), kT, 0),
                resident_blocks(reinterpret_cast<const void*>(multi_spmv_dia_kernel<KP, false, true>), kT, 0));
            return CIECU_OK;
        });
        M->gridD = static_cast<int>(std::max<long>(1, std::min<long>(M->gridD, needed)));
        CIECU_TRY(dia_fill_f64(M->A, M->dia, M->diaBuf, st));
        cudaEvent_t e0, e1;
        CIECU_CUDA(cudaEventCreate(&e0));
        CIECU_CUDA(cudaEventCreate(&e1));
        float best[2] = {1e30f, 1e30f};
        cudaError_t e = cudaSuccess;
        for (int variant = 0; variant < 2 && e == cudaSuccess; ++variant) {
            const bool dia = variant == 1;
            launch_multi_residual(M, st, dia, B);
            for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {
                cudaEventRecord(e0, st);
                launch_multi_residual(M, st, dia, B);
                cudaEventRecord(e1, st);
                e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best[variant]) best[variant] = ms;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "multi: SpMM format choice");
        M->useDia = M->formatPin == 1 ? true : (M->formatPin == 0 ? false : best[1] < best[0]);
        return CIECU_OK;
    }
    if (M->diaBuf) CIECU_TRY(dia_fill_f64(M->A, M->dia, M->diaBuf, st));
    if (M->formatPin >= 0) M->useDia = M->diaBuf && M->formatPin == 1;
    return CIECU_OK;
}

int build_multi_graph(ciecu_multi_s* M) {
    if (M->graph) return CIECU_OK;
    cudaStream_t st = M->A->space->stream;
    if (device_loop_enabled()) {
        const int status = build_while_graph(st, [&](cudaGraph_t, cudaGraphConditionalHandle cond) {
            return launch_multi_iteration<true>(M, st, cond);
        }, &M->graph);
        if (status == CIECU_OK) {
            M->deviceLoop = true;
            return CIECU_OK;
        }
        cudaGetLastError();
    }
    M->deviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int status = CIECU_OK;
    for (int i = 0; i < M->chunk && status == CIECU_OK; ++i) status = launch_multi_iteration<false>(M, st, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "multi-rhs graph capture");
    e = cudaGraphInstantiate(&M->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "multi-rhs graph instantiate");
    return CIECU_OK;
}

// T of the refined form (INIT: the set-up residual of every column) in the
// format of the FP64 solve.
template <bool INIT>
int launch_true_residual(ciecu_multi_s* M, cudaStream_t st, const double* B) {
    return with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        if (M->quad && M->useDia && M->triples)
            multi_true_residual_quad_kernel<DiaArgs<double>, INIT, true><<<M->gridQD3, kT, 0, st>>>(
                M->dia, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else if (M->quad && M->useDia)
            multi_true_residual_quad_kernel<DiaArgs<double>, INIT><<<M->gridQD, kT, 0, st>>>(
                M->dia, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else if (M->quad)
            multi_true_residual_quad_kernel<CsrArgs<double>, INIT><<<M->gridQ, kT, 0, st>>>(
                M->A->args<double>(), M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else if (M->useDia && M->k == KP)
            multi_true_residual_dia_kernel<KP, true, INIT><<<M->gridD, kT, 0, st>>>(
                M->dia, M->k, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else if (M->useDia)
            multi_true_residual_dia_kernel<KP, false, INIT><<<M->gridD, kT, 0, st>>>(
                M->dia, M->k, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else if (M->k == KP)
            multi_true_residual_kernel<KP, true, INIT><<<M->grid, kT, 0, st>>>(
                M->A->args<double>(), M->k, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        else
            multi_true_residual_kernel<KP, false, INIT><<<M->grid, kT, 0, st>>>(
                M->A->args<double>(), M->k, M->x, B, M->dinv32, M->r32, M->d_s, M->d_g, M->d_partials, M->d_counter);
        return CIECU_OK;
    });
}

CsrArgs<float> args32(const ciecu_multi_s* M) {
    const CsrArgs<double> a = M->A->args<double>();
    return CsrArgs<float>{a.rowptr, a.col, M->val32, a.nrows, a.nnz, a.blocks, a.nblocks, a.mask, a.threshold,
                          a.aligned16};
}

template <bool COND>
int launch_multi_iteration32(ciecu_multi_s* M, cudaStream_t st, cudaGraph_t root, cudaGraphConditionalHandle cond) {
    cudaGraphConditionalHandle replace = 0;
    if (COND) CIECU_CUDA(cudaGraphConditionalHandleCreate(&replace, root, 0, cudaGraphCondAssignDefault));
    CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        if (M->quad && M->useDia && M->triples)
            multi_spmv_quad3_f32_kernel<COND><<<M->gridQ32D3, kT, 0, st>>>(
                M->diaF, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->quad && M->useDia)
            multi_spmv_quad_kernel<DiaArgs<float>, float, COND><<<M->gridQ32D, kT, 0, st>>>(
                M->diaF, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->quad)
            multi_spmv_quad_kernel<CsrArgs<float>, float, COND><<<M->gridQ32, kT, 0, st>>>(
                args32(M), M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->useDia && M->k == KP)
            multi_spmv32_dia_kernel<KP, true, COND><<<M->grid32D, kT, 0, st>>>(
                M->diaF, M->k, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->useDia)
            multi_spmv32_dia_kernel<KP, false, COND><<<M->grid32D, kT, 0, st>>>(
                M->diaF, M->k, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else if (M->k == KP)
            multi_spmv32_kernel<KP, true, COND><<<M->grid32, kT, 0, st>>>(
                args32(M), M->k, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        else
            multi_spmv32_kernel<KP, false, COND><<<M->grid32, kT, 0, st>>>(
                args32(M), M->k, M->p32, M->q32, M->d_s, M->d_g, M->d_partials, M->d_counter, cond);
        multi_update32_kernel<KP, COND><<<M->gridV, kT, 0, st>>>(M->n, M->k, M->x32, M->r32, M->p32, M->q32,
                                                                  M->dinv32, M->d_s, M->d_g, M->d_partials,
                                                                  M->d_counter, replace);
        return CIECU_OK;
    }));
    auto replacement = [&](cudaStream_t s2) -> int {
        CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
            constexpr int KP = decltype(kk)::value;
            multi_fold32_kernel<KP><<<M->gridV, kT, 0, s2>>>(M->n, M->k, M->x, M->x32, M->d_s, M->d_g);
            return CIECU_OK;
        }));
        return launch_true_residual<false>(M, s2, M->graphB);
    };
    if (COND)
        CIECU_TRY(capture_if(st, M->side, replace, replacement));
    else
        CIECU_TRY(replacement(st));
    CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        multi_direction32_kernel<KP, COND><<<M->gridV, kT, 0, st>>>(M->n, M->k, M->p32, M->r32, M->dinv32, M->d_s,
                                                                    M->d_g, cond);
        return CIECU_OK;
    }));
    CIECU_CHECK_LAUNCH("multi-rhs refined iteration");
    return CIECU_OK;
}

// The FP32 copies of the refined form, refreshed from the FP64 arrays at every
// solve (the caller may change the values between solves): D^-1, and the matrix
// in the format of the FP64 solve (the DIA copy or the CSR values).
int prepare32(ciecu_multi_s* M, cudaStream_t st) {
    const size_t count = std::max<size_t>(1, static_cast<size_t>(M->n) * M->k) + 4;
    cudaError_t e = cudaSuccess;
    if (!M->x32) {
        for (float** v : {&M->x32, &M->r32, &M->p32, &M->q32})
            if (e == cudaSuccess) e = cudaMalloc(v, sizeof(float) * count);
        if (e == cudaSuccess) e = cudaMalloc(&M->dinv32, sizeof(float) * (static_cast<size_t>(M->n) + 4));
        if (e == cudaSuccess && !M->side) e = cudaStreamCreateWithFlags(&M->side, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "multi: FP32 blocks");
        with_group(M->kp, [&](auto kk) -> int {
            constexpr int KP = decltype(kk)::value;
            const long needed = (M->n + static_cast<long>(kWarps) * (32 / KP) - 1) / (static_cast<long>(kWarps) * (32 / KP));
            M->grid32 = static_cast<int>(std::max<long>(1, std::min<long>(needed, std::min(
                resident_blocks(reinterpret_cast<const void*>(multi_spmv32_kernel<KP, true, true>), kT, 0),
                resident_blocks(reinterpret_cast<const void*>(multi_spmv32_kernel<KP, false, true>), kT, 0)))));
            M->grid32D = static_cast<int>(std::max<long>(1, std::min<long>(needed, std::min(
                resident_blocks(reinterpret_cast<const void*>(multi_spmv32_dia_kernel<KP, true, true>), kT, 0),
                resident_blocks(reinterpret_cast<const void*>(multi_spmv32_dia_kernel<KP, false, true>), kT, 0)))));
            return CIECU_OK;
        });
    }
    if (M->n > 0) {
        multi_to_f32_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, M->dinv, M->dinv32);
        count_launch();
    }
    if (M->useDia) {
        if (!M->dia32) {
            DiaArgs<float> a{};
            a.nrows = M->dia.nrows;
            a.ndiag = M->dia.ndiag;
            a.ld = M->dia.ld;
            for (int d = 0; d < kMaxDiagonals; ++d) a.off[d] = M->dia.off[d];
            const size_t bytes = sizeof(float) * static_cast<size_t>(a.ndiag) * static_cast<size_t>(a.ld);
            e = cudaMalloc(&M->dia32, bytes);
            if (e == cudaSuccess) e = cudaMemsetAsync(M->dia32, 0, bytes, st);
            if (e != cudaSuccess) return cuda_fail(e, "multi: FP32 diagonal copy");
            a.val = M->dia32;
            M->diaF = a;
        }
        CIECU_TRY(dia_fill_f32(M->A, M->diaF, M->dia32, nullptr, st));
    } else {
        if (!M->val32) {
            e = cudaMalloc(&M->val32, sizeof(float) * std::max<size_t>(1, static_cast<size_t>(M->A->nnz)));
            if (e != cudaSuccess) return cuda_fail(e, "multi: FP32 values");
        }
        if (M->A->nnz > 0) {
            multi_to_f32_kernel<<<grid_for(M->A->nnz, kT, 8), kT, 0, st>>>(M->A->nnz, static_cast<const double*>(M->A->val),
                                                                    M->val32);
            count_launch();
        }
    }
    CIECU_CHECK_LAUNCH("multi: FP32 copies");
    return CIECU_OK;
}

int build_multi_graph32(ciecu_multi_s* M, const double* B) {
    if (M->graph32 && M->graphB == B) return CIECU_OK;
    if (M->graph32) {
        cudaGraphExecDestroy(M->graph32);
        M->graph32 = nullptr;
    }
    M->graphB = B;
    cudaStream_t st = M->A->space->stream;
    if (device_loop_enabled()) {
        const int status = build_while_graph(st, [&](cudaGraph_t root, cudaGraphConditionalHandle cond) {
            return launch_multi_iteration32<true>(M, st, root, cond);
        }, &M->graph32);
        if (status == CIECU_OK) {
            M->deviceLoop32 = true;
            return CIECU_OK;
        }
        cudaGetLastError();
    }
    M->deviceLoop32 = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int status = CIECU_OK;
    for (int i = 0; i < M->chunk && status == CIECU_OK; ++i) status = launch_multi_iteration32<false>(M, st, nullptr, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "multi-rhs refined graph capture");
    e = cudaGraphInstantiate(&M->graph32, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "multi-rhs refined graph instantiate");
    return CIECU_OK;
}

// The solve of the refined form: set-up residual, P = D^-1 R, then the graph
// until every column is done; the column state lands in s.
int refined_solve(ciecu_multi_s* M, const double* B, std::vector<ColumnScalars>& s) {
    cudaStream_t st = M->A->space->stream;
    const long count = M->n * M->k;
    MultiGlobal g{};
    g.maxIter = M->settings.iterationCount;
    g.absTol = M->settings.absoluteResidual;
    g.relTol = M->settings.relativeResidual;
    g.delta = M->refineDelta;
    *M->h_g = g;
    CIECU_CUDA(cudaMemcpyAsync(M->d_g, M->h_g, sizeof(MultiGlobal), cudaMemcpyHostToDevice, st));
    CIECU_TRY(prepare_dia(M, st, B));
    CIECU_TRY(prepare32(M, st));
    CIECU_CUDA(cudaMemsetAsync(M->x32, 0, sizeof(float) * count, st));
    CIECU_CUDA(cudaMemsetAsync(M->p32, 0, sizeof(float) * count, st));
    CIECU_TRY(launch_true_residual<true>(M, st, B));
    CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        multi_direction32_kernel<KP, false><<<M->gridV, kT, 0, st>>>(M->n, M->k, M->p32, M->r32, M->dinv32, M->d_s,
                                                                     M->d_g, 0);
        return CIECU_OK;
    }));
    count_launch(2);
    CIECU_CHECK_LAUNCH("multi-rhs refined set-up");
    CIECU_TRY(build_multi_graph32(M, B));
    const long long limit = M->deviceLoop32 ? 4096 : M->chunk;
    for (;;) {
        CIECU_CUDA(cudaMemcpyAsync(M->h_g, M->d_g, sizeof(MultiGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (M->h_g->finished >= static_cast<unsigned>(M->k)) break;
        const long long before = M->h_g->replacements;
        M->h_g->chunkIter = 0;
        M->h_g->chunkLimit = limit;
        CIECU_CUDA(cudaMemcpyAsync(&M->d_g->chunkIter, &M->h_g->chunkIter, 2 * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaGraphLaunch(M->graph32, st));
        CIECU_CUDA(cudaMemcpyAsync(M->h_g, M->d_g, sizeof(MultiGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        count_launch(M->deviceLoop32 ? 3LL * M->h_g->chunkIter + 2LL * (M->h_g->replacements - before)
                                     : 5LL * M->chunk);
        if (M->h_g->finished >= static_cast<unsigned>(M->k)) break;
    }
    CIECU_CUDA(cudaMemcpyAsync(s.data(), M->d_s, sizeof(ColumnScalars) * M->k, cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    return CIECU_OK;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_multi_create(ciecu_csr lhs, int rhsCount, const double* d_inverseDiagonal, ciecu_statistics settings,
                       ciecu_multi* out) {
    CIECU_REQUIRE(lhs && out && d_inverseDiagonal, "multi_create: null argument");
    CIECU_REQUIRE(lhs->valueType == CIECU_F64 && lhs->rows == lhs->cols, "multi_create: square FP64 matrix expected");
    CIECU_REQUIRE(rhsCount >= 1 && rhsCount <= 32, "multi_create: 1 to 32 right-hand sides");
    auto* M = new ciecu_multi_s();
    M->A = lhs;
    M->dinv = d_inverseDiagonal;
    M->settings = settings;
    M->n = lhs->rows;
    M->k = rhsCount;
    while (M->kp < rhsCount) M->kp <<= 1;
    cudaStream_t st = lhs->space->stream;
    const size_t count = std::max<size_t>(1, static_cast<size_t>(M->n) * M->k);
    cudaError_t e = cudaSuccess;
    for (double** v : {&M->x, &M->r, &M->p, &M->q})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(double) * count);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_s, sizeof(ColumnScalars) * 32);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_g, sizeof(MultiGlobal));
    if (e == cudaSuccess) e = cudaMallocHost(&M->h_g, sizeof(MultiGlobal));
    const long needed = (M->n + static_cast<long>(kWarps) * (32 / M->kp) - 1) / (static_cast<long>(kWarps) * (32 / M->kp));
    with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        M->grid = std::min(resident_blocks(reinterpret_cast<const void*>(multi_spmv_kernel<KP, true, true>), kT, 0),
                           resident_blocks(reinterpret_cast<const void*>(multi_spmv_kernel<KP, false, true>), kT, 0));
        M->gridV = resident_blocks(reinterpret_cast<const void*>(multi_update_kernel<KP>), kT, 0);
        return CIECU_OK;
    });
    M->grid = static_cast<int>(std::max<long>(1, std::min<long>(M->grid, needed)));
    M->gridV = static_cast<int>(std::max<long>(1, std::min<long>(M->gridV, needed)));
    // partial sums for the widest grid of any kernel of either form (the DIA and
    // FP32 grids are fixed later, at most their resident blocks), so that the
    // buffer captured by a graph is never replaced
    if (M->k == 32) {
        const long rowsQ = (M->n + kWarps * kQuadRows - 1) / (kWarps * kQuadRows);
        auto fit = [&](const void* k, long need) {
            return static_cast<int>(std::max<long>(1, std::min<long>(need, resident_blocks(k, kT, 0))));
        };
        const long blocks = std::max<long>(1, lhs->nblocks);
        M->gridQ = fit(reinterpret_cast<const void*>(multi_spmv_quad_kernel<CsrArgs<double>, double, true>), blocks);
        M->gridQD = fit(reinterpret_cast<const void*>(multi_spmv_quad_kernel<DiaArgs<double>, double, true>), rowsQ);
        M->gridQ32 = fit(reinterpret_cast<const void*>(multi_spmv_quad_kernel<CsrArgs<float>, float, true>), blocks);
        M->gridQ32D = fit(reinterpret_cast<const void*>(multi_spmv_quad_kernel<DiaArgs<float>, float, true>), rowsQ);
        const long rows3 = (M->n + kWarps * 16 - 1) / (kWarps * 16);
        M->gridQD3 = fit(reinterpret_cast<const void*>(multi_spmv_quad_kernel<DiaArgs<double>, double, true, true>),
                         rows3);
        M->gridQ32D3 = fit(reinterpret_cast<const void*>(multi_spmv_quad3_f32_kernel<true>),
                           rows3);
        M->quad = quad_enabled();
    }
    int widest = std::max({M->grid, M->gridV, M->gridQ, M->gridQD, M->gridQ32, M->gridQ32D, M->gridQD3,
                           M->gridQ32D3});
    with_group(M->kp, [&](auto kk) -> int {
        constexpr int KP = decltype(kk)::value;
        for (const void* k : {reinterpret_cast<const void*>(multi_spmv_dia_kernel<KP, true, true>),
                              reinterpret_cast<const void*>(multi_spmv_dia_kernel<KP, false, true>),
                              reinterpret_cast<const void*>(multi_spmv32_kernel<KP, true, true>),
                              reinterpret_cast<const void*>(multi_spmv32_kernel<KP, false, true>),
                              reinterpret_cast<const void*>(multi_spmv32_dia_kernel<KP, true, true>),
                              reinterpret_cast<const void*>(multi_spmv32_dia_kernel<KP, false, true>)})
            widest = std::max(widest, resident_blocks(k, kT, 0));
        return CIECU_OK;
    });
    if (e == cudaSuccess) e = cudaMalloc(&M->d_partials, sizeof(double) * 2 * 32 * widest);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_counter, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_counter, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_s, 0, sizeof(ColumnScalars) * 32, st);
    if (e != cudaSuccess) {
        ciecu_multi_destroy(M);
        return cuda_fail(e, "multi_create: allocation");
    }
    *out = M;
    return CIECU_OK;
}

int ciecu_multi_destroy(ciecu_multi M) {
    if (!M) return CIECU_OK;
    if (M->graph) cudaGraphExecDestroy(M->graph);
    cudaFree(M->x);
    cudaFree(M->r);
    cudaFree(M->p);
    cudaFree(M->q);
    cudaFree(M->d_s);
    cudaFree(M->d_g);
    if (M->h_g) cudaFreeHost(M->h_g);
    cudaFree(M->d_partials);
    cudaFree(M->d_counter);
    cudaFree(M->diaBuf);
    if (M->graph32) cudaGraphExecDestroy(M->graph32);
    if (M->side) cudaStreamDestroy(M->side);
    for (float* v : {M->x32, M->r32, M->p32, M->q32, M->dinv32, M->val32, M->dia32}) cudaFree(v);
    delete M;
    return CIECU_OK;
}

int ciecu_multi_info(ciecu_multi M, int* lanesPerRow, int* deviceLoop) {
    CIECU_REQUIRE(M, "multi_info: null solver");
    if (lanesPerRow) *lanesPerRow = M->quad ? kQuadLanes : M->kp;
    if (deviceLoop) *deviceLoop = M->deviceLoop ? 1 : 0;
    return CIECU_OK;
}

int ciecu_multi_set_refinement(ciecu_multi M, double delta) {
    CIECU_REQUIRE(M, "multi_set_refinement: null solver");
    CIECU_REQUIRE(delta == 0.0 || (delta > 0.0 && delta < 1.0), "multi_set_refinement: delta must be 0 or in (0, 1)");
    M->refineDelta = delta;
    return CIECU_OK;
}

int ciecu_multi_refinements(ciecu_multi M, int64_t* h_perColumn) {
    CIECU_REQUIRE(M && h_perColumn, "multi_refinements: null argument");
    for (int c = 0; c < M->k; ++c)
        h_perColumn[c] = c < static_cast<int>(M->last.size()) ? M->last[c].refinements : 0;
    return CIECU_OK;
}

int ciecu_multi_set_format(ciecu_multi M, int format) {
    CIECU_REQUIRE(M, "multi_set_format: null solver");
    CIECU_REQUIRE(format >= -1 && format <= 1, "multi_set_format: format must be -1 (timed), 0 (CSR) or 1 (DIA)");
    M->formatPin = format;
    if (format == 1 && !M->diaBuf) M->diaChecked = false;  // build the copy at the next solve
    if (format >= 0) {
        if (M->graph) {
            cudaGraphExecDestroy(M->graph);
            M->graph = nullptr;
        }
        if (M->graph32) {
            cudaGraphExecDestroy(M->graph32);
            M->graph32 = nullptr;
        }
    }
    return CIECU_OK;
}

int ciecu_multi_format(ciecu_multi M, int* diagonals) {
    CIECU_REQUIRE(M && diagonals, "multi_format: null argument");
    *diagonals = M->useDia ? M->dia.ndiag : 0;
    return CIECU_OK;
}

int ciecu_multi_product(ciecu_multi M, double inScale, const double* d_in, double outScale, double* d_out,
                        ciecu_statistics* h_stats) {
    CIECU_REQUIRE(M && d_in && d_out, "multi_product: null argument");
    // the k = 32 kernels read the right-hand sides in 16-byte vectors
    if (M->k == 32) {
        const bool want = quad_enabled() && reinterpret_cast<std::uintptr_t>(d_in) % 16 == 0;
        if (want != M->quad) {
            M->quad = want;
            for (cudaGraphExec_t* gr : {&M->graph, &M->graph32})
                if (*gr) {
                    cudaGraphExecDestroy(*gr);
                    *gr = nullptr;
                }
        }
    }
    cudaStream_t st = M->A->space->stream;
    const long n = M->n;
    const long count = n * M->k;
    CIECU_CUDA(cudaMemcpyAsync(M->x, d_out, sizeof(double) * count, cudaMemcpyDeviceToDevice, st));
    std::vector<ColumnScalars> s(static_cast<size_t>(M->k));
    if (M->settings.iterationCount > 0 && M->refineDelta > 0.0) {
        CIECU_TRY(refined_solve(M, d_in, s));
    } else if (M->settings.iterationCount > 0) {
        MultiGlobal g{};
        g.maxIter = M->settings.iterationCount;
        g.absTol = M->settings.absoluteResidual;
        g.relTol = M->settings.relativeResidual;
        *M->h_g = g;
        CIECU_CUDA(cudaMemcpyAsync(M->d_g, M->h_g, sizeof(MultiGlobal), cudaMemcpyHostToDevice, st));
        CIECU_TRY(prepare_dia(M, st, d_in));
        CIECU_TRY(launch_multi_residual(M, st, M->useDia, d_in));
        CIECU_TRY(with_group(M->kp, [&](auto kk) -> int {
            constexpr int KP = decltype(kk)::value;
            multi_init_kernel<KP><<<M->gridV, kT, 0, st>>>(n, M->k, M->r, M->dinv, M->p, M->d_s, M->d_g,
                                                          M->d_partials, M->d_counter);
            return CIECU_OK;
        }));
        count_launch();
        CIECU_CHECK_LAUNCH("multi-rhs set-up");
        CIECU_TRY(build_multi_graph(M));
        const long long limit = M->deviceLoop ? 4096 : M->chunk;
        for (;;) {
            CIECU_CUDA(cudaMemcpyAsync(M->h_g, M->d_g, sizeof(MultiGlobal), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            if (M->h_g->finished >= static_cast<unsigned>(M->k)) break;
            M->h_g->chunkIter = 0;
            M->h_g->chunkLimit = limit;
            CIECU_CUDA(cudaMemcpyAsync(&M->d_g->chunkIter, &M->h_g->chunkIter, 2 * sizeof(long long),
                                       cudaMemcpyHostToDevice, st));
            CIECU_CUDA(cudaGraphLaunch(M->graph, st));
            CIECU_CUDA(cudaMemcpyAsync(M->h_g, M->d_g, sizeof(MultiGlobal), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            count_launch(3LL * (M->deviceLoop ? M->h_g->chunkIter : M->chunk));
            if (M->h_g->finished >= static_cast<unsigned>(M->k)) break;
        }
        CIECU_CUDA(cudaMemcpyAsync(s.data(), M->d_s, sizeof(ColumnScalars) * M->k, cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
    }
    multi_output_kernel<<<grid_for(count, kT, 8), kT, 0, st>>>(count, inScale, outScale, M->x, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("multi_output_kernel");
    CIECU_CUDA(cudaStreamSynchronize(st));
    M->last = s;
    int firstError = -1;
    for (int c = 0; c < M->k; ++c) {
        const ColumnScalars& sc = s[c];
        if (h_stats) {
            if (M->settings.iterationCount > 0)
                h_stats[c] = ciecu_statistics{sc.done == 3 ? sc.errorIter : sc.iter, sc.absres, sc.relres};
            else
                h_stats[c] = ciecu_statistics{0, 1.7976931348623157e308, 1.7976931348623157e308};
        }
        if (sc.done == 3 && firstError < 0) firstError = c;
    }
    if (firstError >= 0) {
        const ColumnScalars& sc = s[firstError];
        return fail(CIECU_ERR_BREAKDOWN,
                    "right-hand side " + std::to_string(firstError) + ": " +
                        (sc.errorKind == 1 ? std::string("preconditioned norm vanished in iteration 0 (r^T @ z = 0)")
                                           : "p^T @ A @ p vanished in iteration " + std::to_string(sc.errorIter)));
    }
    return CIECU_OK;
}

}  // extern "C"
