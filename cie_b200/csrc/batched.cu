// Batched Jacobi-preconditioned CG: many independent SPD systems of different
// sizes solved together, each with its own scalars and stopping test
// (ConjugateGradients_impl.hpp:49-201 per system; the reference runs one solver
// object per system).
//
// The systems are one block-diagonal CSR matrix: system s owns rows and columns
// rowOffsets[s] .. rowOffsets[s+1]-1.  The rows are cut into tiles of at most
// kTileRows rows that never cross a system, so one CTA handles one tile at a
// time and every tile belongs to exactly one system.  A dot product of system s
// is reduced deterministically: each tile writes its partial, and the last of the
// system's tiles to finish (a per-system ticket) sums them in tile order and
// forms the system's alpha / beta / stopping decision.  Tiles of finished systems
// return at once, so the work shrinks as systems converge.
//
// One iteration = three kernels over all systems (K1 SpMV + p^T q, K2 update +
// dots + decision, K3 direction), run by the same device-side graph loop as the
// single-system solver; K3 ends the loop when every system is finished.
#include "graph.cuh"
#include "pcg.cuh"
#include "ciecu_batch.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <vector>

namespace ciecu {
namespace {

constexpr int kT = 256;
constexpr int kTileRows = 2048;

struct BatchScalars {
    double rz, pq, alpha, beta, rr, r0, absres, relres;
    long long iter;
    int done;   // 0 running, 1 converged, 2 iteration limit, 3 breakdown
    int errorKind;  // 1: r^T z <= 0 at start, 2: p^T A p <= 0
    long long errorIter;
    // reliable-update form: state of the system's FP32 recursion
    double maxrx, maxrr;  // largest FP32 residual norm since the last x / r replacement
    double rzPending;
    long long refinements;
    int pending;  // a replacement is due at the end of this iteration
    int updateX;
    int restart;  // an FP32 breakdown: no step, direction restarted after the replacement
    int breakdowns;
};

struct BatchGlobal {
    unsigned finished;   // systems that are done
    unsigned pad;
    long long chunkIter, chunkLimit;
    long long maxIter;
    double absTol, relTol;
    int badColumn;       // an entry outside its system's block (set-up check)
    int pad2;
    // reliable-update form
    double delta;           // replacement trigger
    unsigned anyPending;    // some system asked for a replacement in this iteration
    unsigned ctaDone;       // CTAs of the current kernel that finished (last-CTA decision)
    long long replacements; // launches of the replacement pair that had work
};

// FP32 breakdowns a system may recover from by a replacement with a restarted
// direction before it reports the breakdown.
constexpr int kMaxSystemBreakdowns = 64;

struct Tile {
    int system;
    int rowBegin, rowEnd;
    int slot;  // position among the system's tiles
};

template <bool COND>
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle cond, unsigned value) {
    if constexpr (COND) cudaGraphSetConditional(cond, value);
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Tile-level reduction of K values; the CTA holding the system's last tile gets
// the system totals (in tile order) in every thread and returns true.
template <int K>
__device__ __forceinline__ bool system_reduce_last(const double (&mine)[K], const Tile& t, const int* tileBegin,
                                                   const int* tileCount, double* partials, unsigned* counter,
                                                   double (&out)[K]) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double sums[K];
#pragma unroll
    for (int k = 0; k < K; ++k) sums[k] = block_sum<double, kT>(mine[k], s_red);
    const int first = tileBegin[t.system];
    const int count = tileCount[t.system];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[static_cast<long>(first + t.slot) * K + k] = sums[k];
        __threadfence();
        const unsigned ticket = atomicAdd(&counter[t.system], 1u);
        s_last = ticket == static_cast<unsigned>(count - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double acc = 0.0;
        const volatile double* p = partials;
        for (int j = threadIdx.x; j < count; j += kT) acc += p[static_cast<long>(first + j) * K + k];
        out[k] = block_sum<double, kT>(acc, s_red);
    }
    if (threadIdx.x == 0) counter[t.system] = 0u;
    return true;
}

// Rows [rb, re) of the tile: VS lanes per row, the CTA's warps striding over rows.
template <int VS, typename T, typename Op>
__device__ __forceinline__ void tile_rows(const CsrArgs<T>& A, int rb, int re, const T* __restrict__ x, Op& op) {
    constexpr int RPW = 32 / VS;
    constexpr int UNROLL = VS <= 4 ? 8 : 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sub = lane % VS, slot = lane / VS;
    for (int base = rb + warp * RPW; base < re; base += (kT / 32) * RPW) {
        const int r = base + slot;
        const bool valid = r < re;
        typename Op::Pre pre{};
        if (valid && sub == 0) pre = op.pre(r);
        T sum = T(0);
        if (valid) {
            const int k1 = A.rowptr[r + 1];
            for (int k = A.rowptr[r] + sub; k < k1; k += UNROLL * VS) {
                T v[UNROLL];
                int c[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) {
                    const int kk = k + u * VS;
                    const bool in = kk < k1;
                    v[u] = in ? stream_ld(A.val + kk) : T(0);
                    c[u] = in ? stream_ld(A.col + kk) : -1;
                }
                T xv[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : T(0);
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) sum = fma(v[u], xv[u], sum);
            }
        }
#pragma unroll
        for (int offset = VS / 2; offset > 0; offset >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, offset, VS);
        if (valid && sub == 0) op.post(r, pre, sum);
    }
}

template <typename T>
struct PqOp {
    using Pre = T;
    const T* __restrict__ p;
    T* __restrict__ q;
    double acc;
    __device__ __forceinline__ T pre(int r) const { return p[r]; }
    __device__ __forceinline__ void post(int r, T pr, T sum) {
        q[r] = sum;
        acc = fma(static_cast<double>(pr), static_cast<double>(sum), acc);
    }
};

// Set-up check: every entry of row r lies in the column block of r's system.
__global__ void batch_check_kernel(CsrArgs<double> A, const Tile* __restrict__ tiles, int ntiles,
                                   const long long* __restrict__ rowOffsets, BatchGlobal* g) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tile = tiles[t];
        const long long c0 = rowOffsets[tile.system], c1 = rowOffsets[tile.system + 1];
        for (int r = tile.rowBegin + threadIdx.x; r < tile.rowEnd; r += kT)
            for (int k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k)
                if (A.col[k] < c0 || A.col[k] >= c1) atomicMin(&g->badColumn, r);
    }
}

// r = b - A x is formed before; z = D^-1 r, p = z, rr, rz and the initial test.
// Systems preset to done = 4 (skipped: already converged in the outer FP64
// refinement) take no work.
template <typename T>
__global__ void __launch_bounds__(kT) batch_init_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                        const int* tileBegin, const int* tileCount,
                                                        const T* __restrict__ r, const T* __restrict__ dinv,
                                                        T* __restrict__ p, BatchScalars* S, BatchGlobal* g,
                                                        double* partials, unsigned* counter) {
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        if (S[t.system].done == 4) continue;
        double rr = 0.0, rz = 0.0;
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) {
            const T ri = r[i];
            const T zi = ri * dinv[i];
            p[i] = zi;
            rr = fma(static_cast<double>(ri), static_cast<double>(ri), rr);
            rz = fma(static_cast<double>(ri), static_cast<double>(zi), rz);
        }
        double mine[2] = {rr, rz}, tot[2];
        if (system_reduce_last<2>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0) {
            BatchScalars& s = S[t.system];
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
        __syncthreads();
    }
}

// K1: q = A p and p^T q per system; alpha.
// RELIABLE (the reliable-update form): an FP32 breakdown takes no step and asks
// for a replacement with a restarted direction, up to kMaxSystemBreakdowns.
// Five CTAs per SM (at most 51 registers, against 60 and four CTAs by the
// compiler's own choice): over the 512 Q2 systems 970 -> 958 ms in FP64 and
// 887 -> 842 ms in FP32 with reliable updates on one B200; three CTAs (71
// registers) measured 1.11 s.
template <int VS, typename T, bool RELIABLE = false>
__global__ void __launch_bounds__(kT, 5) batch_spmv_kernel(CsrArgs<T> A, const Tile* __restrict__ tiles, int ntiles,
                                                        const int* tileBegin, const int* tileCount,
                                                        const T* __restrict__ p, T* __restrict__ q,
                                                        BatchScalars* S, BatchGlobal* g, double* partials,
                                                        unsigned* counter) {
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        if (*reinterpret_cast<volatile int*>(&S[t.system].done)) continue;
        PqOp<T> op{p, q, 0.0};
        tile_rows<VS>(A, t.rowBegin, t.rowEnd, p, op);
        double mine[1] = {op.acc}, tot[1];
        if (system_reduce_last<1>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0) {
            BatchScalars& s = S[t.system];
            s.pq = tot[0];
            if (RELIABLE && !(0.0 < tot[0]) && s.breakdowns < kMaxSystemBreakdowns) {
                s.alpha = 0.0;
                s.restart = 1;
                s.breakdowns += 1;
            } else if (!(0.0 < tot[0])) {
                s.done = 3;
                s.errorKind = 2;
                s.errorIter = s.iter;
                atomicAdd(&g->finished, 1u);
            } else {
                s.alpha = s.rz / tot[0];
            }
        }
        __syncthreads();
    }
}

// K2: x += alpha p; r -= alpha q; rr, rz; beta and the stopping test per system.
template <typename T>
__global__ void __launch_bounds__(kT) batch_update_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                          const int* tileBegin, const int* tileCount,
                                                          T* __restrict__ x, T* __restrict__ r,
                                                          const T* __restrict__ p, const T* __restrict__ q,
                                                          const T* __restrict__ dinv, BatchScalars* S,
                                                          BatchGlobal* g, double* partials, unsigned* counter) {
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        BatchScalars& s = S[t.system];
        if (*reinterpret_cast<volatile int*>(&s.done)) continue;
        const T alpha = static_cast<T>(s.alpha), malpha = -alpha;
        double rr = 0.0, rz = 0.0;
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) {
            x[i] = fma(alpha, p[i], x[i]);
            const T ri = fma(malpha, q[i], r[i]);
            r[i] = ri;
            rr = fma(static_cast<double>(ri), static_cast<double>(ri), rr);
            rz = fma(static_cast<double>(ri), static_cast<double>(ri * dinv[i]), rz);
        }
        double mine[2] = {rr, rz}, tot[2];
        if (system_reduce_last<2>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0) {
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
        __syncthreads();
    }
}

// K3: p = beta p + z (the rounding of space.scale + space.add, as the single
// solver); ends the loop when every system is finished.
template <typename T, bool COND>
__global__ void __launch_bounds__(kT) batch_direction_kernel(const Tile* __restrict__ tiles, int ntiles, int systems,
                                                             T* __restrict__ p, const T* __restrict__ r,
                                                             const T* __restrict__ dinv,
                                                             const BatchScalars* S, BatchGlobal* g,
                                                             cudaGraphConditionalHandle cond) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g->chunkIter += 1;
        const bool more = *reinterpret_cast<volatile unsigned*>(&g->finished) < static_cast<unsigned>(systems);
        set_loop<COND>(cond, (more && g->chunkIter < g->chunkLimit) ? 1u : 0u);
    }
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        const BatchScalars& s = S[t.system];
        if (*reinterpret_cast<const volatile int*>(&s.done)) continue;
        const T beta = static_cast<T>(s.beta);
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT)
            p[i] = add_rn(mul_rn(p[i], beta), mul_rn(r[i], dinv[i]));
    }
}

// ---- reliable-update form: FP32 iterations, FP64 residual replacements ------
//
// Per system the iteration of the mixed-precision solver: K1 (batch_spmv_kernel
// on the FP32 copy, RELIABLE: an FP32 breakdown restarts instead of failing);
// K2 x32 += alpha p32, r32 -= alpha q32, the FP32 recursion's r^T r and r^T z in
// FP64 and the replacement decision (FP32 residual norm below delta times its
// maximum since the last replacement, below the stopping tolerance, or the
// iteration limit); when any system asks, F folds x32 into the FP64 solution
// and T recomputes r = b - A64 x64 in FP64 for those systems (float(r) kept),
// with the FP64 stopping test; K3 p32 = D^-1 r32 + beta p32.

// The last CTA of a kernel to finish (a grid-wide ticket) runs f(); CTAs call
// this once, after all their work.
template <typename F>
__device__ __forceinline__ void last_cta(BatchGlobal* g, F&& f) {
    __shared__ bool s_lastCta;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_lastCta = atomicAdd(&g->ctaDone, 1u) == gridDim.x - 1;
        if (s_lastCta) {
            __threadfence();
            g->ctaDone = 0u;
            f();
        }
    }
}

template <bool COND>
__global__ void __launch_bounds__(kT) batch_update_rel_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                              const int* tileBegin, const int* tileCount,
                                                              float* __restrict__ x, float* __restrict__ r,
                                                              const float* __restrict__ p, const float* __restrict__ q,
                                                              const float* __restrict__ dinv, BatchScalars* S,
                                                              BatchGlobal* g, double* partials, unsigned* counter,
                                                              cudaGraphConditionalHandle replace) {
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        BatchScalars& s = S[t.system];
        if (*reinterpret_cast<volatile int*>(&s.done)) continue;
        const bool step = !s.restart;
        const float alpha = static_cast<float>(s.alpha), malpha = -alpha;
        double rr = 0.0, rz = 0.0;
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) {
            float ri = r[i];
            if (step) {
                x[i] = fmaf(alpha, p[i], x[i]);
                ri = fmaf(malpha, q[i], ri);
                r[i] = ri;
            }
            rr = fma(static_cast<double>(ri), static_cast<double>(ri), rr);
            rz = fma(static_cast<double>(ri), static_cast<double>(ri * dinv[i]), rz);
        }
        double mine[2] = {rr, rz}, tot[2];
        if (system_reduce_last<2>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0) {
            const double rnorm = sqrt(tot[0]);
            s.iter += 1;
            if (rnorm > s.maxrx) s.maxrx = rnorm;
            if (rnorm > s.maxrr) s.maxrr = rnorm;
            const bool updateX = rnorm < g->delta * s.maxrx;
            const bool update = updateX || rnorm < g->delta * s.maxrr || rnorm < g->relTol * s.r0 ||
                                rnorm < g->absTol || s.iter >= g->maxIter || s.restart;
            s.updateX = updateX ? 1 : 0;
            if (update) {
                s.pending = 1;
                s.rzPending = tot[1];
                atomicOr(&g->anyPending, 1u);
            } else {
                s.beta = tot[1] / s.rz;
                s.rz = tot[1];
            }
        }
        __syncthreads();
    }
    last_cta(g, [&] { set_loop<COND>(replace, *reinterpret_cast<volatile unsigned*>(&g->anyPending) ? 1u : 0u); });
}

// F: x64 += x32, x32 = 0 on the rows of systems with a replacement due.
__global__ void __launch_bounds__(kT) batch_fold_rel_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                            double* __restrict__ x64, float* __restrict__ x32,
                                                            const BatchScalars* S, const BatchGlobal* g) {
    if (!*reinterpret_cast<const volatile unsigned*>(&g->anyPending)) return;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        if (!S[t.system].pending) continue;
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) {
            x64[i] += static_cast<double>(x32[i]);
            x32[i] = 0.0f;
        }
    }
}

// T: r = b - A64 x64 in FP64, r32 = float(r), ||r||^2 in FP64 and r32^T z32.
struct TrueResidualOp {
    struct Pre {
        double b;
        float d;
    };
    const double* __restrict__ b;
    const float* __restrict__ dinv;
    float* __restrict__ r32;
    double rr, rz;
    __device__ __forceinline__ Pre pre(int i) const { return Pre{b[i], dinv[i]}; }
    __device__ __forceinline__ void post(int i, const Pre& pr, double sum) {
        const double ri = pr.b - sum;
        const float rf = static_cast<float>(ri);
        r32[i] = rf;
        rr = fma(ri, ri, rr);
        rz = fma(static_cast<double>(rf), static_cast<double>(rf * pr.d), rz);
    }
};

template <bool INIT>
__device__ __forceinline__ void system_replace(BatchScalars& s, const double (&tot)[2], BatchGlobal* g) {
    const double rnorm = sqrt(tot[0]);
    if (INIT) {
        s = BatchScalars{};
        s.rr = tot[0];
        s.r0 = rnorm;
        s.absres = rnorm;
        s.relres = 1.0;
        s.maxrx = s.maxrr = rnorm;
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

template <int VS, bool INIT>
__global__ void __launch_bounds__(kT) batch_true_residual_kernel(CsrArgs<double> A, const Tile* __restrict__ tiles,
                                                                 int ntiles, const int* tileBegin,
                                                                 const int* tileCount, const double* __restrict__ b,
                                                                 const double* __restrict__ x64,
                                                                 const float* __restrict__ dinv,
                                                                 float* __restrict__ r32, BatchScalars* S,
                                                                 BatchGlobal* g, double* partials,
                                                                 unsigned* counter) {
    if (!INIT && !*reinterpret_cast<volatile unsigned*>(&g->anyPending)) return;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        BatchScalars& s = S[t.system];
        if (!INIT && (s.done || !s.pending)) continue;
        TrueResidualOp op{b, dinv, r32, 0.0, 0.0};
        tile_rows<VS>(A, t.rowBegin, t.rowEnd, x64, op);
        double mine[2] = {op.rr, op.rz}, tot[2];
        if (system_reduce_last<2>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0)
            system_replace<INIT>(s, tot, g);
        __syncthreads();
    }
    if (!INIT)
        last_cta(g, [&] {
            g->anyPending = 0u;
            g->replacements += 1;
        });
}

// K3 of the reliable-update form: p32 = D^-1 r32 + beta p32 (beta = 0: a new
// direction, the old one may not be finite after a breakdown); ends the loop
// when every system is finished.
template <bool COND>
__global__ void __launch_bounds__(kT) batch_direction_rel_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                                 int systems, float* __restrict__ p,
                                                                 const float* __restrict__ r,
                                                                 const float* __restrict__ dinv,
                                                                 const BatchScalars* S, BatchGlobal* g,
                                                                 cudaGraphConditionalHandle cond) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g->chunkIter += 1;
        const bool more = *reinterpret_cast<volatile unsigned*>(&g->finished) < static_cast<unsigned>(systems);
        set_loop<COND>(cond, (more && g->chunkIter < g->chunkLimit) ? 1u : 0u);
    }
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        const BatchScalars& s = S[t.system];
        if (*reinterpret_cast<const volatile int*>(&s.done)) continue;
        const float beta = static_cast<float>(s.beta);
        if (beta == 0.0f)
            for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) p[i] = r[i] * dinv[i];
        else
            for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) p[i] = fmaf(beta, p[i], r[i] * dinv[i]);
    }
}

__global__ void batch_output_kernel(long n, double inScale, double outScale, const double* __restrict__ x,
                                    double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
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

// Calls f(std::integral_constant<int, VS>) for VS in {2, 4, 8, 16, 32}.
template <typename F>
int with_lanes(int vs, F&& f) {
    switch (vs) {
        case 2: return f(std::integral_constant<int, 2>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        default: return f(std::integral_constant<int, 4>{});
    }
}

}  // namespace
}  // namespace ciecu

namespace ciecu {
namespace {

// Comparison::less with the default tolerances (Comparison_impl.hpp:32-63), on the host.
bool host_float_less(double a, double b) {
    const double norm = std::fmin(std::fabs(a) + std::fabs(b), std::numeric_limits<double>::max());
    const double tol = std::fmax(std::numeric_limits<double>::min(), std::numeric_limits<double>::epsilon() * norm);
    return a < b && !(std::fabs(a - b) < tol);
}

// FP64 residual norms per system (outer refinement): norm2[s] = ||r_s||^2.
__global__ void __launch_bounds__(kT) batch_norm_kernel(const Tile* __restrict__ tiles, int ntiles,
                                                        const int* tileBegin, const int* tileCount,
                                                        const double* __restrict__ r, double* __restrict__ norm2,
                                                        double* partials, unsigned* counter) {
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const Tile t = tiles[ti];
        double rr = 0.0;
        for (int i = t.rowBegin + threadIdx.x; i < t.rowEnd; i += kT) rr = fma(r[i], r[i], rr);
        double mine[1] = {rr}, tot[1];
        if (system_reduce_last<1>(mine, t, tileBegin, tileCount, partials, counter, tot) && threadIdx.x == 0)
            norm2[t.system] = tot[0];
        __syncthreads();
    }
}

__global__ void batch_to_f32_kernel(long n, const double* __restrict__ a, float* __restrict__ b) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        b[i] = static_cast<float>(a[i]);
}

// x64 += x32 (the correction of one refinement round)
__global__ void batch_fold_kernel(long n, double* __restrict__ x64, const float* __restrict__ x32) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        x64[i] += static_cast<double>(x32[i]);
}

// One precision of the batched iteration: the matrix values, the vectors, the
// tuned lanes per row and the graph of the loop.
template <typename T>
struct Level {
    CsrArgs<T> A{};
    const T* dinv = nullptr;
    T *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
    int lanes = 4;
    cudaGraphExec_t graph = nullptr;
    bool deviceLoop = false;
};

}  // namespace
}  // namespace ciecu

struct ciecu_batch_s {
    ciecu_csr_s* A = nullptr;
    ciecu_statistics settings{};
    long n = 0;
    int systems = 0, ntiles = 0;
    ciecu::Tile* d_tiles = nullptr;
    int* d_tileBegin = nullptr;
    int* d_tileCount = nullptr;
    long long* d_rowOffsets = nullptr;
    ciecu::Level<double> f64;
    ciecu::Level<float> f32;  // FP32 inner level of the refined solve (allocated by set_refinement)
    float* val32 = nullptr;
    float* dinv32 = nullptr;
    double* norm2 = nullptr;  // per-system ||r||^2 of the outer refinement
    double innerTolerance = 0.0;  // > 0: FP32 inner solves with FP64 refinement
    double reliableDelta = 0.0;   // > 0: FP32 iterations with FP64 reliable updates (takes precedence)
    cudaGraphExec_t relGraph = nullptr;
    bool relDeviceLoop = false;
    const double* relB = nullptr;  // right-hand side the reliable-update graph reads
    cudaStream_t side = nullptr;   // captures the IF body of the replacement
    std::vector<long long> lastRefinements;  // FP64 replacements per system in the last reliable-update solve
    ciecu::BatchScalars* d_s = nullptr;
    ciecu::BatchGlobal* d_g = nullptr;
    ciecu::BatchGlobal* h_g = nullptr;
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    int chunk = 16;
    int grid = 1;
};

namespace ciecu {
namespace {

template <typename T, bool COND>
int launch_batch_iteration(ciecu_batch_s* B, Level<T>& L, cudaStream_t st, cudaGraphConditionalHandle cond) {
    CIECU_TRY(with_lanes(L.lanes, [&](auto v) -> int {
        constexpr int VS = decltype(v)::value;
        batch_spmv_kernel<VS, T><<<B->grid, kT, 0, st>>>(L.A, B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount,
                                                         L.p, L.q, B->d_s, B->d_g, B->d_partials, B->d_counter);
        return CIECU_OK;
    }));
    batch_update_kernel<T><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount, L.x, L.r,
                                                   L.p, L.q, L.dinv, B->d_s, B->d_g, B->d_partials, B->d_counter);
    batch_direction_kernel<T, COND><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->systems, L.p, L.r, L.dinv,
                                                            B->d_s, B->d_g, cond);
    CIECU_CHECK_LAUNCH("batched pcg iteration");
    return CIECU_OK;
}

template <typename T>
int build_batch_graph(ciecu_batch_s* B, Level<T>& L) {
    if (L.graph) return CIECU_OK;
    cudaStream_t st = B->A->space->stream;
    if (device_loop_enabled()) {
        const int status = build_while_graph(st, [&](cudaGraph_t, cudaGraphConditionalHandle cond) {
            return launch_batch_iteration<T, true>(B, L, st, cond);
        }, &L.graph);
        if (status == CIECU_OK) {
            L.deviceLoop = true;
            return CIECU_OK;
        }
        cudaGetLastError();
    }
    L.deviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int status = CIECU_OK;
    for (int i = 0; i < B->chunk && status == CIECU_OK; ++i) status = launch_batch_iteration<T, false>(B, L, st, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "batched graph capture");
    e = cudaGraphInstantiate(&L.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "batched graph instantiate");
    return CIECU_OK;
}

// Times K1 for each lane count on the level's buffers (p = D^-1 > 0, every
// system running) and keeps the fastest.
template <typename T>
int tune_batch(ciecu_batch_s* B, Level<T>& L) {
    cudaStream_t st = B->A->space->stream;
    std::vector<BatchScalars> scratch(B->systems);
    for (auto& s : scratch) {
        s = BatchScalars{};
        s.rz = 1.0;
    }
    CIECU_CUDA(cudaMemcpyAsync(B->d_s, scratch.data(), sizeof(BatchScalars) * B->systems, cudaMemcpyHostToDevice, st));
    CIECU_CUDA(cudaMemcpyAsync(L.p, L.dinv, sizeof(T) * B->n, cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0, e1;
    CIECU_CUDA(cudaEventCreate(&e0));
    CIECU_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestLanes = 4;
    cudaError_t e = cudaSuccess;
    const double avg = B->n > 0 ? static_cast<double>(B->A->nnz) / B->n : 0.0;
    for (int vs : {2, 4, 8, 16, 32}) {
        if (vs >= 16 && avg < vs) continue;
        auto launch = [&]() {
            with_lanes(vs, [&](auto v) -> int {
                constexpr int VS = decltype(v)::value;
                batch_spmv_kernel<VS, T><<<B->grid, kT, 0, st>>>(L.A, B->d_tiles, B->ntiles, B->d_tileBegin,
                                                                 B->d_tileCount, L.p, L.q, B->d_s, B->d_g,
                                                                 B->d_partials, B->d_counter);
                return CIECU_OK;
            });
        };
        launch();
        for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {
            cudaEventRecord(e0, st);
            for (int rep = 0; rep < 3; ++rep) launch();
            cudaEventRecord(e1, st);
            e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms < best) {
                best = ms;
                bestLanes = vs;
            }
        }
        count_launch(10);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batched pcg: autotune");
    L.lanes = bestLanes;
    return CIECU_OK;
}

// One batched PCG solve on level L from x = 0 (or the level's current x) for
// every system whose scalars are not preset to done = 4; the right-hand side is
// in L.r on entry (it becomes the residual).  Returns when every system is done.
template <typename T>
int run_level(ciecu_batch_s* B, Level<T>& L, const BatchGlobal& g0, unsigned preset) {
    cudaStream_t st = B->A->space->stream;
    *B->h_g = g0;
    B->h_g->finished = preset;
    CIECU_CUDA(cudaMemcpyAsync(B->d_g, B->h_g, sizeof(BatchGlobal), cudaMemcpyHostToDevice, st));
    batch_init_kernel<T><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount, L.r, L.dinv,
                                                 L.p, B->d_s, B->d_g, B->d_partials, B->d_counter);
    count_launch();
    CIECU_CHECK_LAUNCH("batch_init_kernel");
    CIECU_TRY(build_batch_graph(B, L));
    const long long limit = L.deviceLoop ? 4096 : B->chunk;
    for (;;) {
        CIECU_CUDA(cudaMemcpyAsync(B->h_g, B->d_g, sizeof(BatchGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (B->h_g->finished >= static_cast<unsigned>(B->systems)) break;
        B->h_g->chunkIter = 0;
        B->h_g->chunkLimit = limit;
        CIECU_CUDA(cudaMemcpyAsync(&B->d_g->chunkIter, &B->h_g->chunkIter, 2 * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaGraphLaunch(L.graph, st));
        CIECU_CUDA(cudaMemcpyAsync(B->h_g, B->d_g, sizeof(BatchGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        count_launch(3LL * (L.deviceLoop ? B->h_g->chunkIter : B->chunk));
        if (B->h_g->finished >= static_cast<unsigned>(B->systems)) break;
    }
    return CIECU_OK;
}

// FP32 copies of the matrix values and of D^-1 and the FP32 vectors (first use),
// with the lane count of their SpMV tuned.
int ensure_f32(ciecu_batch_s* B) {
    if (B->val32) return CIECU_OK;
    cudaStream_t st = B->A->space->stream;
    const size_t n = static_cast<size_t>(std::max<long>(1, B->n));
    cudaError_t e = cudaMalloc(&B->val32, sizeof(float) * std::max<long>(1, B->A->nnz));
    if (e == cudaSuccess) e = cudaMalloc(&B->dinv32, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&B->norm2, sizeof(double) * B->systems);
    for (float** v : {&B->f32.x, &B->f32.r, &B->f32.p, &B->f32.q})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(float) * n);
    if (e == cudaSuccess && B->A->nnz > 0) {
        batch_to_f32_kernel<<<grid_for(B->A->nnz, kT, 8), kT, 0, st>>>(
            B->A->nnz, static_cast<const double*>(B->A->val), B->val32);
        batch_to_f32_kernel<<<grid_for(B->n, kT, 8), kT, 0, st>>>(B->n, B->f64.dinv, B->dinv32);
        count_launch(2);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "batched pcg: FP32 copies");
    B->f32.A = CsrArgs<float>{B->A->rowptr, B->A->col, B->val32, B->A->rows, B->A->nnz, B->A->d_blocks,
                              B->A->nblocks, nullptr, 0, B->A->aligned16};
    B->f32.dinv = B->dinv32;
    return tune_batch(B, B->f32);
}

template <bool INIT>
int launch_true_residual(ciecu_batch_s* B, cudaStream_t st, const double* b) {
    return with_lanes(B->f64.lanes, [&](auto v) -> int {
        constexpr int VS = decltype(v)::value;
        batch_true_residual_kernel<VS, INIT><<<B->grid, kT, 0, st>>>(
            B->f64.A, B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount, b, B->f64.x, B->dinv32, B->f32.r,
            B->d_s, B->d_g, B->d_partials, B->d_counter);
        return CIECU_OK;
    });
}

template <bool COND>
int launch_reliable_iteration(ciecu_batch_s* B, cudaStream_t st, cudaGraph_t root, cudaGraphConditionalHandle cond) {
    Level<float>& F = B->f32;
    cudaGraphConditionalHandle replace = 0;
    if (COND) CIECU_CUDA(cudaGraphConditionalHandleCreate(&replace, root, 0, cudaGraphCondAssignDefault));
    CIECU_TRY(with_lanes(F.lanes, [&](auto v) -> int {
        constexpr int VS = decltype(v)::value;
        batch_spmv_kernel<VS, float, true><<<B->grid, kT, 0, st>>>(F.A, B->d_tiles, B->ntiles, B->d_tileBegin,
                                                                   B->d_tileCount, F.p, F.q, B->d_s, B->d_g,
                                                                   B->d_partials, B->d_counter);
        return CIECU_OK;
    }));
    batch_update_rel_kernel<COND><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount, F.x,
                                                          F.r, F.p, F.q, F.dinv, B->d_s, B->d_g, B->d_partials,
                                                          B->d_counter, replace);
    auto replacement = [&](cudaStream_t s2) -> int {
        batch_fold_rel_kernel<<<B->grid, kT, 0, s2>>>(B->d_tiles, B->ntiles, B->f64.x, F.x, B->d_s, B->d_g);
        return launch_true_residual<false>(B, s2, B->relB);
    };
    if (COND)
        CIECU_TRY(capture_if(st, B->side, replace, replacement));
    else
        CIECU_TRY(replacement(st));
    batch_direction_rel_kernel<COND><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->systems, F.p, F.r, F.dinv,
                                                             B->d_s, B->d_g, cond);
    CIECU_CHECK_LAUNCH("batched reliable-update iteration");
    return CIECU_OK;
}

int build_reliable_graph(ciecu_batch_s* B, const double* b) {
    if (B->relGraph && B->relB == b) return CIECU_OK;
    if (B->relGraph) {
        cudaGraphExecDestroy(B->relGraph);
        B->relGraph = nullptr;
    }
    B->relB = b;
    cudaStream_t st = B->A->space->stream;
    if (!B->side) CIECU_CUDA(cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking));
    if (device_loop_enabled()) {
        const int status = build_while_graph(st, [&](cudaGraph_t root, cudaGraphConditionalHandle cond) {
            return launch_reliable_iteration<true>(B, st, root, cond);
        }, &B->relGraph);
        if (status == CIECU_OK) {
            B->relDeviceLoop = true;
            return CIECU_OK;
        }
        cudaGetLastError();
    }
    B->relDeviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int status = CIECU_OK;
    for (int i = 0; i < B->chunk && status == CIECU_OK; ++i)
        status = launch_reliable_iteration<false>(B, st, nullptr, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "batched reliable-update graph capture");
    e = cudaGraphInstantiate(&B->relGraph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "batched reliable-update graph instantiate");
    return CIECU_OK;
}

// The reliable-update solve from x64 (the initial guesses): the set-up residual
// of every system, p32 = D^-1 r32, then the graph until every system is done.
int reliable_solve(ciecu_batch_s* B, const double* b, const BatchGlobal& g0, std::vector<BatchScalars>& s) {
    cudaStream_t st = B->A->space->stream;
    Level<float>& F = B->f32;
    *B->h_g = g0;
    B->h_g->delta = B->reliableDelta;
    CIECU_CUDA(cudaMemcpyAsync(B->d_g, B->h_g, sizeof(BatchGlobal), cudaMemcpyHostToDevice, st));
    CIECU_CUDA(cudaMemsetAsync(F.x, 0, sizeof(float) * std::max<long>(1, B->n), st));
    CIECU_TRY(launch_true_residual<true>(B, st, b));
    batch_direction_rel_kernel<false><<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->systems, F.p, F.r, F.dinv,
                                                              B->d_s, B->d_g, 0);
    count_launch(2);
    CIECU_CHECK_LAUNCH("batched reliable-update set-up");
    CIECU_TRY(build_reliable_graph(B, b));
    const long long limit = B->relDeviceLoop ? 4096 : B->chunk;
    for (;;) {
        CIECU_CUDA(cudaMemcpyAsync(B->h_g, B->d_g, sizeof(BatchGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (B->h_g->finished >= static_cast<unsigned>(B->systems)) break;
        const long long before = B->h_g->replacements;
        B->h_g->chunkIter = 0;
        B->h_g->chunkLimit = limit;
        CIECU_CUDA(cudaMemcpyAsync(&B->d_g->chunkIter, &B->h_g->chunkIter, 2 * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaGraphLaunch(B->relGraph, st));
        CIECU_CUDA(cudaMemcpyAsync(B->h_g, B->d_g, sizeof(BatchGlobal), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        count_launch(B->relDeviceLoop ? 3LL * B->h_g->chunkIter + 2LL * (B->h_g->replacements - before)
                                      : 5LL * B->chunk);
        if (B->h_g->finished >= static_cast<unsigned>(B->systems)) break;
    }
    CIECU_CUDA(cudaMemcpyAsync(s.data(), B->d_s, sizeof(BatchScalars) * B->systems, cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    return CIECU_OK;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_batch_create(ciecu_csr lhs, int64_t systems, const int64_t* h_rowOffsets, const double* d_inverseDiagonal,
                       ciecu_statistics settings, ciecu_batch* out) {
    CIECU_REQUIRE(lhs && out && h_rowOffsets && d_inverseDiagonal, "batch_create: null argument");
    CIECU_REQUIRE(lhs->valueType == CIECU_F64 && lhs->rows == lhs->cols, "batch_create: square FP64 matrix expected");
    CIECU_REQUIRE(systems >= 1 && systems <= (1 << 24), "batch_create: system count out of range");
    CIECU_REQUIRE(h_rowOffsets[0] == 0 && h_rowOffsets[systems] == lhs->rows,
                  "batch_create: row offsets must start at 0 and end at the row count");
    std::vector<Tile> tiles;
    std::vector<int> tileBegin(static_cast<size_t>(systems)), tileCount(static_cast<size_t>(systems));
    for (int64_t s = 0; s < systems; ++s) {
        CIECU_REQUIRE(h_rowOffsets[s + 1] > h_rowOffsets[s], "batch_create: every system needs at least one row");
        tileBegin[s] = static_cast<int>(tiles.size());
        int slot = 0;
        for (int64_t r = h_rowOffsets[s]; r < h_rowOffsets[s + 1]; r += kTileRows)
            tiles.push_back(Tile{static_cast<int>(s), static_cast<int>(r),
                                 static_cast<int>(std::min<int64_t>(r + kTileRows, h_rowOffsets[s + 1])), slot++});
        tileCount[s] = slot;
    }
    auto* B = new ciecu_batch_s();
    B->A = lhs;
    B->f64.dinv = d_inverseDiagonal;
    B->f64.A = lhs->args<double>();
    B->settings = settings;
    B->n = lhs->rows;
    B->systems = static_cast<int>(systems);
    B->ntiles = static_cast<int>(tiles.size());
    cudaStream_t st = lhs->space->stream;
    const size_t n = static_cast<size_t>(B->n);
    cudaError_t e = cudaMalloc(&B->d_tiles, sizeof(Tile) * tiles.size());
    if (e == cudaSuccess) e = cudaMalloc(&B->d_tileBegin, sizeof(int) * systems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_tileCount, sizeof(int) * systems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_rowOffsets, sizeof(long long) * (systems + 1));
    for (double** v : {&B->f64.x, &B->f64.r, &B->f64.p, &B->f64.q})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(double) * std::max<size_t>(1, n));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_s, sizeof(BatchScalars) * systems);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_g, sizeof(BatchGlobal));
    if (e == cudaSuccess) e = cudaMallocHost(&B->h_g, sizeof(BatchGlobal));
    if (e == cudaSuccess) e = cudaMalloc(&B->d_partials, sizeof(double) * 2 * tiles.size());
    if (e == cudaSuccess) e = cudaMalloc(&B->d_counter, sizeof(unsigned) * systems);
    if (e == cudaSuccess) e = cudaMemsetAsync(B->d_counter, 0, sizeof(unsigned) * systems, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_tileBegin, tileBegin.data(), sizeof(int) * systems, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_tileCount, tileCount.data(), sizeof(int) * systems, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->d_rowOffsets, h_rowOffsets, sizeof(long long) * (systems + 1), cudaMemcpyHostToDevice,
                            st);
    if (e != cudaSuccess) {
        ciecu_batch_destroy(B);
        return cuda_fail(e, "batch_create: allocation");
    }
    // every entry inside its system's block
    BatchGlobal g{};
    g.badColumn = 0x7fffffff;
    e = cudaMemcpyAsync(B->d_g, &g, sizeof(BatchGlobal), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        batch_check_kernel<<<grid_for(B->ntiles * static_cast<long>(kT), kT, 8), kT, 0, st>>>(
            lhs->args<double>(), B->d_tiles, B->ntiles, B->d_rowOffsets, B->d_g);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&g, B->d_g, sizeof(BatchGlobal), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ciecu_batch_destroy(B);
        return cuda_fail(e, "batch_create: block check");
    }
    if (g.badColumn != 0x7fffffff) {
        const int row = g.badColumn;
        ciecu_batch_destroy(B);
        return fail(CIECU_ERR_ARGUMENT, "batch_create: row " + std::to_string(row) +
                                            " has an entry outside its system's column block");
    }
    B->grid = std::max(1, std::min(B->ntiles, resident_blocks(reinterpret_cast<const void*>(
                                                                   batch_spmv_kernel<4, double>), kT, 0)));
    const int status = tune_batch(B, B->f64);
    if (status != CIECU_OK) {
        ciecu_batch_destroy(B);
        return status;
    }
    *out = B;
    return CIECU_OK;
}

int ciecu_batch_destroy(ciecu_batch B) {
    if (!B) return CIECU_OK;
    if (B->f64.graph) cudaGraphExecDestroy(B->f64.graph);
    if (B->f32.graph) cudaGraphExecDestroy(B->f32.graph);
    if (B->relGraph) cudaGraphExecDestroy(B->relGraph);
    if (B->side) cudaStreamDestroy(B->side);
    cudaFree(B->d_tiles);
    cudaFree(B->d_tileBegin);
    cudaFree(B->d_tileCount);
    cudaFree(B->d_rowOffsets);
    for (double* v : {B->f64.x, B->f64.r, B->f64.p, B->f64.q}) cudaFree(v);
    for (float* v : {B->f32.x, B->f32.r, B->f32.p, B->f32.q}) cudaFree(v);
    cudaFree(B->val32);
    cudaFree(B->dinv32);
    cudaFree(B->norm2);
    cudaFree(B->d_s);
    cudaFree(B->d_g);
    if (B->h_g) cudaFreeHost(B->h_g);
    cudaFree(B->d_partials);
    cudaFree(B->d_counter);
    delete B;
    return CIECU_OK;
}

int ciecu_batch_info(ciecu_batch B, int* lanesPerRow, int* deviceLoop, int64_t* tiles) {
    CIECU_REQUIRE(B, "batch_info: null solver");
    // the form the next solve runs: reliable updates (FP32 lanes, its own graph),
    // restarted refinement (FP32 lanes) or FP64
    const bool reliable = B->reliableDelta > 0.0;
    const bool f32 = reliable || B->innerTolerance > 0.0;
    if (lanesPerRow) *lanesPerRow = f32 ? B->f32.lanes : B->f64.lanes;
    if (deviceLoop)
        *deviceLoop = (reliable ? B->relDeviceLoop : (f32 ? B->f32.deviceLoop : B->f64.deviceLoop)) ? 1 : 0;
    if (tiles) *tiles = B->ntiles;
    return CIECU_OK;
}

int ciecu_batch_set_refinement(ciecu_batch B, double innerTolerance) {
    CIECU_REQUIRE(B, "batch_set_refinement: null solver");
    CIECU_REQUIRE(innerTolerance >= 0.0 && innerTolerance < 1.0, "batch_set_refinement: tolerance must be in [0, 1)");
    B->innerTolerance = innerTolerance;
    if (innerTolerance == 0.0) return CIECU_OK;
    return ensure_f32(B);
}

int ciecu_batch_set_reliable_updates(ciecu_batch B, double delta) {
    CIECU_REQUIRE(B, "batch_set_reliable_updates: null solver");
    CIECU_REQUIRE(delta == 0.0 || (delta > 0.0 && delta < 1.0),
                  "batch_set_reliable_updates: delta must be 0 or in (0, 1)");
    B->reliableDelta = delta;
    if (delta == 0.0) return CIECU_OK;
    return ensure_f32(B);
}

int ciecu_batch_refinements(ciecu_batch B, int64_t* h_perSystem) {
    CIECU_REQUIRE(B && h_perSystem, "batch_refinements: null argument");
    for (int i = 0; i < B->systems; ++i)
        h_perSystem[i] = i < static_cast<int>(B->lastRefinements.size()) ? B->lastRefinements[i] : 0;
    return CIECU_OK;
}

int ciecu_batch_product(ciecu_batch B, double inScale, const double* d_in, double outScale, double* d_out,
                        ciecu_statistics* h_stats) {
    CIECU_REQUIRE(B && d_in && d_out, "batch_product: null argument");
    ciecu_csr_s* A = B->A;
    cudaStream_t st = A->space->stream;
    const long n = B->n;
    Level<double>& L = B->f64;
    CIECU_CUDA(cudaMemcpyAsync(L.x, d_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    std::vector<BatchScalars> s(static_cast<size_t>(B->systems));
    std::vector<ciecu_statistics> out(static_cast<size_t>(B->systems),
                                      ciecu_statistics{0, 1.7976931348623157e308, 1.7976931348623157e308});
    std::vector<int> failedKind(static_cast<size_t>(B->systems), 0);
    std::vector<long long> failedIter(static_cast<size_t>(B->systems), 0);
    if (B->settings.iterationCount > 0) {
        BatchGlobal g{};
        g.maxIter = B->settings.iterationCount;
        g.absTol = B->settings.absoluteResidual;
        g.relTol = B->settings.relativeResidual;
        g.badColumn = 0x7fffffff;
        if (B->reliableDelta == 0.0) {
            CIECU_CUDA(cudaMemcpyAsync(L.r, d_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            CIECU_TRY(ciecu_csr_spmv_f64(A, 1.0, L.x, -1.0, L.r));  // r = b - A x0 (block diagonal: per system)
        }
        if (B->reliableDelta > 0.0) {
            CIECU_TRY(reliable_solve(B, d_in, g, s));
            B->lastRefinements.assign(static_cast<size_t>(B->systems), 0);
            for (int i = 0; i < B->systems; ++i) {
                out[i] = ciecu_statistics{s[i].done == 3 ? s[i].errorIter : s[i].iter, s[i].absres, s[i].relres};
                B->lastRefinements[i] = s[i].refinements;
                if (s[i].done == 3) {
                    failedKind[i] = s[i].errorKind;
                    failedIter[i] = s[i].errorIter;
                }
            }
        } else if (B->innerTolerance == 0.0) {
            // FP64: every system runs ConjugateGradients_impl.hpp:49-201 as it is
            CIECU_CUDA(cudaMemsetAsync(B->d_s, 0, sizeof(BatchScalars) * B->systems, st));
            CIECU_TRY(run_level(B, L, g, 0u));
            CIECU_CUDA(cudaMemcpyAsync(s.data(), B->d_s, sizeof(BatchScalars) * B->systems, cudaMemcpyDeviceToHost,
                                       st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            for (int i = 0; i < B->systems; ++i) {
                out[i] = ciecu_statistics{s[i].done == 3 ? s[i].errorIter : s[i].iter, s[i].absres, s[i].relres};
                if (s[i].done == 3) {
                    failedKind[i] = s[i].errorKind;
                    failedIter[i] = s[i].errorIter;
                }
            }
        } else {
            // FP32 inner solves, FP64 refinement: each round solves A32 c = float(r) to
            // innerTolerance for the systems not yet converged, x += c, r = b - A x in FP64;
            // a system stops on its true FP64 residual (Comparison::less against the
            // absolute or the relative limit, relative to its initial residual).
            Level<float>& F = B->f32;
            std::vector<double> r0(static_cast<size_t>(B->systems)), nrm(static_cast<size_t>(B->systems));
            std::vector<int> state(static_cast<size_t>(B->systems), 0);  // 0 running, 1 converged, 2 limit, 3 failed
            std::vector<long long> used(static_cast<size_t>(B->systems), 0);
            BatchGlobal gi = g;
            gi.relTol = B->innerTolerance;
            gi.absTol = 0.0;
            for (int round = 0;; ++round) {
                batch_norm_kernel<<<B->grid, kT, 0, st>>>(B->d_tiles, B->ntiles, B->d_tileBegin, B->d_tileCount, L.r,
                                                           B->norm2, B->d_partials, B->d_counter);
                count_launch();
                CIECU_CHECK_LAUNCH("batch_norm_kernel");
                CIECU_CUDA(cudaMemcpyAsync(nrm.data(), B->norm2, sizeof(double) * B->systems,
                                           cudaMemcpyDeviceToHost, st));
                CIECU_CUDA(cudaStreamSynchronize(st));
                unsigned preset = 0;
                for (int i = 0; i < B->systems; ++i) {
                    const double absres = std::sqrt(nrm[i]);
                    if (round == 0) r0[i] = absres;
                    const double relres = r0[i] > 0.0 ? absres / r0[i] : 0.0;
                    if (state[i] == 0) {
                        out[i] = ciecu_statistics{used[i], absres, relres};
                        if (host_float_less(absres, g.absTol) || host_float_less(relres, g.relTol)) state[i] = 1;
                        else if (used[i] >= g.maxIter) state[i] = 2;
                    }
                    s[i] = BatchScalars{};
                    if (state[i] != 0) {
                        s[i].done = 4;
                        ++preset;
                    }
                }
                if (preset == static_cast<unsigned>(B->systems)) break;
                long long budget = g.maxIter;
                for (int i = 0; i < B->systems; ++i)
                    if (state[i] == 0) budget = std::min(budget, g.maxIter - used[i]);
                gi.maxIter = std::max<long long>(1, budget);
                CIECU_CUDA(cudaMemcpyAsync(B->d_s, s.data(), sizeof(BatchScalars) * B->systems, cudaMemcpyHostToDevice,
                                           st));
                batch_to_f32_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, L.r, F.r);
                CIECU_CUDA(cudaMemsetAsync(F.x, 0, sizeof(float) * n, st));
                count_launch();
                CIECU_TRY(run_level(B, F, gi, preset));
                batch_fold_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, L.x, F.x);
                count_launch();
                CIECU_CUDA(cudaMemcpyAsync(L.r, d_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
                CIECU_TRY(ciecu_csr_spmv_f64(A, 1.0, L.x, -1.0, L.r));
                std::vector<BatchScalars> si(static_cast<size_t>(B->systems));
                CIECU_CUDA(cudaMemcpyAsync(si.data(), B->d_s, sizeof(BatchScalars) * B->systems,
                                           cudaMemcpyDeviceToHost, st));
                CIECU_CUDA(cudaStreamSynchronize(st));
                for (int i = 0; i < B->systems; ++i) {
                    if (state[i] != 0) continue;
                    used[i] += si[i].done == 3 ? si[i].errorIter : si[i].iter;
                    if (si[i].done == 3 && si[i].iter == 0 && si[i].errorIter == 0) {
                        state[i] = 3;  // no progress possible in FP32
                        failedKind[i] = si[i].errorKind;
                        failedIter[i] = used[i];
                    }
                }
            }
        }
    }
    batch_output_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, inScale, outScale, L.x, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("batch_output_kernel");
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (h_stats)
        for (int i = 0; i < B->systems; ++i) h_stats[i] = out[i];
    for (int i = 0; i < B->systems; ++i)
        if (failedKind[i])
            return fail(CIECU_ERR_BREAKDOWN,
                        "system " + std::to_string(i) + ": " +
                            (failedKind[i] == 1 ? std::string("preconditioned norm vanished in iteration 0 (r^T @ z = 0)")
                                                : "p^T @ A @ p vanished in iteration " + std::to_string(failedIter[i])));
    return CIECU_OK;
}

}  // extern "C"
