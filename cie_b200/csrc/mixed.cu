// Mixed-precision Jacobi-PCG: FP32 inner iterations, FP64 refinement.
//
// No reference counterpart (the reference solves in one precision,
// ConjugateGradients_impl.hpp:49-201); the inner iteration is that algorithm in
// FP32 and the FP64 part is defect correction:
//
//   FP64 (kept on the GPU only here): the solution x64, the residual
//        r = b - A64 x64 recomputed with the FP64 matrix, and every dot-product
//        accumulator (the FP32 vectors are reduced in double).
//   FP32: the matrix values (a converted copy in the SELL-32 layout of sell.cuh:
//        one thread per row, every load warp-coalesced), the vectors r, p, q,
//        x-increment and the inverse diagonal.  Column indices are stored as
//        16-bit offsets from the row (col - row) when the matrix bandwidth allows
//        -- a lossless, checked re-encoding of the int32 CSR that halves the
//        index bytes (int32 otherwise).
//
// mode 0 (reliable updates; Sleijpen & van der Vorst 1996, the residual
//   replacement used for mixed-precision CG by Clark et al. 2010): whenever the
//   FP32 residual norm has dropped below delta times its maximum since the last
//   replacement, or claims convergence, the FP32 increment is folded into x64,
//   r is recomputed in FP64 and replaces the FP32 residual; the search direction
//   is kept, so the Krylov space is not restarted.
// mode 1 (classic iterative refinement): the inner CG is restarted (p = z)
//   after every correction; a correction is triggered when the FP32 residual has
//   dropped by delta relative to the start of the inner solve.
//
// The solve stops only on the TRUE FP64 residual: ||b - A64 x64|| <= tol ||r0||.
//
// One inner iteration = 3 kernels (M1 SpMV+p^T q, M2 update+dots+decision,
// M3 direction), 2 when the direction is formed inside M1 (fuseDirection 1), or
// 1 over the DIA copy (fuseDirection 2, mixed_single_dia_kernel); the two
// refinement kernels (R1 fold, R2 FP64 residual) are in the same CUDA graph and
// return at once unless a replacement was asked for.
#include "ciecu_mixed.h"
#include "graph.cuh"
#include "pcg.cuh"
#include "sell.cuh"
#include "dia.cuh"
#include "sell_tma.cuh"

#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>
#include <tuple>
#include <mutex>
#include <map>

namespace ciecu {
namespace {

constexpr int kT = 256;
constexpr int kDiaInner = -2;  // innerKernel / unroll code of the DIA inner kernels


struct MixedScalars {
    double rz, pq, alpha, beta, rzPending;
    double r0, absres, relres, rnorm;  // true residual norms
    double sloppy;                      // FP32 residual norm of the last iteration
    double maxrx, maxrr, cycleStart;
    double absTol, relTol, delta;
    long long iter, maxIter, refinements;
    int done, error, update, updateX, mode, pad;
    long long chunkIter, chunkLimit;  // iterations of the current graph launch / per launch
    unsigned tmaError;                // a bounded TMA pipeline wait gave up
    int scaled;                       // inner system symmetrically Jacobi-scaled
    double r0s;                       // initial residual norm in the inner (scaled) units
    int restart;                      // an FP32 breakdown asked for a replacement + restart
    int breakdowns;                   // FP32 breakdowns of this solve
};

// FP32 breakdowns (p^T q <= 0 in the inner precision) a solve survives by a
// residual replacement and a restarted direction before it reports a breakdown.
constexpr int kMaxInnerBreakdowns = 64;

// M1 epilogue: alpha, or -- when the FP32 p^T q is not positive -- no step, and a
// residual replacement with a restarted direction (up to kMaxInnerBreakdowns).
__device__ __forceinline__ bool inner_breakdown(MixedScalars* s) {
    s->alpha = 0.0;
    s->restart = 1;
    s->breakdowns += 1;
    if (s->breakdowns <= kMaxInnerBreakdowns) return false;
    s->done = 3;
    s->error = CIECU_ERR_BREAKDOWN;
    return true;
}

// COND selects the instantiation with conditional-node calls (device loop) or
// without any (plain captured graphs, profilable).
template <bool COND>
__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle cond, unsigned value) {
    if constexpr (COND) cudaGraphSetConditional(cond, value);
}


// ---- SELL-32 FP32 matrix ------------------------------------------------------

// Padded length of each 32-row slice; negative when its rows differ in length.
__global__ void sell_len_kernel(int nrows, const int* __restrict__ rowptr, int* __restrict__ sliceLen,
                                unsigned* tooLong) {
    const int nslices = (nrows + 31) >> 5;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nslices; s += gridDim.x * blockDim.x) {
        int mx = 0, mn = 0x7fffffff;
        for (int r = s << 5; r < min(nrows, (s << 5) + 32); ++r) {
            const int len = rowptr[r + 1] - rowptr[r];
            mx = max(mx, len);
            mn = min(mn, len);
        }
        if (mx > 65535) atomicOr(tooLong, 1u);
        sliceLen[s] = (mn == mx) ? mx : -mx;
    }
}

// Copies row r into its slice (values in FP32, columns as 16-bit row offsets or
// int32) and zero-fills its padding; layout of sell.cuh.
template <typename CI>
__global__ void sell_fill_kernel(int nrows, const int* __restrict__ rowptr, const int* __restrict__ col,
                                 const double* __restrict__ val, const int* __restrict__ sliceLen,
                                 const long long* __restrict__ sliceStart, float* __restrict__ sval,
                                 CI* __restrict__ scol, unsigned short* __restrict__ rowLen, unsigned* tooFar,
                                 const double* __restrict__ sdiag) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
        const int s = r >> 5;
        const int padded = ((abs(sliceLen[s]) + 3) >> 2) << 2;
        const int k0 = rowptr[r], len = rowptr[r + 1] - k0;
        rowLen[r] = static_cast<unsigned short>(len);
        const long long base = sliceStart[s] + 4 * (r & 31);
        for (int j = 0; j < padded; ++j) {
            const long long idx = base + 128LL * (j >> 2) + (j & 3);
            if (j < len) {
                const int c = col[k0 + j];
                sval[idx] = static_cast<float>(sdiag ? val[k0 + j] * sdiag[r] * sdiag[c] : val[k0 + j]);
                if constexpr (sizeof(CI) == 2) {
                    const int off = c - r;
                    if (off < -32768 || off > 32767) atomicOr(tooFar, 1u);
                    scol[idx] = static_cast<CI>(off);
                } else {
                    scol[idx] = c;
                }
            } else {
                sval[idx] = 0.0f;
                scol[idx] = sizeof(CI) == 2 ? CI(0) : static_cast<CI>(r);
            }
        }
    }
}

// out = A32 in (the inner operator on its own).
struct StoreOp {
    using Pre = NoPre;
    float* __restrict__ y;
    __device__ __forceinline__ NoPre pre(int) const { return NoPre{}; }
    __device__ __forceinline__ void post(int r, NoPre, float sum) const { y[r] = sum; }
};

template <int U, typename CI>
__global__ void __launch_bounds__(kT) mixed_apply_kernel(SellArgs<float, CI> A, const float* __restrict__ x,
                                                         float* __restrict__ y) {
    StoreOp op{y};
    sell_rows<U, float, float, CI>(A, x, op);
}

// M1: q = A32 p, p^T q (FP64 accumulation), alpha.
struct MixedPqOp {
    using Pre = float;
    const float* __restrict__ p;
    float* __restrict__ q;
    double acc;
    __device__ __forceinline__ float pre(int r) const { return p[r]; }
    __device__ __forceinline__ void post(int r, float pr, float sum) {
        q[r] = sum;
        acc = fma(static_cast<double>(pr), static_cast<double>(sum), acc);
    }
};

// M1 of the fused form (options.fuseDirection): w = A32 z with z = D^-1 r kept as
// a vector, then on the own rows p = z + beta p and q = w + beta q (the search
// direction and its product by recurrence; p = z, q = w after a restart,
// beta = 0), p^T q.  One vector is gathered, and the separate direction pass
// over p, r and D^-1 is gone.
struct MixedDirOp {
    struct Pre {
        float z, p, q;
    };
    const float* __restrict__ z;
    float* __restrict__ p;
    float* __restrict__ q;
    float beta;
    bool restart;
    double acc;
    __device__ __forceinline__ Pre pre(int r) const {
        return restart ? Pre{z[r], 0.0f, 0.0f} : Pre{z[r], p[r], q[r]};
    }
    __device__ __forceinline__ void post(int r, const Pre& pr, float sum) {
        const float pn = restart ? pr.z : fmaf(beta, pr.p, pr.z);
        const float qn = restart ? sum : fmaf(beta, pr.q, sum);
        p[r] = pn;
        q[r] = qn;
        acc = fma(static_cast<double>(pn), static_cast<double>(qn), acc);
    }
};

// The M1 epilogue of either form: q = A32 p (plain: the gathered vector is p) or
// the recurrences above (fused: the gathered vector is z).
template <bool FUSED>
struct M1Op;
template <>
struct M1Op<false> {
    using Type = MixedPqOp;
    static __device__ __forceinline__ MixedPqOp make(const float* x, float* p, float* q, const MixedScalars*) {
        (void)p;
        return MixedPqOp{x, q, 0.0};
    }
};
template <>
struct M1Op<true> {
    using Type = MixedDirOp;
    static __device__ __forceinline__ MixedDirOp make(const float* z, float* p, float* q, const MixedScalars* s) {
        const double beta = *reinterpret_cast<const volatile double*>(&s->beta);
        return MixedDirOp{z, p, q, static_cast<float>(beta), beta == 0.0, 0.0};
    }
};

template <int U, typename CI, bool COND, bool FUSED>
__global__ void __launch_bounds__(kT) mixed_spmv_kernel(SellArgs<float, CI> A, const float* __restrict__ x,
                                                        float* __restrict__ p, float* __restrict__ q, MixedScalars* s,
                                                        double* partials, unsigned* counter,
                                                        cudaGraphConditionalHandle loop) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond<COND>(loop, 0);
        return;
    }
    auto op = M1Op<FUSED>::make(x, p, q, s);
    sell_rows<U, float, float, CI>(A, x, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (!(0.0 < tot[0])) {
            if (inner_breakdown(s)) set_cond<COND>(loop, 0);
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// DIA variants of the two kernels above, for inner matrices of at most 32
// diagonals (dia.cuh): FP32 values only, no column indices.  The full copy is read
// even when it is symmetric: reading the lower half back from the upper one (as
// the FP64 PCG does) measured slower here, where every row pass is already a
// four-row, 16-byte-load stream.
// TRIPLES: the offsets come in consecutive triples (dia_rows4_triples).
template <int ND, bool TRIPLES, typename Op>
__device__ __forceinline__ void mixed_dia_rows(const DiaArgs<float>& A, const float* __restrict__ x, Op& op) {
    if constexpr (TRIPLES)
        dia_rows4_triples<ND>(A, x, op);
    else
        dia_rows4<ND>(A, x, op);
}

template <int ND, bool TRIPLES>
__global__ void __launch_bounds__(kT) mixed_apply_dia_kernel(DiaArgs<float> A, const float* __restrict__ x,
                                                            float* __restrict__ y) {
    StoreOp op{y};
    mixed_dia_rows<ND, TRIPLES>(A, x, op);
}

// M1 over the DIA copy and M2 (below) run three CTAs per SM with up to 85
// registers (the compiler's own choice: 60 and 64 registers, four CTAs): the
// 128^3 mixed solve measured 28.3 -> 26.3 ms with the same iterations.
template <int ND, bool COND, bool FUSED, bool TRIPLES>
__global__ void __launch_bounds__(kT, 3) mixed_spmv_dia_kernel(DiaArgs<float> A, const float* __restrict__ x,
                                                           float* __restrict__ p, float* __restrict__ q,
                                                           MixedScalars* s, double* partials, unsigned* counter,
                                                           cudaGraphConditionalHandle loop) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond<COND>(loop, 0);
        return;
    }
    auto op = M1Op<FUSED>::make(x, p, q, s);
    mixed_dia_rows<ND, TRIPLES>(A, x, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (!(0.0 < tot[0])) {
            if (inner_breakdown(s)) set_cond<COND>(loop, 0);
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// ---- single-pass inner iteration (options.fuseDirection == 2, DIA inner matrix) ----
//
// One kernel per inner iteration instead of two or three.  Kernel k+1 receives
// alpha_k and beta_{k+1} and, for its own rows,
//   x += alpha_k p_k,  r_{k+1} = r_k - alpha_k q_k,  z = D^-1 r_{k+1},
//   p_{k+1} = z + beta_{k+1} p_k,  q_{k+1} = A32 p_{k+1};
// the operand entries p_{k+1}[j] of the row sums are formed the same way from the
// gathered r_k[j], q_k[j], p_k[j], D^-1[j] (bit for bit the values the owning row
// stores).  beta_{k+1} = rho_{k+1} / rho_k needs rho_{k+1} = r_{k+1}^T D^-1 r_{k+1}
// before r_{k+1} exists; with r_{k+1} = r_k - alpha_k q_k it is the quadratic
//   rho_{k+1} = (r_k^T D^-1 r_k) - 2 alpha_k (r_k^T D^-1 q_k) + alpha_k^2 (q_k^T D^-1 q_k),
// whose three sums (and the three of ||r_{k+1}||^2) kernel k reduces in FP64
// beside p_k^T q_k.  alpha_k = rho_k / p_k^T q_k uses the rho of the stored FP32
// r_k, as the three-kernel form does; beta and the replacement decision use the
// expansion, which differs from the FP32-rounded vector's sums by its rounding.
// A residual replacement due after step k (decided on the expanded ||r_{k+1}||)
// folds x + alpha_k p_k into x64, recomputes r in FP64 and restarts the step
// with alpha = 0, so the Krylov direction is kept exactly as in the other forms.
// r, p and q are double-buffered (set iter & 1 read, the other written): rows of
// other blocks gather the old values while this block writes the new ones.
// Over the Q1 triple stencils the operand windows come from 16-byte loads and
// warp shuffles (dia_rows4_triples_window).  It moves 36N vector bytes per
// iteration against 52N for the two-kernel form, but forming each operand entry
// from four gathered vectors takes 80 registers and 2.6x the instructions of the
// fused SpMV, and the pass becomes latency-bound: at 128^3 it measured 38.0 ms
// per solve against 27.7 ms (33.5 ms on the Jacobi-scaled inner system, which
// gathers three).
struct SingleVectors {
    float* r[2];
    float* p[2];
    float* q[2];
};

template <bool SCALED>
struct SingleStep {
    const float* __restrict__ r;
    const float* __restrict__ q;
    const float* __restrict__ p;
    const float* __restrict__ dinv;
    float alpha, beta;
    bool step;   // alpha != 0: apply the pending step to x and r
    bool fresh;  // beta == 0: p = z (first iteration, restart)

    // r_{k+1}, then p_{k+1} from it; the same operations in every caller.
    __device__ __forceinline__ float residual(float rk, float qk) const { return step ? fmaf(-alpha, qk, rk) : rk; }
    __device__ __forceinline__ float direction(float rn, float pk, float d) const {
        const float z = SCALED ? rn : __fmul_rn(rn, d);
        return fresh ? z : fmaf(beta, pk, z);
    }
    // operand entry of column c (inside [0, n))
    __device__ __forceinline__ float operator()(int c) const {
        const float rk = __ldg(r + c);
        const float rn = residual(rk, step ? __ldg(q + c) : 0.f);
        return direction(rn, fresh ? 0.f : __ldg(p + c), SCALED ? 1.f : __ldg(dinv + c));
    }
    // operand entries of columns 4b .. 4b + 3 (inside [0, n)), from 16-byte loads
    __device__ __forceinline__ float4 block(int b) const {
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f), one = make_float4(1.f, 1.f, 1.f, 1.f);
        const float4 rk = __ldg(reinterpret_cast<const float4*>(r) + b);
        const float4 qk = step ? __ldg(reinterpret_cast<const float4*>(q) + b) : zero;
        const float4 pk = fresh ? zero : __ldg(reinterpret_cast<const float4*>(p) + b);
        const float4 dk = SCALED ? one : __ldg(reinterpret_cast<const float4*>(dinv) + b);
        return make_float4(direction(residual(rk.x, qk.x), pk.x, dk.x), direction(residual(rk.y, qk.y), pk.y, dk.y),
                           direction(residual(rk.z, qk.z), pk.z, dk.z), direction(residual(rk.w, qk.w), pk.w, dk.w));
    }
};

template <bool SCALED>
struct SingleOp {
    struct Pre {
        float x, r, p, d;
    };
    static constexpr int K = SCALED ? 4 : 7;
    SingleStep<SCALED> in;
    float* __restrict__ x;
    float* __restrict__ r;  // write set
    float* __restrict__ p;
    float* __restrict__ q;
    int n;
    // p^T q, then ||r||^2, r^T q, ||q||^2, then (unscaled) the same three weighted by D^-1
    double acc[K];

    __device__ __forceinline__ Pre make(float xk, float rk, float pk, float qk, float d) const {
        Pre o;
        o.r = in.residual(rk, qk);
        o.x = in.step ? fmaf(in.alpha, pk, xk) : xk;
        o.p = in.direction(o.r, pk, d);
        o.d = d;
        return o;
    }
    __device__ __forceinline__ void pre4(int row, Pre (&pre)[4]) const {
        if (row + 3 < n) {
            const float4 rk = *reinterpret_cast<const float4*>(in.r + row);
            const float4 qk = in.step ? *reinterpret_cast<const float4*>(in.q + row) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 pk = (in.step || !in.fresh) ? *reinterpret_cast<const float4*>(in.p + row)
                                                    : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 xk = in.step ? *reinterpret_cast<const float4*>(x + row) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 dk = SCALED ? make_float4(1.f, 1.f, 1.f, 1.f) : *reinterpret_cast<const float4*>(in.dinv + row);
            pre[0] = make(xk.x, rk.x, pk.x, qk.x, dk.x);
            pre[1] = make(xk.y, rk.y, pk.y, qk.y, dk.y);
            pre[2] = make(xk.z, rk.z, pk.z, qk.z, dk.z);
            pre[3] = make(xk.w, rk.w, pk.w, qk.w, dk.w);
            return;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (row + i < n) {
                const int j = row + i;
                pre[i] = make(in.step ? x[j] : 0.f, in.r[j], (in.step || !in.fresh) ? in.p[j] : 0.f,
                              in.step ? in.q[j] : 0.f, SCALED ? 1.f : in.dinv[j]);
            }
    }
    __device__ __forceinline__ void sums(const Pre& o, float qn) {
        const double rv = o.r, qv = qn;
        acc[0] = fma(static_cast<double>(o.p), qv, acc[0]);
        acc[1] = fma(rv, rv, acc[1]);
        acc[2] = fma(rv, qv, acc[2]);
        acc[3] = fma(qv, qv, acc[3]);
        if constexpr (!SCALED) {
            const double d = o.d;
            acc[4] = fma(d * rv, rv, acc[4]);
            acc[5] = fma(d * rv, qv, acc[5]);
            acc[6] = fma(d * qv, qv, acc[6]);
        }
    }
    __device__ __forceinline__ void post4(int row, Pre (&pre)[4], const float (&sum)[4]) {
        if (row + 3 < n) {
            if (in.step)
                *reinterpret_cast<float4*>(x + row) = make_float4(pre[0].x, pre[1].x, pre[2].x, pre[3].x);
            *reinterpret_cast<float4*>(r + row) = make_float4(pre[0].r, pre[1].r, pre[2].r, pre[3].r);
            *reinterpret_cast<float4*>(p + row) = make_float4(pre[0].p, pre[1].p, pre[2].p, pre[3].p);
            *reinterpret_cast<float4*>(q + row) = make_float4(sum[0], sum[1], sum[2], sum[3]);
#pragma unroll
            for (int i = 0; i < 4; ++i) sums(pre[i], sum[i]);
            return;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (row + i < n) {
                const int j = row + i;
                if (in.step) x[j] = pre[i].x;
                r[j] = pre[i].r;
                p[j] = pre[i].p;
                q[j] = sum[i];
                sums(pre[i], sum[i]);
            }
    }
};

// Last block of a single-pass iteration: alpha_k, the expanded rho_{k+1} and
// ||r_{k+1}||, the replacement decision of mixed_update_kernel, beta_{k+1}.
// tot: p^T q, ||r||^2, r^T q, ||q||^2 and (unscaled) r^T D^-1 r, r^T D^-1 q, q^T D^-1 q.
template <bool COND, int K>
__device__ void single_decide(MixedScalars* s, const double (&tot)[K], cudaGraphConditionalHandle loop,
                              cudaGraphConditionalHandle refine) {
    const int w = K == 7 ? 4 : 1;  // first of the three D^-1-weighted sums
    const double rho = tot[w];
    s->pq = tot[0];
    s->iter += 1;
    s->rz = rho;
    s->updateX = 0;
    bool update;
    if (!(0.0 < tot[0])) {  // FP32 breakdown: no step, replacement with a restarted direction
        s->alpha = 0.0;
        s->restart = 1;
        s->breakdowns += 1;
        if (s->breakdowns > kMaxInnerBreakdowns) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
            set_cond<COND>(refine, 0);
            set_cond<COND>(loop, 0);
            return;
        }
        update = true;
    } else {
        const double alpha = rho / tot[0];
        const double rr = fma(alpha, fma(alpha, tot[3], -2.0 * tot[2]), tot[1]);
        const double rhoNext = fma(alpha, fma(alpha, tot[w + 2], -2.0 * tot[w + 1]), tot[w]);
        const double rnorm = rr > 0.0 ? sqrt(rr) : 0.0;
        s->alpha = alpha;
        s->sloppy = rnorm;
        if (s->mode == 0) {
            if (rnorm > s->maxrx) s->maxrx = rnorm;
            if (rnorm > s->maxrr) s->maxrr = rnorm;
            const bool updateX = rnorm < s->delta * s->maxrx;
            update = updateX || rnorm < s->delta * s->maxrr;
            s->updateX = updateX ? 1 : 0;
        } else {
            update = rnorm < s->delta * s->cycleStart;
        }
        update = update || rnorm < s->relTol * s->r0s || rnorm < s->absTol || s->iter >= s->maxIter ||
                 !(0.0 < rhoNext);
        if (!update) s->beta = rhoNext / rho;
    }
    if (update) s->update = 1;
    s->chunkIter += 1;
    set_cond<COND>(refine, update ? 1u : 0u);
    set_cond<COND>(loop, s->chunkIter < s->chunkLimit ? 1u : 0u);
}

template <int ND, bool COND, bool SCALED, bool TRIPLES>
__global__ void __launch_bounds__(kT, 3) mixed_single_dia_kernel(DiaArgs<float> A, float* __restrict__ x,
                                                             SingleVectors v, const float* __restrict__ dinv,
                                                             MixedScalars* s, double* partials, unsigned* counter,
                                                             cudaGraphConditionalHandle loop,
                                                             cudaGraphConditionalHandle refine) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            set_cond<COND>(refine, 0);
            set_cond<COND>(loop, 0);
        }
        return;
    }
    const int rd = static_cast<int>(*reinterpret_cast<const volatile long long*>(&s->iter) & 1);
    const double alpha = *reinterpret_cast<const volatile double*>(&s->alpha);
    const double beta = *reinterpret_cast<const volatile double*>(&s->beta);
    // (selects, not an index: a runtime index would put v in local memory)
    const SingleStep<SCALED> in{rd ? v.r[1] : v.r[0], rd ? v.q[1] : v.q[0], rd ? v.p[1] : v.p[0], dinv,
                                static_cast<float>(alpha), static_cast<float>(beta), alpha != 0.0, beta == 0.0};
    SingleOp<SCALED> op{in, x, rd ? v.r[0] : v.r[1], rd ? v.p[0] : v.p[1], rd ? v.q[0] : v.q[1], A.nrows, {}};
    if constexpr (TRIPLES)
        dia_rows4_triples_window<ND>(A, in, op);
    else
        dia_rows4_gather<ND>(A, in, op);
    constexpr int K = SingleOp<SCALED>::K;
    double tot[K];
    if (grid_reduce_last<K, kT>(op.acc, partials, counter, tot) && threadIdx.x == 0)
        single_decide<COND, K>(s, tot, loop, refine);
}

// R1 of the single-pass form: x64 += x32 + alpha p (the step decided but not yet
// applied; alpha = 0 after an FP32 breakdown), x32 = 0.
__global__ void __launch_bounds__(kT) mixed_fold_pending_kernel(long n, double* __restrict__ x64,
                                                                float* __restrict__ x32, SingleVectors v,
                                                                const double* __restrict__ sdiag,
                                                                const MixedScalars* s) {
    if (!*reinterpret_cast<const volatile int*>(&s->update)) return;
    const float* p = (s->iter & 1) ? v.p[1] : v.p[0];
    const float alpha = static_cast<float>(s->alpha);
    const bool step = s->alpha != 0.0;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long i = static_cast<long>(blockIdx.x) * kT + threadIdx.x; i < n; i += stride) {
        const float xi = step ? fmaf(alpha, p[i], x32[i]) : x32[i];
        x64[i] += sdiag ? static_cast<double>(xi) * sdiag[i] : static_cast<double>(xi);
        x32[i] = 0.0f;
    }
}

// TMA-pipelined variants of the two kernels above (sell_tma.cuh): one CTA of
// kTmaWarps warps per SM, the matrix streamed through shared memory.
template <typename CI>
__global__ void __launch_bounds__(kTmaWarps * 32) mixed_apply_tma_kernel(SellArgs<float, CI> A,
                                                                         const float* __restrict__ x,
                                                                         float* __restrict__ y, unsigned* error) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    StoreOp op{y};
    sell_rows_tma<CI>(A, x, op, tma_smem, error);
}

template <typename CI, bool COND, bool FUSED>
__global__ void __launch_bounds__(kTmaWarps * 32) mixed_spmv_tma_kernel(SellArgs<float, CI> A,
                                                                        const float* __restrict__ x,
                                                                        float* __restrict__ p, float* __restrict__ q,
                                                                        MixedScalars* s, double* partials,
                                                                        unsigned* counter,
                                                                        cudaGraphConditionalHandle loop) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond<COND>(loop, 0);
        return;
    }
    auto op = M1Op<FUSED>::make(x, p, q, s);
    sell_rows_tma<CI>(A, x, op, tma_smem, &s->tmaError);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, kTmaWarps * 32>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (s->tmaError) {
            s->done = 3;
            s->error = CIECU_ERR_TIMEOUT;
            set_cond<COND>(loop, 0);
        } else if (!(0.0 < tot[0])) {
            if (inner_breakdown(s)) set_cond<COND>(loop, 0);
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// Raises the dynamic shared memory limit of a TMA kernel once (before any
// occupancy query, launch or capture).
template <typename K>
int allow_tma_smem(K* kernel, int bytes) {
    CIECU_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    bytes));
    return CIECU_OK;
}

// M2: x32 += alpha p; r32 -= alpha q; rr, rz in FP64; replacement decision.  The
// fused form also stores z = D^-1 r for the next M1.
template <bool COND, bool FUSED>
__global__ void __launch_bounds__(kT, 3) mixed_update_kernel(long n, float* __restrict__ x, float* __restrict__ r,
                                                          float* __restrict__ z,
                                                          const float* __restrict__ p, const float* __restrict__ q,
                                                          const float* __restrict__ dinv, MixedScalars* s,
                                                          double* partials, unsigned* counter,
                                                          cudaGraphConditionalHandle loop,
                                                          cudaGraphConditionalHandle refine) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            set_cond<COND>(loop, 0);
            set_cond<COND>(refine, 0);
        }
        return;
    }
    const float alpha = static_cast<float>(s->alpha);
    const bool step = !s->restart;  // after an FP32 breakdown: no step (p may not be finite)
    double rr = 0.0, rz = 0.0;
    const long quads = n >> 2;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long j = static_cast<long>(blockIdx.x) * kT + threadIdx.x; j < quads; j += stride) {
        const float4 dj = reinterpret_cast<const float4*>(dinv)[j];
        float4 rj = reinterpret_cast<const float4*>(r)[j];
        if (step) {
            const float4 pj = reinterpret_cast<const float4*>(p)[j];
            const float4 qj = reinterpret_cast<const float4*>(q)[j];
            float4 xj = reinterpret_cast<const float4*>(x)[j];
            xj.x = fmaf(alpha, pj.x, xj.x); xj.y = fmaf(alpha, pj.y, xj.y);
            xj.z = fmaf(alpha, pj.z, xj.z); xj.w = fmaf(alpha, pj.w, xj.w);
            rj.x = fmaf(-alpha, qj.x, rj.x); rj.y = fmaf(-alpha, qj.y, rj.y);
            rj.z = fmaf(-alpha, qj.z, rj.z); rj.w = fmaf(-alpha, qj.w, rj.w);
            reinterpret_cast<float4*>(x)[j] = xj;
            reinterpret_cast<float4*>(r)[j] = rj;
        }
        const float4 zj = make_float4(rj.x * dj.x, rj.y * dj.y, rj.z * dj.z, rj.w * dj.w);
        if (FUSED) reinterpret_cast<float4*>(z)[j] = zj;
        rr = fma(double(rj.x), double(rj.x), rr); rr = fma(double(rj.y), double(rj.y), rr);
        rr = fma(double(rj.z), double(rj.z), rr); rr = fma(double(rj.w), double(rj.w), rr);
        rz = fma(double(rj.x), double(zj.x), rz); rz = fma(double(rj.y), double(zj.y), rz);
        rz = fma(double(rj.z), double(zj.z), rz); rz = fma(double(rj.w), double(zj.w), rz);
    }
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
        const long i = (quads << 2) + threadIdx.x;
        float ri = r[i];
        if (step) {
            x[i] = fmaf(alpha, p[i], x[i]);
            ri = fmaf(-alpha, q[i], ri);
            r[i] = ri;
        }
        const float zi = ri * dinv[i];
        if (FUSED) z[i] = zi;
        rr = fma(double(ri), double(ri), rr);
        rz = fma(double(ri), double(zi), rz);
    }
    double mine[2] = {rr, rz}, tot[2];
    if (grid_reduce_last<2, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        const double rnorm = sqrt(tot[0]);
        s->sloppy = rnorm;
        s->iter += 1;
        bool update;
        s->updateX = 0;
        if (s->mode == 0) {
            if (rnorm > s->maxrx) s->maxrx = rnorm;
            if (rnorm > s->maxrr) s->maxrr = rnorm;
            const bool updateX = rnorm < s->delta * s->maxrx;
            update = updateX || rnorm < s->delta * s->maxrr;
            s->updateX = updateX ? 1 : 0;
        } else {
            update = rnorm < s->delta * s->cycleStart;
        }
        update = update || rnorm < s->relTol * s->r0s || rnorm < s->absTol || s->iter >= s->maxIter || s->restart;
        if (update) {
            s->rzPending = tot[1];
            s->update = 1;
        } else {
            s->beta = tot[1] / s->rz;
            s->rz = tot[1];
        }
        s->chunkIter += 1;
        set_cond<COND>(refine, update ? 1u : 0u);
        set_cond<COND>(loop, s->chunkIter < s->chunkLimit ? 1u : 0u);
    }
}

// R1: x64 += x32; x32 = 0 (only when a replacement was requested).
__global__ void __launch_bounds__(kT) mixed_fold_kernel(long n, double* __restrict__ x64, float* __restrict__ x32,
                                                        const double* __restrict__ sdiag, const MixedScalars* s) {
    if (!*reinterpret_cast<const volatile int*>(&s->update)) return;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long i = static_cast<long>(blockIdx.x) * kT + threadIdx.x; i < n; i += stride) {
        x64[i] += sdiag ? static_cast<double>(x32[i]) * sdiag[i] : static_cast<double>(x32[i]);
        x32[i] = 0.0f;
    }
}

struct ResidualOp {
    struct Pre {
        double b;
        float d;
        double s;
    };
    const double* __restrict__ b;
    const float* __restrict__ dinv;
    float* __restrict__ r32;
    float* __restrict__ z32;           // the fused form keeps z = D^-1 r (or null)
    const double* __restrict__ sdiag;  // inner scaling (or null)
    double rr, rz;
    __device__ __forceinline__ Pre pre(int row) const { return Pre{b[row], dinv[row], sdiag ? sdiag[row] : 1.0}; }
    __device__ __forceinline__ void post(int row, const Pre& p, double sum) {
        const double ri = p.b - sum;
        const float rf = static_cast<float>(sdiag ? ri * p.s : ri);
        const float zf = rf * p.d;
        r32[row] = rf;
        if (z32) z32[row] = zf;
        rr = fma(ri, ri, rr);
        rz = fma(double(rf), double(zf), rz);
    }
};

// R2 (and set-up): r = b - A64 x64 in FP64; r32 = float(r); ||r||^2 and r32^T z32
// in FP64.  INIT: first residual of a solve.  r32alt (the single-pass form's
// second residual buffer, else null) takes r when the iteration count is odd.
template <int KERNEL, bool INIT, bool COND>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    mixed_residual_kernel(CsrArgs<double> A, const double* __restrict__ b, const double* __restrict__ x64,
                          const float* __restrict__ dinv, float* __restrict__ r32, float* __restrict__ r32alt,
                          float* __restrict__ z32, const double* __restrict__ sdiag, MixedScalars* s,
                          double* partials, unsigned* counter, cudaGraphConditionalHandle loop) {
    if (!INIT && !*reinterpret_cast<volatile int*>(&s->update)) return;
    constexpr int T = csr_threads<KERNEL>();
    float* rdst = (r32alt && (*reinterpret_cast<const volatile long long*>(&s->iter) & 1)) ? r32alt : r32;
    ResidualOp op{b, dinv, rdst, z32, sdiag, 0.0, 0.0};
    csr_rows<KERNEL, double, double, false>(A, x64, op);
    const double rr = op.rr, rz = op.rz;
    double mine[2] = {rr, rz}, tot[2];
    if (grid_reduce_last<2, T>(mine, partials, counter, tot) && threadIdx.x == 0) {
        const double rnorm = sqrt(tot[0]);
        // the FP32 recursion's norms are in the inner units: scaled when the inner
        // system is scaled (then z32 = r32 and tot[1] = ||r32||^2)
        const double rs = s->scaled ? sqrt(tot[1]) : rnorm;
        s->rnorm = rnorm;
        if (INIT) {
            s->r0 = rnorm;
            s->r0s = rs;
            s->absres = rnorm;
            s->relres = 1.0;
            s->maxrx = s->maxrr = s->cycleStart = rs;
            s->iter = 0;
            s->refinements = 0;
            s->update = 0;
            s->done = 0;
            s->error = 0;
            s->alpha = 0.0;
            s->beta = 0.0;
            s->rz = tot[1];
            if (float_less(rnorm, s->absTol) || float_less(1.0, s->relTol)) {
                s->done = 1;
            } else if (!(0.0 < tot[1])) {
                s->done = 3;
                s->error = CIECU_ERR_BREAKDOWN;
            } else if (s->maxIter <= 0) {
                s->done = 2;
            }
            return;
        }
        s->refinements += 1;
        s->update = 0;
        s->absres = rnorm;
        s->relres = rnorm / s->r0;
        if (float_less(s->absres, s->absTol) || float_less(s->relres, s->relTol)) {
            s->done = 1;
        } else if (s->iter >= s->maxIter) {
            s->done = 2;
        } else if (!(0.0 < tot[1])) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
        } else {
            if (s->mode == 0) {
                s->maxrr = rs;
                if (s->updateX) s->maxrx = rs;
                s->beta = s->restart ? 0.0 : tot[1] / s->rz;  // after an FP32 breakdown: p = z
            } else {
                s->cycleStart = rs;
                s->beta = 0.0;  // restart the inner CG: p = z
            }
            s->rz = tot[1];
        }
        s->alpha = 0.0;  // the single-pass form's pending step is folded into x64
        s->restart = 0;
        if (s->done) set_cond<COND>(loop, 0);
    }
}

// M3: p = z + beta p, z = D^-1 r (FP32).
__global__ void __launch_bounds__(kT) mixed_direction_kernel(long n, float* __restrict__ p, const float* __restrict__ r,
                                                             const float* __restrict__ dinv, const MixedScalars* s) {
    if (*reinterpret_cast<const volatile int*>(&s->done)) return;
    const float beta = static_cast<float>(s->beta);
    const long quads = n >> 2;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long j = static_cast<long>(blockIdx.x) * kT + threadIdx.x; j < quads; j += stride) {
        const float4 rj = reinterpret_cast<const float4*>(r)[j];
        const float4 dj = reinterpret_cast<const float4*>(dinv)[j];
        float4 pj = reinterpret_cast<const float4*>(p)[j];
        pj.x = fmaf(beta, pj.x, rj.x * dj.x);
        pj.y = fmaf(beta, pj.y, rj.y * dj.y);
        pj.z = fmaf(beta, pj.z, rj.z * dj.z);
        pj.w = fmaf(beta, pj.w, rj.w * dj.w);
        reinterpret_cast<float4*>(p)[j] = pj;
    }
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
        const long i = (quads << 2) + threadIdx.x;
        p[i] = fmaf(beta, p[i], r[i] * dinv[i]);
    }
}

__global__ void fill_f32_kernel(long n, float v, float* __restrict__ b) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) b[i] = v;
}

__global__ void sqrt_kernel(long n, const double* __restrict__ a, double* __restrict__ b) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) b[i] = sqrt(a[i]);
}

__global__ void to_f32_kernel(long n, const double* __restrict__ a, float* __restrict__ b) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        b[i] = static_cast<float>(a[i]);
}

__global__ void mixed_output_kernel(long n, double inScale, double outScale, const double* __restrict__ x,
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

}  // namespace
}  // namespace ciecu

struct ciecu_mixed_s {
    ciecu_csr_s* A = nullptr;
    const double* dinv64 = nullptr;
    ciecu_statistics settings{};
    ciecu_mixed_options options{};
    long n = 0;
    bool idx16 = false;
    int unroll = 2;  // SELL groups of four entries in flight per thread (autotuned; 0 = TMA pipeline,
                     // kDiaInner = the DIA copy)
    bool sellBuilt = false;  // the SELL copy exists (not built when the DIA copy is the known choice)
    float* dia32 = nullptr;  // DIA copy of the inner matrix (few-diagonal matrices only)
    bool diaTriples = false;  // its offsets come in consecutive triples (dia_rows4_triples)
    ciecu::DiaArgs<float> dia{};
    // SELL-32 inner matrix
    int nslices = 0;
    long long paddedEntries = 0;
    int* sliceLen = nullptr;
    long long* sliceStart = nullptr;
    unsigned short* rowLen = nullptr;
    float* val32 = nullptr;
    void* col32or16 = nullptr;
    ciecu::SellArgs<float, short> a16{};
    ciecu::SellArgs<float, int> a32{};
    float* dinv32 = nullptr;
    double* sdiag = nullptr;  // sqrt(D^-1) when the inner system is scaled
    float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
    float* z32 = nullptr;  // z = D^-1 r, kept only by the fused form (options.fuseDirection)
    int form = 0;          // options.fuseDirection: kernels per inner iteration 3 (0), 2 (1), 1 (2, DIA inner)
    float *r32b = nullptr, *p32b = nullptr, *q32b = nullptr;  // second buffers of the single-pass form
    double* x64 = nullptr;
    const double* b = nullptr;
    ciecu::MixedScalars* d_s = nullptr;
    ciecu::MixedScalars* h_s = nullptr;
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* graphB = nullptr;
    bool deviceLoop = false;
    cudaStream_t side = nullptr;  // captures the IF body of the refinement
    int chunk = 16;
};

namespace ciecu {
namespace {

// Calls f(std::integral_constant<int, U>) for the group unroll U in {1, 2, 4}.
template <typename F>
int with_unroll(int u, F&& f) {
    switch (u) {
        case 1: return f(std::integral_constant<int, 1>{});
        case 4: return f(std::integral_constant<int, 4>{});
        default: return f(std::integral_constant<int, 2>{});
    }
}

// M1 with the autotuned variant: TMA pipeline (unroll == 0), the DIA copy
// (unroll == kDiaInner) or U register groups.  FUSED gathers z (the direction
// recurrences run in the epilogue), otherwise p.
template <bool COND, bool FUSED>
int launch_inner_spmv_form(ciecu_mixed_s* M, cudaStream_t st, cudaGraphConditionalHandle loop) {
    const long needA = (M->n + kT - 1) / kT;
    const float* x = FUSED ? M->z32 : M->p32;
    if (M->unroll == kDiaInner) {
        CIECU_TRY(with_diagonals(M->dia.ndiag, [&](auto nd) -> int {
            constexpr int ND = decltype(nd)::value;
            auto* kernel = M->diaTriples ? mixed_spmv_dia_kernel<ND, COND, FUSED, true>
                                         : mixed_spmv_dia_kernel<ND, COND, FUSED, false>;
            kernel<<<fit_grid(kernel, kT, (needA + 3) / 4), kT, 0, st>>>(M->dia, x, M->p32, M->q32, M->d_s,
                                                                         M->d_partials, M->d_counter, loop);
            return CIECU_OK;
        }));
        CIECU_CHECK_LAUNCH("mixed_spmv_dia_kernel");
        return CIECU_OK;
    }
    if (M->unroll == 0) {
        if (M->idx16) {
            constexpr int smem = TmaShape<float, short>::SMEM;
            auto* kernel = mixed_spmv_tma_kernel<short, COND, FUSED>;
            kernel<<<fit_grid(kernel, kTmaWarps * 32, (M->n + 511) / 512, smem), kTmaWarps * 32, smem, st>>>(
                M->a16, x, M->p32, M->q32, M->d_s, M->d_partials, M->d_counter, loop);
        } else {
            constexpr int smem = TmaShape<float, int>::SMEM;
            auto* kernel = mixed_spmv_tma_kernel<int, COND, FUSED>;
            kernel<<<fit_grid(kernel, kTmaWarps * 32, (M->n + 511) / 512, smem), kTmaWarps * 32, smem, st>>>(
                M->a32, x, M->p32, M->q32, M->d_s, M->d_partials, M->d_counter, loop);
        }
        CIECU_CHECK_LAUNCH("mixed_spmv_tma_kernel");
        return CIECU_OK;
    }
    return with_unroll(M->unroll, [&](auto uu) -> int {
        constexpr int U = decltype(uu)::value;
        if (M->idx16) {
            auto* kernel = mixed_spmv_kernel<U, short, COND, FUSED>;
            kernel<<<fit_grid(kernel, kT, needA), kT, 0, st>>>(M->a16, x, M->p32, M->q32, M->d_s, M->d_partials,
                                                               M->d_counter, loop);
        } else {
            auto* kernel = mixed_spmv_kernel<U, int, COND, FUSED>;
            kernel<<<fit_grid(kernel, kT, needA), kT, 0, st>>>(M->a32, x, M->p32, M->q32, M->d_s, M->d_partials,
                                                               M->d_counter, loop);
        }
        return CIECU_OK;
    });
}

template <bool COND>
int launch_inner_spmv(ciecu_mixed_s* M, cudaStream_t st, cudaGraphConditionalHandle loop) {
    return M->z32 ? launch_inner_spmv_form<COND, true>(M, st, loop) : launch_inner_spmv_form<COND, false>(M, st, loop);
}

// The single-pass form runs over the DIA copy only; with another inner kernel a
// solver created with fuseDirection = 2 runs the fused two-kernel form.
bool single_pass(const ciecu_mixed_s* M) { return M->form == 2 && M->unroll == kDiaInner; }

SingleVectors single_vectors(const ciecu_mixed_s* M) {
    return SingleVectors{{M->r32, M->r32b}, {M->p32, M->p32b}, {M->q32, M->q32b}};
}

template <bool COND>
int launch_single(ciecu_mixed_s* M, cudaStream_t st, cudaGraphConditionalHandle loop,
                  cudaGraphConditionalHandle refine) {
    const long needA = (M->n + kT - 1) / kT;
    const bool scaled = M->sdiag != nullptr;
    CIECU_TRY(with_diagonals(M->dia.ndiag, [&](auto nd) -> int {
        constexpr int ND = decltype(nd)::value;
        auto* kernel = M->diaTriples ? (scaled ? mixed_single_dia_kernel<ND, COND, true, true>
                                               : mixed_single_dia_kernel<ND, COND, false, true>)
                                     : (scaled ? mixed_single_dia_kernel<ND, COND, true, false>
                                               : mixed_single_dia_kernel<ND, COND, false, false>);
        kernel<<<fit_grid(kernel, kT, (needA + 3) / 4), kT, 0, st>>>(M->dia, M->x32, single_vectors(M), M->dinv32,
                                                                     M->d_s, M->d_partials, M->d_counter, loop, refine);
        return CIECU_OK;
    }));
    CIECU_CHECK_LAUNCH("mixed_single_dia_kernel");
    return CIECU_OK;
}

// One inner iteration.  With conditional nodes (useCond) the refinement pair
// R1/R2 sits under IF(refine); otherwise it is launched unconditionally and
// returns at once unless M2 requested a replacement.
template <bool COND>
int launch_inner(ciecu_mixed_s* M, cudaStream_t st, cudaGraph_t root, cudaGraphConditionalHandle loop) {
    constexpr bool useCond = COND;
    const long needA = (M->n + kT - 1) / kT;
    const long needV = ((M->n + 3) / 4 + kT - 1) / kT;
    ciecu_csr_s* A = M->A;
    cudaGraphConditionalHandle refine = 0;
    if (useCond) CIECU_CUDA(cudaGraphConditionalHandleCreate(&refine, root, 0, cudaGraphCondAssignDefault));
    const bool single = single_pass(M);
    if (single) {
        CIECU_TRY(launch_single<COND>(M, st, loop, refine));
    } else {
        CIECU_TRY(launch_inner_spmv<COND>(M, st, loop));
        auto* kernel = M->z32 ? mixed_update_kernel<COND, true> : mixed_update_kernel<COND, false>;
        kernel<<<fit_grid(kernel, kT, needV), kT, 0, st>>>(M->n, M->x32, M->r32, M->z32, M->p32, M->q32, M->dinv32,
                                                           M->d_s, M->d_partials, M->d_counter, loop, refine);
    }
    auto refinement = [&](cudaStream_t s2) -> int {
        if (single)
            mixed_fold_pending_kernel<<<fit_grid(mixed_fold_pending_kernel, kT, needA), kT, 0, s2>>>(
                M->n, M->x64, M->x32, single_vectors(M), M->sdiag, M->d_s);
        else
            mixed_fold_kernel<<<fit_grid(mixed_fold_kernel, kT, needA), kT, 0, s2>>>(M->n, M->x64, M->x32, M->sdiag,
                                                                                    M->d_s);
        const int needR = csr_grid(A, A->kernel);
        CIECU_TRY(with_schedule(A->kernel, [&](auto k) -> int {
            constexpr int K = decltype(k)::value;
            mixed_residual_kernel<K, false, COND><<<fit_grid(mixed_residual_kernel<K, false, COND>, csr_threads<K>(),
                                                             needR),
                                                    csr_threads<K>(), 0, s2>>>(
                A->args<double>(), M->b, M->x64, M->dinv32, M->r32, single ? M->r32b : nullptr,
                single ? nullptr : M->z32, M->sdiag, M->d_s, M->d_partials, M->d_counter, loop);
            return CIECU_OK;
        }));
        return CIECU_OK;
    };
    if (useCond)
        CIECU_TRY(capture_if(st, M->side, refine, refinement));
    else
        CIECU_TRY(refinement(st));
    if (!M->z32 && !single)
        mixed_direction_kernel<<<fit_grid(mixed_direction_kernel, kT, needV), kT, 0, st>>>(M->n, M->p32, M->r32,
                                                                                           M->dinv32, M->d_s);
    CIECU_CHECK_LAUNCH("mixed inner iteration");
    return CIECU_OK;
}

int build_mixed_graph(ciecu_mixed_s* M) {
    if (M->graph && M->graphB == M->b) return CIECU_OK;
    if (M->graph) {
        cudaGraphExecDestroy(M->graph);
        M->graph = nullptr;
    }
    cudaStream_t st = M->A->space->stream;
    int status = CIECU_ERR_ARGUMENT;
    if (device_loop_enabled())
        status = build_while_graph(st, [&](cudaGraph_t root, cudaGraphConditionalHandle loop) {
        return launch_inner<true>(M, st, root, loop);
    }, &M->graph);
    if (status == CIECU_OK) {
        M->deviceLoop = true;
        M->graphB = M->b;
        return CIECU_OK;
    }
    cudaGetLastError();
    M->deviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    status = CIECU_OK;
    for (int i = 0; i < M->chunk && status == CIECU_OK; ++i) status = launch_inner<false>(M, st, nullptr, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "mixed graph capture");
    e = cudaGraphInstantiate(&M->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "mixed graph instantiate");
    M->graphB = M->b;
    return CIECU_OK;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

namespace ciecu {
namespace {

// SELL-32x4 copy of the inner matrix (sell.cuh): slice lengths on the device,
// their prefix sum on the host, then the FP32 values and 16-bit or int32 columns.
int build_sell(ciecu_mixed_s* M, ciecu_csr_s* lhs, const ciecu_mixed_options& options, cudaStream_t st) {
    const size_t n = static_cast<size_t>(std::max<long>(M->n, 1)) + 4;
    cudaError_t e = cudaMalloc(&M->sliceLen, sizeof(int) * std::max(1, M->nslices));
    if (e == cudaSuccess) e = cudaMalloc(&M->sliceStart, sizeof(long long) * (M->nslices + 1));
    if (e == cudaSuccess) e = cudaMalloc(&M->rowLen, sizeof(unsigned short) * n);
    if (e != cudaSuccess) return cuda_fail(e, "mixed_create: SELL allocation");
    // Slice lengths on the device, their prefix sum on the host.
    unsigned* d_flag = reinterpret_cast<unsigned*>(lhs->space->d_result);
    unsigned flags[2] = {0, 0};
    e = cudaMemsetAsync(d_flag, 0, 2 * sizeof(unsigned), st);
    if (M->n > 0 && e == cudaSuccess) {
        sell_len_kernel<<<grid_for(M->nslices, kT, 8), kT, 0, st>>>(static_cast<int>(M->n), lhs->rowptr, M->sliceLen,
                                                                    d_flag);
        count_launch();
        e = cudaGetLastError();
    }
    std::vector<int> lens(static_cast<size_t>(M->nslices));
    std::vector<long long> starts(static_cast<size_t>(M->nslices) + 1, 0);
    if (e == cudaSuccess && M->nslices)
        e = cudaMemcpyAsync(lens.data(), M->sliceLen, sizeof(int) * lens.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "mixed_create: slice lengths");
    if (flags[0]) return fail(CIECU_ERR_ARGUMENT, "mixed_create: rows longer than 65535 entries are not supported");
    for (int sl = 0; sl < M->nslices; ++sl) starts[sl + 1] = starts[sl] + 128LL * ((std::abs(lens[sl]) + 3) / 4);
    M->paddedEntries = starts.back();
    e = cudaMemcpyAsync(M->sliceStart, starts.data(), sizeof(long long) * starts.size(), cudaMemcpyHostToDevice, st);
    const size_t padded = static_cast<size_t>(std::max<long long>(1, M->paddedEntries));
    if (e == cudaSuccess) e = cudaMalloc(&M->val32, sizeof(float) * padded);
    const bool try16 = options.compressColumns != 0;
    if (e == cudaSuccess) e = cudaMalloc(&M->col32or16, (try16 ? sizeof(short) : sizeof(int)) * padded);
    // lanes past the last row of the final slice are never written by the fill
    if (e == cudaSuccess) e = cudaMemsetAsync(M->val32, 0, sizeof(float) * padded, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->col32or16, 0, (try16 ? sizeof(short) : sizeof(int)) * padded, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, sizeof(unsigned), st);
    if (e == cudaSuccess && M->n > 0) {
        const int grid = grid_for(M->n, kT, 8);
        if (try16)
            sell_fill_kernel<short><<<grid, kT, 0, st>>>(static_cast<int>(M->n), lhs->rowptr, lhs->col,
                                                         static_cast<const double*>(lhs->val), M->sliceLen,
                                                         M->sliceStart, M->val32, static_cast<short*>(M->col32or16),
                                                         M->rowLen, d_flag, M->sdiag);
        else
            sell_fill_kernel<int><<<grid, kT, 0, st>>>(static_cast<int>(M->n), lhs->rowptr, lhs->col,
                                                       static_cast<const double*>(lhs->val), M->sliceLen,
                                                       M->sliceStart, M->val32, static_cast<int*>(M->col32or16),
                                                       M->rowLen, d_flag, M->sdiag);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "mixed_create: conversion");
    M->idx16 = try16 && !flags[0];
    if (try16 && flags[0]) {
        // bandwidth too large for 16-bit offsets: int32 columns
        cudaFree(M->col32or16);
        M->col32or16 = nullptr;
        e = cudaMalloc(&M->col32or16, sizeof(int) * padded);
        if (e == cudaSuccess) e = cudaMemsetAsync(M->col32or16, 0, sizeof(int) * padded, st);
        if (e == cudaSuccess && M->n > 0) {
            sell_fill_kernel<int><<<grid_for(M->n, kT, 8), kT, 0, st>>>(
                static_cast<int>(M->n), lhs->rowptr, lhs->col, static_cast<const double*>(lhs->val), M->sliceLen,
                M->sliceStart, M->val32, static_cast<int*>(M->col32or16), M->rowLen, d_flag, M->sdiag);
            count_launch();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "mixed_create: int32 columns");
    }
    M->a16 = SellArgs<float, short>{static_cast<int>(M->n), M->sliceLen, M->sliceStart, M->rowLen, M->val32,
                                    static_cast<const short*>(M->col32or16)};
    M->a32 = SellArgs<float, int>{static_cast<int>(M->n), M->sliceLen, M->sliceStart, M->rowLen, M->val32,
                                  static_cast<const int*>(M->col32or16)};
    M->sellBuilt = true;
    return CIECU_OK;
}

// Inner-kernel choice of the autotuner per matrix shape (rows, nonzeros,
// diagonals, 16-bit columns requested, scaled inner system): later solvers of the
// same shape skip the timing and, when the choice is the DIA copy, the SELL copy.
std::mutex g_innerMutex;
std::map<std::tuple<int, long, int, int, int>, int> g_innerChoice;

}  // namespace
}  // namespace ciecu

extern "C" {

int ciecu_mixed_create(ciecu_csr lhs, const double* d_inverseDiagonal, ciecu_statistics settings,
                       ciecu_mixed_options options, ciecu_mixed* out) {
    CIECU_REQUIRE(lhs && out && d_inverseDiagonal, "mixed_create: null argument");
    CIECU_REQUIRE(lhs->valueType == CIECU_F64 && lhs->rows == lhs->cols, "mixed_create: square FP64 matrix expected");
    CIECU_REQUIRE(options.mode == 0 || options.mode == 1, "mixed_create: mode must be 0 or 1");
    CIECU_REQUIRE(options.scaleInner == 0 || options.scaleInner == 1, "mixed_create: scaleInner must be 0 or 1");
    CIECU_REQUIRE(options.fuseDirection >= 0 && options.fuseDirection <= 2,
                  "mixed_create: fuseDirection must be 0, 1 or 2");
    CIECU_REQUIRE(options.delta > 0.0 && options.delta < 1.0, "mixed_create: delta must be in (0, 1)");
    CIECU_REQUIRE(options.innerKernel == 0 || options.innerKernel == 1 || options.innerKernel == 2 ||
                      options.innerKernel == 4 || options.innerKernel == -1 || options.innerKernel == kDiaInner,
                  "mixed_create: innerKernel must be 0 (autotune), 1, 2, 4, -1 (TMA pipeline) or -2 (DIA copy)");
    CIECU_TRY(ensure_tuned(lhs));
    auto* M = new ciecu_mixed_s();
    M->A = lhs;
    M->dinv64 = d_inverseDiagonal;
    M->settings = settings;
    M->options = options;
    M->n = lhs->rows;
    cudaStream_t st = lhs->space->stream;
    const size_t n = static_cast<size_t>(std::max<long>(M->n, 1)) + 4;
    M->nslices = static_cast<int>((M->n + 31) / 32);
    cudaError_t e = cudaSuccess;
    // solver buffers come from the library's stream-ordered pool (pool_alloc): a
    // solver of a size created before maps no new memory
    for (float** v : {&M->dinv32, &M->x32, &M->r32, &M->p32, &M->q32})
        if (e == cudaSuccess) e = pool_alloc(v, sizeof(float) * n, st);
    M->form = options.fuseDirection;
    if (e == cudaSuccess && options.fuseDirection) e = pool_alloc(&M->z32, sizeof(float) * n, st);
    if (options.fuseDirection == 2)
        for (float** v : {&M->r32b, &M->p32b, &M->q32b})
            if (e == cudaSuccess) e = pool_alloc(v, sizeof(float) * n, st);
    if (e == cudaSuccess) e = pool_alloc(&M->x64, sizeof(double) * n, st);
    if (e == cudaSuccess) e = pool_alloc(&M->d_s, sizeof(MixedScalars), st);
    M->h_s = new MixedScalars();  // read back once per graph launch: pageable is enough
    if (e == cudaSuccess) e = pool_alloc(&M->d_partials, sizeof(double) * kMaxPartials * 2, st);
    if (e == cudaSuccess) e = pool_alloc(&M->d_counter, sizeof(unsigned) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_counter, 0, sizeof(unsigned) * 4, st);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&M->side, cudaStreamNonBlocking);
    if (e == cudaSuccess && options.scaleInner) {
        e = pool_alloc(&M->sdiag, sizeof(double) * n, st);
        if (e == cudaSuccess && M->n > 0) {
            sqrt_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, d_inverseDiagonal, M->sdiag);
            count_launch();
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && M->n > 0) {
        if (M->sdiag)
            fill_f32_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, 1.0f, M->dinv32);  // D^-1 of the scaled matrix
        else
            to_f32_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, d_inverseDiagonal, M->dinv32);
        count_launch();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        ciecu_mixed_destroy(M);
        return cuda_fail(e, "mixed_create: allocation");
    }
    // DIA copy of the inner matrix when its nonzeros lie on few diagonals.
    if (M->n > 0 && (options.innerKernel == 0 || options.innerKernel == kDiaInner)) {
        const std::vector<int>* offsets = nullptr;
        int status = dia_offsets(lhs, &offsets);
        if (status == CIECU_OK && !offsets->empty()) {
            DiaArgs<float> a = dia_shape<float>(lhs, *offsets);
            const size_t bytes = sizeof(float) * static_cast<size_t>(a.ndiag) * static_cast<size_t>(a.ld);
            if (pool_alloc(&M->dia32, bytes, st) == cudaSuccess) {
                e = cudaMemsetAsync(M->dia32, 0, bytes, st);
                a.val = M->dia32;
                M->dia = a;
                if (e == cudaSuccess) status = dia_fill_f32(lhs, M->dia, M->dia32, M->sdiag, st);
                M->diaTriples = dia_has_triples(M->dia) && dia_triples_enabled();
                if (e != cudaSuccess) status = cuda_fail(e, "mixed_create: DIA copy");
            } else {
                cudaGetLastError();  // no room for the copy: the SELL kernels stay
                M->dia32 = nullptr;
            }
        }
        if (status != CIECU_OK) {
            ciecu_mixed_destroy(M);
            return status;
        }
        if (options.innerKernel == kDiaInner && !M->dia32) {
            ciecu_mixed_destroy(M);
            return fail(CIECU_ERR_ARGUMENT, "mixed_create: innerKernel -2 needs a matrix of at most 32 diagonals");
        }
    }
    const auto key = std::make_tuple(lhs->rows, lhs->nnz, M->dia32 ? M->dia.ndiag : 0, options.compressColumns ? 1 : 0,
                                     options.scaleInner);
    int cached = 1000;  // none
    if (options.innerKernel == 0) {
        std::lock_guard<std::mutex> lock(g_innerMutex);
        auto it = g_innerChoice.find(key);
        if (it != g_innerChoice.end() && (it->second != kDiaInner || M->dia32)) cached = it->second;
    }
    const bool diaOnly = (options.innerKernel == kDiaInner) || (cached == kDiaInner);
    if (!diaOnly) {
        const int status = build_sell(M, lhs, options, st);
        if (status != CIECU_OK) {
            ciecu_mixed_destroy(M);
            return status;
        }
    }
    {
        constexpr int s16 = TmaShape<float, short>::SMEM, s32 = TmaShape<float, int>::SMEM;
        int st2 = allow_tma_smem(mixed_spmv_tma_kernel<short, false, false>, s16);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<short, true, false>, s16);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<short, false, true>, s16);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<short, true, true>, s16);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<int, false, false>, s32);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<int, true, false>, s32);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<int, false, true>, s32);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_spmv_tma_kernel<int, true, true>, s32);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_apply_tma_kernel<short>, TmaShape<float, short>::SMEM);
        if (st2 == CIECU_OK) st2 = allow_tma_smem(mixed_apply_tma_kernel<int>, TmaShape<float, int>::SMEM);
        if (st2 != CIECU_OK) {
            ciecu_mixed_destroy(M);
            return st2;
        }
    }
    if (cached != 1000) M->unroll = cached;
    // Autotune the group unroll of the inner SpMV on the solver's own matrix,
    // timing the fused kernel the iteration runs (q = A32 p with the p^T q
    // reduction) on scratch vectors p32 = 0 -> q32.
    if (options.innerKernel != 0)
        M->unroll = options.innerKernel == kDiaInner ? kDiaInner : (options.innerKernel < 0 ? 0 : options.innerKernel);
    if (M->n > 0 && options.innerKernel == 0 && cached == 1000) {
        // p = D^-1 > 0: p^T A p > 0 for an SPD matrix, so no timed launch trips the
        // breakdown flag (which would make the later candidates return at once).
        MixedScalars scratch{};
        scratch.rz = 1.0;
        e = cudaMemcpyAsync(M->d_s, &scratch, sizeof(MixedScalars), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(M->p32, M->dinv32, sizeof(float) * M->n, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && M->z32)  // the fused form gathers z (beta = 0: p = z, q = A z)
            e = cudaMemcpyAsync(M->z32, M->dinv32, sizeof(float) * M->n, cudaMemcpyDeviceToDevice, st);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (e == cudaSuccess) e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        float best = 1e30f, bestTma = 1e30f;
        int bestU = 2;
        for (int u : {1, 2, 4, 0, kDiaInner}) {
            if (e != cudaSuccess) break;
            if (u == kDiaInner && !M->dia32) continue;
            M->unroll = u;
            auto launch = [&]() { launch_inner_spmv<false>(M, st, 0); };
            for (int rep = 0; rep < 2; ++rep) launch();
            for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {  // best of three
                cudaEventRecord(e0, st);
                for (int rep = 0; rep < 3; ++rep) launch();
                cudaEventRecord(e1, st);
                e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
                if (e == cudaSuccess && u == 0 && ms < bestTma) bestTma = ms;
                if (e == cudaSuccess && u != 0 && ms < best) {
                    best = ms;
                    bestU = u;
                }
            }
        }
        count_launch(44);
        // the TMA pipeline competes only when every one of its waits completed
        if (e == cudaSuccess) e = cudaMemcpyAsync(&scratch, M->d_s, sizeof(MixedScalars), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && scratch.tmaError == 0 && scratch.done == 0 && bestTma < best) bestU = 0;
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            ciecu_mixed_destroy(M);
            return cuda_fail(e, "mixed_create: autotune");
        }
        M->unroll = bestU;
        std::lock_guard<std::mutex> lock(g_innerMutex);
        g_innerChoice[key] = bestU;
    }
    *out = M;
    return CIECU_OK;
}

int ciecu_mixed_destroy(ciecu_mixed M) {
    if (!M) return CIECU_OK;
    // No access to M->A (it may already be gone); cudaFree and pool_release
    // synchronise the device.
    if (M->graph) cudaGraphExecDestroy(M->graph);
    if (M->side) cudaStreamDestroy(M->side);
    cudaFree(M->sliceLen);
    cudaFree(M->sliceStart);
    cudaFree(M->rowLen);
    cudaFree(M->val32);
    cudaFree(M->col32or16);
    pool_release({M->dia32, M->dinv32, M->sdiag, M->x32, M->r32, M->p32, M->q32, M->z32, M->r32b, M->p32b,
                  M->q32b, M->x64, M->d_s, M->d_partials, M->d_counter});
    delete M->h_s;
    delete M;
    return CIECU_OK;
}

int ciecu_mixed_info(ciecu_mixed M, int* compressedColumns, int* lanesPerRow) {
    CIECU_REQUIRE(M, "mixed_info: null solver");
    if (compressedColumns) *compressedColumns = M->idx16 ? 1 : 0;
    if (lanesPerRow) *lanesPerRow = M->unroll;  // SELL: one thread per row, `unroll` groups of 4 in flight
    if (M->unroll == 0) {
        // error word of ciecu_mixed_apply_f32's TMA pipeline (sticky)
        unsigned flag = 0;
        cudaStream_t st = M->A->space->stream;
        CIECU_CUDA(cudaMemcpyAsync(&flag, M->d_counter + 3, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (flag) return fail(CIECU_ERR_TIMEOUT, "mixed_apply_f32: a bounded TMA pipeline wait gave up");
    }
    return CIECU_OK;
}

int ciecu_mixed_apply_f32(ciecu_mixed M, const float* d_in, float* d_out) {
    CIECU_REQUIRE(M && (M->n == 0 || (d_in && d_out)), "mixed_apply_f32: null argument");
    if (M->n == 0) return CIECU_OK;
    cudaStream_t st = M->A->space->stream;
    const long need = (M->n + kT - 1) / kT;
    if (M->unroll == kDiaInner) {
        CIECU_TRY(with_diagonals(M->dia.ndiag, [&](auto nd) -> int {
            constexpr int ND = decltype(nd)::value;
            auto* kernel = M->diaTriples ? mixed_apply_dia_kernel<ND, true> : mixed_apply_dia_kernel<ND, false>;
            kernel<<<fit_grid(kernel, kT, (need + 3) / 4), kT, 0, st>>>(M->dia, d_in, d_out);
            return CIECU_OK;
        }));
        count_launch();
        CIECU_CHECK_LAUNCH("mixed_apply_dia_kernel");
        return CIECU_OK;
    }
    if (M->unroll == 0) {
        if (M->idx16) {
            constexpr int smem = TmaShape<float, short>::SMEM;
            mixed_apply_tma_kernel<short><<<fit_grid(mixed_apply_tma_kernel<short>, kTmaWarps * 32, (M->n + 511) / 512,
                                                     smem),
                                            kTmaWarps * 32, smem, st>>>(M->a16, d_in, d_out, M->d_counter + 3);
        } else {
            constexpr int smem = TmaShape<float, int>::SMEM;
            mixed_apply_tma_kernel<int><<<fit_grid(mixed_apply_tma_kernel<int>, kTmaWarps * 32, (M->n + 511) / 512,
                                                   smem),
                                          kTmaWarps * 32, smem, st>>>(M->a32, d_in, d_out, M->d_counter + 3);
        }
        count_launch();
        CIECU_CHECK_LAUNCH("mixed_apply_tma_kernel");
        return CIECU_OK;
    }
    CIECU_TRY(with_unroll(M->unroll, [&](auto uu) -> int {
        constexpr int U = decltype(uu)::value;
        if (M->idx16)
            mixed_apply_kernel<U, short><<<fit_grid(mixed_apply_kernel<U, short>, kT, need), kT, 0, st>>>(M->a16, d_in,
                                                                                                       d_out);
        else
            mixed_apply_kernel<U, int><<<fit_grid(mixed_apply_kernel<U, int>, kT, need), kT, 0, st>>>(M->a32, d_in,
                                                                                                   d_out);
        return CIECU_OK;
    }));
    count_launch();
    CIECU_CHECK_LAUNCH("mixed_apply_kernel");
    return CIECU_OK;
}

int ciecu_mixed_padded_entries(ciecu_mixed M, int64_t* h_entries) {
    CIECU_REQUIRE(M && h_entries, "mixed_padded_entries: null argument");
    *h_entries = M->paddedEntries;
    return CIECU_OK;
}

int ciecu_mixed_dia_info(ciecu_mixed M, int* diagonals, int* triples) {
    CIECU_REQUIRE(M && diagonals && triples, "mixed_dia_info: null argument");
    *diagonals = M->dia32 ? M->dia.ndiag : 0;
    *triples = M->dia32 && M->diaTriples ? 1 : 0;
    return CIECU_OK;
}

int ciecu_mixed_form(ciecu_mixed M, int* kernelsPerIteration) {
    CIECU_REQUIRE(M && kernelsPerIteration, "mixed_form: null argument");
    *kernelsPerIteration = single_pass(M) ? 1 : (M->z32 ? 2 : 3);
    return CIECU_OK;
}

int ciecu_mixed_set_graph_chunk(ciecu_mixed M, int iterations) {
    CIECU_REQUIRE(M && iterations >= 1 && iterations <= 4096, "mixed_set_graph_chunk: chunk must be in [1, 4096]");
    if (M->chunk != iterations && M->graph) {
        cudaGraphExecDestroy(M->graph);
        M->graph = nullptr;
    }
    M->chunk = iterations;
    return CIECU_OK;
}

int ciecu_mixed_product(ciecu_mixed M, double inScale, const double* d_in, double outScale, double* d_out,
                        ciecu_mixed_statistics* h_stats) {
    CIECU_REQUIRE(M, "mixed_product: null solver");
    const long n = M->n;
    CIECU_REQUIRE(n == 0 || (d_in && d_out), "mixed_product: null vector");
    ciecu_csr_s* A = M->A;
    cudaStream_t st = A->space->stream;
    if (n == 0) {
        if (h_stats) *h_stats = ciecu_mixed_statistics{0, 0.0, 0.0, 0, 0, 0.0};
        return CIECU_OK;
    }
    M->b = d_in;
    CIECU_CUDA(cudaMemcpyAsync(M->x64, d_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    ciecu_mixed_statistics stats{0, 1.7976931348623157e308, 1.7976931348623157e308, 0, 0, 1.7976931348623157e308};
    if (M->settings.iterationCount > 0) {
        MixedScalars init{};
        init.maxIter = M->settings.iterationCount;
        init.absTol = M->settings.absoluteResidual;
        init.relTol = M->settings.relativeResidual;
        init.delta = M->options.delta;
        init.mode = M->options.mode;
        init.scaled = M->sdiag ? 1 : 0;
        *M->h_s = init;
        CIECU_CUDA(cudaMemcpyAsync(M->d_s, M->h_s, sizeof(MixedScalars), cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaMemsetAsync(M->x32, 0, sizeof(float) * n, st));
        CIECU_CUDA(cudaMemsetAsync(M->p32, 0, sizeof(float) * n, st));
        const int needR = csr_grid(A, A->kernel);
        CIECU_TRY(with_schedule(A->kernel, [&](auto k) -> int {
            constexpr int K = decltype(k)::value;
            mixed_residual_kernel<K, true, false><<<fit_grid(mixed_residual_kernel<K, true, false>, csr_threads<K>(),
                                                             needR),
                                                    csr_threads<K>(), 0, st>>>(
                A->args<double>(), d_in, M->x64, M->dinv32, M->r32, nullptr, single_pass(M) ? nullptr : M->z32,
                M->sdiag, M->d_s, M->d_partials, M->d_counter, 0);
            return CIECU_OK;
        }));
        if (!M->z32) {  // the fused form's first M1 forms p = z from the z the residual kernel stored
            mixed_direction_kernel<<<fit_grid(mixed_direction_kernel, kT, ((n + 3) / 4 + kT - 1) / kT), kT, 0, st>>>(
                n, M->p32, M->r32, M->dinv32, M->d_s);
            count_launch();
        }
        count_launch();
        CIECU_CHECK_LAUNCH("mixed set-up");
        CIECU_TRY(build_mixed_graph(M));
        const long long limit = M->deviceLoop ? 4096 : M->chunk;
        for (;;) {
            CIECU_CUDA(cudaMemcpyAsync(M->h_s, M->d_s, sizeof(MixedScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            if (M->h_s->done) break;
            const long long before = M->h_s->iter, refBefore = M->h_s->refinements;
            M->h_s->chunkIter = 0;
            M->h_s->chunkLimit = limit;
            CIECU_CUDA(cudaMemcpyAsync(&M->d_s->chunkIter, &M->h_s->chunkIter, 2 * sizeof(long long),
                                       cudaMemcpyHostToDevice, st));
            CIECU_CUDA(cudaGraphLaunch(M->graph, st));
            CIECU_CUDA(cudaMemcpyAsync(M->h_s, M->d_s, sizeof(MixedScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            const long long perIteration = single_pass(M) ? 1 : (M->z32 ? 2 : 3);
            count_launch(M->deviceLoop ? perIteration * (M->h_s->iter - before) + 2LL * (M->h_s->refinements - refBefore)
                                       : (perIteration + 2) * M->chunk);
            if (M->h_s->done) break;
        }
        const MixedScalars& s = *M->h_s;
        if (s.error == CIECU_ERR_TIMEOUT)
            return fail(CIECU_ERR_TIMEOUT, "mixed-precision CG: a bounded TMA pipeline wait gave up");
        if (s.error) {
            if (h_stats) *h_stats = ciecu_mixed_statistics{s.iter, s.absres, s.relres, s.iter, s.refinements, s.relres};
            return fail(CIECU_ERR_BREAKDOWN, "mixed-precision CG breakdown (p^T A p <= 0 or r^T z <= 0) in iteration " +
                                                 std::to_string(s.iter));
        }
        stats = ciecu_mixed_statistics{s.iter, s.absres, s.relres, s.iter, s.refinements, s.relres};
    }
    mixed_output_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, inScale, outScale, M->x64, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("mixed_output_kernel");
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (h_stats) *h_stats = stats;
    return CIECU_OK;
}

}  // extern "C"
