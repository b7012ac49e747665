// Two-level multigrid-preconditioned conjugate gradients, entirely on the device.
//
// One outer iteration (the stopping rule and statistics of
// ConjugateGradients_impl.hpp:49-201):
//   M1  q = A p, p^T q, alpha = r^T z / p^T q
//   M2  x += alpha p, r -= alpha q, ||r|| and the stop decision
//   z = cycle(r):  z = S r;  t = r - A z;  z += P C(R t);  t = r - A z;  z += S t
//   M3  r^T z (and r^T z_old: flexible beta), beta
//   M4  p = z + beta p
// S is a Chebyshev polynomial smoother in D^-1 A (FP64 on the solver's matrix,
// or FP32 on a single-precision copy), C a fixed number of Jacobi-PCG
// iterations on the coarse matrix from zero in the pipelined form (one kernel per
// iteration, on the device scalars, no host round trip).  The body runs under a WHILE conditional node of a CUDA
// graph; M1 / M2 end the loop.  Every reduction is deterministic (per-block
// partials summed in block order by the last block).
#include "ciecu_mg.h"
#include "dia.cuh"
#include "graph.cuh"
#include "pcg.cuh"

#include <cooperative_groups.h>

#include <cmath>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace ciecu {
namespace {

constexpr int kT = 256;

struct MgScalars {
    double rz, pq, alpha, beta, rr, r0, absres, relres, absTol, relTol;
    long long iter, maxIter;
    int done, error, errorKind, flexible;
    long long errorIter, chunkIter, chunkLimit, cycles;
    double cgamma, calpha, cbeta;  // coarse solve
    int cfrozen;
};

template <bool COND>
__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle cond, unsigned value) {
    if constexpr (COND) cudaGraphSetConditional(cond, value);
}

__device__ __forceinline__ bool halted(const MgScalars* s) { return *reinterpret_cast<const volatile int*>(&s->done) != 0; }

// ---- outer iteration -----------------------------------------------------------

struct PqOp {
    using Pre = double;
    const double* __restrict__ p;
    double* __restrict__ q;
    double acc;
    __device__ __forceinline__ double pre(int r) const { return p[r]; }
    __device__ __forceinline__ void post(int r, double pr, double sum) {
        q[r] = sum;
        acc = fma(pr, sum, acc);
    }
};

template <int K, bool COND>
__global__ void __launch_bounds__(csr_threads<K>())
    mg_spmv_kernel(CsrArgs<double> A, const double* __restrict__ p, double* __restrict__ q, MgScalars* s,
                   double* partials, unsigned* counter, cudaGraphConditionalHandle loop) {
    if (halted(s)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond<COND>(loop, 0);
        return;
    }
    PqOp op{p, q, 0.0};
    csr_rows<K, double, double, false>(A, p, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, csr_threads<K>()>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (!(0.0 < tot[0])) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
            s->errorKind = 2;
            s->errorIter = s->iter;
            set_cond<COND>(loop, 0);
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

template <bool COND>
__global__ void __launch_bounds__(kT) mg_update_kernel(long n, double* __restrict__ x, double* __restrict__ r,
                                                       const double* __restrict__ p, const double* __restrict__ q,
                                                       MgScalars* s, double* partials, unsigned* counter,
                                                       cudaGraphConditionalHandle loop) {
    if (halted(s)) return;
    const double alpha = s->alpha;
    double rr = 0.0;
    for (long i = blockIdx.x * static_cast<long>(kT) + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * kT) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        rr = fma(ri, ri, rr);
    }
    double mine[1] = {rr}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->absres = sqrt(tot[0]);
        s->relres = s->absres / s->r0;
        if (float_less(s->absres, s->absTol) || float_less(s->relres, s->relTol)) {
            s->done = 1;
        } else {
            s->iter += 1;
            if (s->iter >= s->maxIter) s->done = 2;
        }
        s->chunkIter += 1;
        set_cond<COND>(loop, (s->done == 0 && s->chunkIter < s->chunkLimit) ? 1u : 0u);
    }
}

// r^T z and r^T z_old (flexible) -> beta; at the start (INIT) r^T z and p = z.
template <bool INIT>
__global__ void __launch_bounds__(kT) mg_beta_kernel(long n, const double* __restrict__ r, const double* __restrict__ z,
                                                     double* __restrict__ zold, double* __restrict__ p, MgScalars* s,
                                                     double* partials, unsigned* counter) {
    if (halted(s)) return;
    double rz = 0.0, rzo = 0.0;
    for (long i = blockIdx.x * static_cast<long>(kT) + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * kT) {
        const double ri = r[i], zi = z[i];
        rz = fma(ri, zi, rz);
        if (!INIT) rzo = fma(ri, zold[i], rzo);
        if (INIT) {
            p[i] = zi;
            zold[i] = zi;
        }
    }
    double mine[2] = {rz, rzo}, tot[2];
    if (grid_reduce_last<2, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        if (!(0.0 < tot[0])) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
            s->errorKind = 1;
            s->errorIter = s->iter;
            return;
        }
        if (!INIT) s->beta = s->flexible ? (tot[0] - tot[1]) / s->rz : tot[0] / s->rz;
        s->rz = tot[0];
    }
}

__global__ void __launch_bounds__(kT) mg_direction_kernel(long n, const double* __restrict__ z, double* __restrict__ p,
                                                          double* __restrict__ zold, const MgScalars* s) {
    if (halted(s)) return;
    const double beta = s->beta;
    for (long i = blockIdx.x * static_cast<long>(kT) + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * kT) {
        const double zi = z[i];
        p[i] = fma(beta, p[i], zi);
        zold[i] = zi;
    }
}

// ||r_0||: the initial residual and the start decision of the reference.
__global__ void __launch_bounds__(kT) mg_init_kernel(long n, const double* __restrict__ r, MgScalars* s,
                                                     double* partials, unsigned* counter) {
    double rr = 0.0;
    for (long i = blockIdx.x * static_cast<long>(kT) + threadIdx.x; i < n; i += static_cast<long>(gridDim.x) * kT)
        rr = fma(r[i], r[i], rr);
    double mine[1] = {rr}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->r0 = sqrt(tot[0]);
        s->absres = s->r0;
        s->relres = 1.0;
        if (float_less(s->absres, s->absTol) || float_less(1.0, s->relTol)) s->done = 1;
        else if (s->maxIter <= 0) s->done = 2;
    }
}

__global__ void mg_output_kernel(long n, double inScale, double outScale, const double* __restrict__ x,
                                 double* __restrict__ out) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        out[i] = combine(inScale, out[i], outScale, x[i]);
}

// ---- Chebyshev smoother (T = double or float vectors and values) ---------------

template <typename T>
__global__ void cheb_first_kernel(long n, const T* __restrict__ in, const T* __restrict__ dinv, T theta,
                                  T* __restrict__ r, T* __restrict__ d, T* __restrict__ x) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const T ri = in[i];
        r[i] = ri;
        const T di = dinv[i] * ri / theta;
        d[i] = di;
        x[i] = di;
    }
}

template <typename T>
struct ChebStep {
    struct Pre {
        T r, d, dinv, x;
    };
    const T* __restrict__ dinv;
    T c1, c2;
    T* __restrict__ r;
    const T* __restrict__ dold;
    T* __restrict__ dnew;
    T* __restrict__ x;
    __device__ __forceinline__ Pre pre(int i) const { return Pre{r[i], dold[i], dinv[i], x[i]}; }
    __device__ __forceinline__ void post(int i, const Pre& p, T sum) const {
        const T ri = p.r - sum;
        r[i] = ri;
        const T di = c1 * p.d + c2 * p.dinv * ri;
        dnew[i] = di;
        x[i] = p.x + di;
    }
};

template <int K, typename T>
__global__ void __launch_bounds__(csr_threads<K>())
    cheb_step_kernel(CsrArgs<T> A, const T* __restrict__ dinv, T c1, T c2, T* __restrict__ r,
                     const T* __restrict__ dold, T* __restrict__ dnew, T* __restrict__ x) {
    ChebStep<T> op{dinv, c1, c2, r, dold, dnew, x};
    csr_rows<K, T, T, false>(A, dold, op);
}

// The FP32 smoother over 16-bit column offsets from the row (6 bytes per entry
// instead of 8): a Chebyshev step and the cycle's residual t = t - A32 z.
template <int VS>
__global__ void __launch_bounds__(kVectorThreads)
    cheb_step16_kernel(CsrArgs<float, short> A, const float* __restrict__ dinv, float c1, float c2,
                       float* __restrict__ r, const float* __restrict__ dold, float* __restrict__ dnew,
                       float* __restrict__ x) {
    ChebStep<float> op{dinv, c1, c2, r, dold, dnew, x};
    vector_rows<float, float, short, VS, kVectorThreads, false>(A, dold, op);
}

struct SubtractOp {  // t = t - A z
    using Pre = float;
    float* __restrict__ t;
    __device__ __forceinline__ float pre(int i) const { return t[i]; }
    __device__ __forceinline__ void post(int i, float ti, float sum) const { t[i] = ti - sum; }
};

template <int VS>
__global__ void __launch_bounds__(kVectorThreads)
    residual16_kernel(CsrArgs<float, short> A, const float* __restrict__ z, float* __restrict__ t) {
    SubtractOp op{t};
    vector_rows<float, float, short, VS, kVectorThreads, false>(A, z, op);
}

// 16-bit offsets col - row of every entry; bad[0] counts offsets outside int16.
__global__ void offsets16_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                 short* __restrict__ out, unsigned* bad) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            const int d = col[k] - r;
            if (d < -32768 || d > 32767) atomicAdd(bad, 1u);
            out[k] = static_cast<short>(d);
        }
}

// Calls f(std::integral_constant<int, VS>) for VS in {4, 8, 16, 32}.
template <typename F>
int with_lanes16(int vs, F&& f) {
    switch (vs) {
        case 4: return f(std::integral_constant<int, 4>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 16: return f(std::integral_constant<int, 16>{});
        default: return f(std::integral_constant<int, 32>{});
    }
}

template <typename T>
__global__ void axpy_out_kernel(long n, const T* __restrict__ x, T* __restrict__ out, int accumulate) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        out[i] = accumulate ? out[i] + x[i] : x[i];
}

template <typename A, typename B>
__global__ void convert_kernel(long n, const A* __restrict__ a, B* __restrict__ b, int accumulate) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        b[i] = accumulate ? static_cast<B>(static_cast<A>(b[i]) + a[i]) : static_cast<B>(a[i]);
}

// ---- coarse solve: a fixed number of Jacobi-PCG iterations from zero ----------
//
// Pipelined form of the preconditioned CG (Ghysels and Vanroose, "Hiding global
// synchronization latency in the preconditioned conjugate gradient algorithm",
// Parallel Computing 40 (2014), Alg. 4): with u = D^-1 r, w = A u, m = D^-1 w and
// n = A m kept by recurrences, the two dot products of an iteration, (r, u) and
// (w, u), come from the same vectors and are reduced together, so an iteration
// is ONE kernel: n = A m, then on the own rows
//   z = n + beta z, q = m + beta q, s = w + beta s, p = u + beta p,
//   x += alpha p, r -= alpha s, u -= alpha q, w -= alpha z, m' = D^-1 w,
// and the partial sums of the next (r, u), (w, u); the last block forms the next
// beta = gamma' / gamma and alpha = gamma' / (delta' - beta gamma' / alpha).  m
// is double-buffered (a block overwrites its rows of m' while other blocks still
// gather m).  In exact arithmetic the iterates are those of the Jacobi-PCG.  A
// non-positive gamma or denominator freezes the solve (alpha = beta = 0: no
// further steps), as converged or broken-down iterations must not move x.

struct CoarseVectors {
    double *x, *r, *u, *w, *z, *q, *s, *p;
    double* m[2];
};

__global__ void __launch_bounds__(kT) coarse_start_kernel(long m, const double* __restrict__ b,
                                                          const double* __restrict__ dinv, CoarseVectors v) {
    for (long i = blockIdx.x * static_cast<long>(kT) + threadIdx.x; i < m; i += static_cast<long>(gridDim.x) * kT) {
        const double bi = b[i];
        v.x[i] = 0.0;
        v.r[i] = bi;
        v.u[i] = dinv[i] * bi;
        v.z[i] = 0.0;
        v.q[i] = 0.0;
        v.s[i] = 0.0;
        v.p[i] = 0.0;
    }
}

// w = A u, m0 = D^-1 w, gamma = (r, u), delta = (w, u) -> the first alpha.
struct CoarseFirstOp {
    struct Pre {
        double r, u, d;
    };
    const double* __restrict__ dinv;
    CoarseVectors v;
    double gamma, delta;
    __device__ __forceinline__ Pre pre(int i) const { return Pre{v.r[i], v.u[i], dinv[i]}; }
    __device__ __forceinline__ void post(int i, const Pre& pr, double sum) {
        v.w[i] = sum;
        v.m[0][i] = pr.d * sum;
        gamma = fma(pr.r, pr.u, gamma);
        delta = fma(sum, pr.u, delta);
    }
};

template <int K>
__global__ void __launch_bounds__(csr_threads<K>())
    coarse_first_kernel(CsrArgs<double> A, const double* __restrict__ dinv, CoarseVectors v, MgScalars* s,
                        double* partials, unsigned* counter) {
    CoarseFirstOp op{dinv, v, 0.0, 0.0};
    csr_rows<K, double, double, false>(A, v.u, op);
    double mine[2] = {op.gamma, op.delta}, tot[2];
    if (grid_reduce_last<2, csr_threads<K>()>(mine, partials, counter, tot) && threadIdx.x == 0) {
        const bool ok = 0.0 < tot[0] && 0.0 < tot[1];
        s->cgamma = tot[0];
        s->calpha = ok ? tot[0] / tot[1] : 0.0;
        s->cbeta = 0.0;
        s->cfrozen = ok ? 0 : 1;
    }
}

struct CoarsePipeOp {
    struct Pre {
        double z, q, s, p, x, r, u, w, m, d;
    };
    const double* __restrict__ dinv;
    CoarseVectors v;
    const double* __restrict__ mcur;
    double* __restrict__ mnext;
    double alpha, beta;
    double gamma, delta;
    __device__ __forceinline__ Pre pre(int i) const {
        return Pre{v.z[i], v.q[i], v.s[i], v.p[i], v.x[i], v.r[i], v.u[i], v.w[i], mcur[i], dinv[i]};
    }
    __device__ __forceinline__ void post(int i, const Pre& a, double n) {
        const double z = fma(beta, a.z, n), q = fma(beta, a.q, a.m), s = fma(beta, a.s, a.w),
                     p = fma(beta, a.p, a.u);
        const double r = fma(-alpha, s, a.r), u = fma(-alpha, q, a.u), w = fma(-alpha, z, a.w);
        v.z[i] = z;
        v.q[i] = q;
        v.s[i] = s;
        v.p[i] = p;
        v.x[i] = fma(alpha, p, a.x);
        v.r[i] = r;
        v.u[i] = u;
        v.w[i] = w;
        mnext[i] = a.d * w;
        gamma = fma(r, u, gamma);
        delta = fma(w, u, delta);
    }
};

template <int K>
__global__ void __launch_bounds__(csr_threads<K>())
    coarse_pipe_kernel(CsrArgs<double> A, const double* __restrict__ dinv, CoarseVectors v, int cur, MgScalars* s,
                       double* partials, unsigned* counter) {
    const volatile MgScalars* vs = s;
    double* const m0 = v.m[0];
    double* const m1 = v.m[1];
    CoarsePipeOp op{dinv, v, cur ? m1 : m0, cur ? m0 : m1, vs->calpha, vs->cbeta, 0.0, 0.0};
    csr_rows<K, double, double, false>(A, op.mcur, op);
    double mine[2] = {op.gamma, op.delta}, tot[2];
    if (grid_reduce_last<2, csr_threads<K>()>(mine, partials, counter, tot) && threadIdx.x == 0) {
        if (s->cfrozen) return;
        const double beta = tot[0] / s->cgamma;
        const double denom = tot[1] - beta * tot[0] / s->calpha;
        if (!(0.0 < tot[0]) || !(0.0 < denom)) {  // converged to rounding or broken down: no further steps
            s->calpha = 0.0;
            s->cbeta = 0.0;
            s->cfrozen = 1;
            return;
        }
        s->cbeta = beta;
        s->calpha = tot[0] / denom;
        s->cgamma = tot[0];
    }
}

// ---- coarse solve in one thread-block cluster ---------------------------------
//
// For a coarse matrix of a structured Q1 stencil (27 diagonals in 3D, 9 in 2D,
// lexicographic order) that is bitwise symmetric, the whole coarse solve runs in
// ONE launch of a cluster of up to 16 CTAs: CTA k owns rows [kC, (k+1)C) and keeps
// in its shared memory
//   - the FP32 upper half U of the matrix (diagonal d holds A[r][r + off[d]]) for
//     rows [kC - H, (k+1)C), H the largest offset, so that the lower entries of
//     its own rows, A[r][r - o] = U_o[r - o], are local too;
//   - the operand u (FP64) for rows [kC - H, (k+1)C + H): its own rows and the
//     halo that the neighbouring CTAs push into it through distributed shared memory.
// The vectors x, r, p, s and D^-1 of the own rows stay in registers (R consecutive
// rows per thread).  The iteration is the Jacobi-PCG in the form of Chronopoulos
// and Gear ("s-step iterative methods for symmetric linear systems", J. Comput.
// Appl. Math. 25 (1989)): with w = A u, both dot products (r, u) and (w, u) of an
// iteration come from the same vectors and are reduced together, and
//   beta = gamma / gamma_old, alpha = gamma / (delta - beta gamma / alpha_old),
//   p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s, u = D^-1 r;
// so an iteration costs one row pass over shared memory and two cluster barriers
// (the reduction, the publication of u).  Its iterates are those of the pipelined
// kernels above in exact arithmetic; the matrix is read in FP32 (the solve is a
// preconditioner), everything else is FP64.  Every CTA forms the cluster-wide
// sums from the per-CTA sums in rank order with the same butterfly, so all
// threads hold bitwise equal scalars and take the same branches: the barrier
// sequence is uniform, and a non-positive gamma or denominator ends the loop in
// every CTA at the same iteration.

constexpr int kClusterThreads = 768;
constexpr int kClusterMaxTriples = 9;
constexpr int kClusterMaxCtas = 16;

struct ClusterCoarse {
    const float* __restrict__ upper;  // diagonal d of U at upper + d * ld
    long ld;
    const double* __restrict__ b;
    const double* __restrict__ dinv;
    double* __restrict__ x;
    int m, rowsPerCta, halo, iterations;
    int center[kClusterMaxTriples];  // triple centres, ascending, centre[NT / 2] = 0
};

// U diagonals of a stencil with NT triples: the main one, offset 1, then the
// upper triples (c - 1, c, c + 1).
template <int NT>
constexpr int cluster_upper_diagonals() {
    return 2 + 3 * (NT / 2);
}

__host__ __device__ constexpr long cluster_align16(long bytes) { return (bytes + 15) / 16 * 16; }

// Shared-memory bytes of a CTA: U rows, operand rows, 32 warp sums x 2 and 2 CTA sums.
__host__ __device__ constexpr long cluster_smem_bytes(int nu, int rowsPerCta, int halo) {
    return cluster_align16(4L * nu * (rowsPerCta + halo)) + 8L * (rowsPerCta + 2L * halo) + 8L * 66;
}

__device__ __forceinline__ double warp_sum_all(double v) {
#pragma unroll
    for (int k = 16; k >= 1; k >>= 1) v += __shfl_xor_sync(0xffffffffu, v, k);
    return v;  // the same bits in every lane: each step adds the same pair in both lanes
}

// Cluster-wide sums of two values, bitwise equal in every thread of every CTA.
__device__ __forceinline__ void cluster_sum2(cooperative_groups::cluster_group& cluster, double v0, double v1,
                                             double* warpSums, double* ctaSums, int nctas, double& t0, double& t1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v0 = warp_sum_all(v0);
    v1 = warp_sum_all(v1);
    if (lane == 0) {
        warpSums[warp] = v0;
        warpSums[32 + warp] = v1;
    }
    __syncthreads();
    if (warp == 0) {
        constexpr int kWarps = kClusterThreads / 32;
        const double a = warp_sum_all(lane < kWarps ? warpSums[lane] : 0.0);
        const double b = warp_sum_all(lane < kWarps ? warpSums[32 + lane] : 0.0);
        if (lane == 0) {
            ctaSums[0] = a;
            ctaSums[1] = b;
        }
    }
    cluster.sync();
    const double a = lane < nctas ? *cluster.map_shared_rank(ctaSums, lane) : 0.0;
    const double b = lane < nctas ? *cluster.map_shared_rank(ctaSums + 1, lane) : 0.0;
    t0 = warp_sum_all(a);
    t1 = warp_sum_all(b);
}

// u of the own rows into the CTA's operand, and into the halo of the neighbours
// whose rows reach them (rows within H of either end of the block).
template <int R>
__device__ __forceinline__ void cluster_publish(cooperative_groups::cluster_group& cluster, double* pe,
                                                const double (&u)[R], int li0, int C, int H, int rank, int nctas) {
    double* prev = rank > 0 ? cluster.map_shared_rank(pe, rank - 1) : nullptr;
    double* next = rank + 1 < nctas ? cluster.map_shared_rank(pe, rank + 1) : nullptr;
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const int li = li0 + j;
        pe[H + li] = u[j];
        if (prev && li < H) prev[C + H + li] = u[j];            // the previous CTA's right halo
        if (next && li >= C - H) next[li - C + H] = u[j];       // the next CTA's left halo
    }
}

// w = A u for the R consecutive own rows starting at operand index e0 (= H + li0;
// U index of those rows is the same): per triple of diagonals the R + 2 operand
// entries are loaded once.  Lower entries are read from U at row r + o.
template <int NT, int R>
__device__ __forceinline__ void cluster_rows(const float* U, int lu, const double* pe, int e0, const int* center,
                                             double (&w)[R]) {
#pragma unroll
    for (int j = 0; j < R; ++j) w[j] = 0.0;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int c = center[t];
        double xv[R + 2];
#pragma unroll
        for (int k = 0; k < R + 2; ++k) xv[k] = pe[e0 + c - 1 + k];
#pragma unroll
        for (int k = 0; k < 3; ++k) {  // offset o = c - 1 + k
#pragma unroll
            for (int j = 0; j < R; ++j) {
                float a;
                if (t < NT / 2)  // o < 0: A[r][r + o] = U_{-o}[r + o], -o = c_mirror + 1 - k
                    a = U[(2 + 3 * (NT / 2 - 1 - t) + (2 - k)) * lu + e0 + j + c - 1 + k];
                else if (t == NT / 2)
                    a = k == 0 ? U[lu + e0 + j - 1] : (k == 1 ? U[e0 + j] : U[lu + e0 + j]);
                else
                    a = U[(2 + 3 * (t - NT / 2 - 1) + k) * lu + e0 + j];
                w[j] = fma(static_cast<double>(a), xv[j + k], w[j]);
            }
        }
    }
}

template <int NT, int R>
__global__ void __launch_bounds__(kClusterThreads, 1) coarse_cluster_kernel(ClusterCoarse a) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    constexpr int NU = cluster_upper_diagonals<NT>();
    extern __shared__ __align__(16) unsigned char smem[];
    const int C = a.rowsPerCta, H = a.halo, lu = C + H, pl = C + 2 * H;
    const int nctas = static_cast<int>(cluster.num_blocks());
    const int rank = static_cast<int>(cluster.block_rank());
    const long start = static_cast<long>(rank) * C;
    float* U = reinterpret_cast<float*>(smem);
    double* pe = reinterpret_cast<double*>(smem + cluster_align16(4L * NU * lu));
    double* warpSums = pe + pl;
    double* ctaSums = warpSums + 64;

    for (int d = 0; d < NU; ++d)
        for (int e = threadIdx.x; e < lu; e += kClusterThreads) {
            const long r = start - H + e;
            U[d * lu + e] = (r >= 0 && r < a.m) ? __ldg(a.upper + d * a.ld + r) : 0.0f;
        }
    for (int e = threadIdx.x; e < pl; e += kClusterThreads) pe[e] = 0.0;
    cluster.sync();  // every CTA has zeroed its operand before any halo is pushed

    const int li0 = R * static_cast<int>(threadIdx.x);
    double xs[R], rs[R], ps[R], ss[R], ds[R], us[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const long row = start + li0 + j;
        const bool in = row < a.m;
        rs[j] = in ? a.b[row] : 0.0;
        ds[j] = in ? a.dinv[row] : 0.0;
        us[j] = ds[j] * rs[j];
        xs[j] = ps[j] = ss[j] = 0.0;
    }
    cluster_publish<R>(cluster, pe, us, li0, C, H, rank, nctas);
    cluster.sync();
    double gammaOld = 0.0, alphaOld = 0.0;
    for (int it = 0; it < a.iterations; ++it) {
        double w[R];
        cluster_rows<NT, R>(U, lu, pe, H + li0, a.center, w);
        double g = 0.0, dl = 0.0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            g = fma(rs[j], us[j], g);
            dl = fma(w[j], us[j], dl);
        }
        cluster_sum2(cluster, g, dl, warpSums, ctaSums, nctas, g, dl);
        const double beta = it == 0 ? 0.0 : g / gammaOld;
        const double den = it == 0 ? dl : dl - beta * g / alphaOld;
        if (!(0.0 < g) || !(0.0 < den)) break;  // converged to rounding or broken down: no further steps
        const double alpha = g / den;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            ps[j] = fma(beta, ps[j], us[j]);
            ss[j] = fma(beta, ss[j], w[j]);
            xs[j] = fma(alpha, ps[j], xs[j]);
            rs[j] = fma(-alpha, ss[j], rs[j]);
            us[j] = ds[j] * rs[j];
        }
        gammaOld = g;
        alphaOld = alpha;
        if (it + 1 == a.iterations) break;
        cluster_publish<R>(cluster, pe, us, li0, C, H, rank, nctas);
        cluster.sync();
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const long row = start + li0 + j;
        if (row < a.m) a.x[row] = xs[j];
    }
    cluster.sync();  // no CTA leaves while another may still read its CTA sums
}

__global__ void count_cycle_kernel(MgScalars* s) { s->cycles += 1; }

}  // namespace
}  // namespace ciecu

struct ciecu_mgcg_s {
    ciecu_csr_s *A = nullptr, *S32 = nullptr, *P = nullptr, *R = nullptr, *Ac = nullptr;
    const double *dinv = nullptr, *dinvc = nullptr;
    ciecu_mg_options options{};
    ciecu_statistics settings{};
    long n = 0, m = 0;
    double lambdaMax = 0.0, lambdaMin = 0.0;
    double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *zold = nullptr, *t = nullptr;
    double* cheb = nullptr;  // 4n (FP64 smoothing)
    float *dinv32 = nullptr, *r32 = nullptr, *z32 = nullptr, *t32 = nullptr, *cheb32 = nullptr;  // FP32 smoothing
    short* col16 = nullptr;  // 16-bit column offsets of the FP32 smoother matrix (when its bandwidth allows)
    int lanes16 = 8;         // lanes per row of the 16-bit-offset smoother kernels (timed at creation)
    double *rc = nullptr, *cx = nullptr, *cr = nullptr, *cz = nullptr, *cp = nullptr, *cq = nullptr;
    double *cu = nullptr, *cw = nullptr, *cs = nullptr, *cm0 = nullptr, *cm1 = nullptr;
    ciecu::MgScalars* d_s = nullptr;
    ciecu::MgScalars* h_s = nullptr;
    double* partials = nullptr;
    unsigned* counter = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool deviceLoop = false;
    // cluster-resident coarse solve (coarse_cluster_kernel): the FP32 DIA copy of the
    // coarse matrix, refilled at every solve, and the launch shape chosen at creation
    float* coarse32 = nullptr;
    ciecu::DiaArgs<float> coarseDia{};
    ciecu::ClusterCoarse cluster{};
    int clusterCtas = 0;  // 0: the coarse matrix's shape rules the cluster form out
    int clusterTriples = 0, clusterRows = 0;
    size_t clusterSmem = 0;
    bool clusterAllowed = true;  // ciecu_mgcg_set_coarse_cluster
    bool clusterActive = false;  // the matrix was bitwise symmetric at the last solve
    bool graphCluster = false;   // the form captured in `graph`
};

namespace ciecu {
namespace {

int grid_of(long n) { return grid_for(n, kT, 8); }

// The FP32 smoother matrix with 16-bit column offsets.
CsrArgs<float, short> args16(const ciecu_mgcg_s* M) {
    const CsrArgs<float> a = M->S32->args<float>();
    return CsrArgs<float, short>{a.rowptr, M->col16, a.val, a.nrows, a.nnz, a.blocks, a.nblocks, nullptr, 0,
                                 a.aligned16};
}

long grid16(const ciecu_mgcg_s* M, int vs) {
    const long rowsPerBlock = kVectorThreads / vs;
    return (M->n + rowsPerBlock - 1) / rowsPerBlock;
}

// t = t - A32 z with the smoother matrix (16-bit offsets when available).
int residual32(ciecu_mgcg_s* M, const float* z, float* t, cudaStream_t st) {
    if (!M->col16) return ciecu_csr_spmv_f32(M->S32, 1.0f, z, -1.0f, t);
    CIECU_TRY(with_lanes16(M->lanes16, [&](auto vv) -> int {
        constexpr int VS = decltype(vv)::value;
        residual16_kernel<VS><<<fit_grid(residual16_kernel<VS>, kVectorThreads, grid16(M, VS)), kVectorThreads, 0,
                                st>>>(args16(M), z, t);
        return CIECU_OK;
    }));
    count_launch();
    CIECU_CHECK_LAUNCH("residual16_kernel");
    return CIECU_OK;
}

// out (+)= S in: Chebyshev polynomial of degree `degree` in D^-1 A applied to in.
template <typename T>
int chebyshev(ciecu_mgcg_s* M, ciecu_csr_s* A, const T* dinv, const T* in, T* out, bool accumulate, T* work,
              cudaStream_t st) {
    const long n = M->n;
    T* r = work;
    T* da = work + n;
    T* db = work + 2 * n;
    T* x = work + 3 * n;
    const double theta = 0.5 * (M->lambdaMax + M->lambdaMin);
    const double delta = 0.5 * (M->lambdaMax - M->lambdaMin);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    cheb_first_kernel<T><<<grid_of(n), kT, 0, st>>>(n, in, dinv, static_cast<T>(theta), r, da, x);
    count_launch();
    const int grid = csr_grid(A, A->kernel);
    for (int k = 1; k < M->options.degree; ++k) {
        const double rhoNew = 1.0 / (2.0 * sigma - rho);
        const T c1 = static_cast<T>(rhoNew * rho), c2 = static_cast<T>(2.0 * rhoNew / delta);
        if constexpr (std::is_same<T, float>::value) {
            if (M->col16) {
                CIECU_TRY(with_lanes16(M->lanes16, [&](auto vv) -> int {
                    constexpr int VS = decltype(vv)::value;
                    cheb_step16_kernel<VS><<<fit_grid(cheb_step16_kernel<VS>, kVectorThreads, grid16(M, VS)),
                                             kVectorThreads, 0, st>>>(args16(M), dinv, c1, c2, r, da, db, x);
                    return CIECU_OK;
                }));
                count_launch();
                std::swap(da, db);
                rho = rhoNew;
                continue;
            }
        }
        CIECU_TRY(with_schedule(A->kernel, [&](auto kk) -> int {
            constexpr int K = decltype(kk)::value;
            cheb_step_kernel<K, T><<<fit_grid(cheb_step_kernel<K, T>, csr_threads<K>(), grid), csr_threads<K>(), 0,
                                     st>>>(A->args<T>(), dinv, c1, c2, r, da, db, x);
            return CIECU_OK;
        }));
        count_launch();
        std::swap(da, db);
        rho = rhoNew;
    }
    axpy_out_kernel<T><<<grid_of(n), kT, 0, st>>>(n, x, out, accumulate ? 1 : 0);
    count_launch();
    return CIECU_OK;
}

using ClusterKernel = void (*)(ClusterCoarse);

ClusterKernel cluster_kernel(int triples, int rows) {
    if (triples == 9) return rows == 1 ? coarse_cluster_kernel<9, 1> : (rows == 3 ? coarse_cluster_kernel<9, 3>
                                                                                 : coarse_cluster_kernel<9, 5>);
    return rows == 1 ? coarse_cluster_kernel<3, 1> : (rows == 3 ? coarse_cluster_kernel<3, 3>
                                                                : coarse_cluster_kernel<3, 5>);
}

cudaLaunchConfig_t cluster_config(const ciecu_mgcg_s* M, cudaStream_t st, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(M->clusterCtas));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = M->clusterSmem;
    cfg.stream = st;
    attr->id = cudaLaunchAttributeClusterDimension;
    attr->val.clusterDim.x = static_cast<unsigned>(M->clusterCtas);
    attr->val.clusterDim.y = 1;
    attr->val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Whether the coarse matrix has the stencil of coarse_cluster_kernel (27 or 9
// diagonals symmetric about 0: the main one, +-1 and triples (c - 1, c, c + 1))
// and fits a cluster: R rows per thread (1, 3 or 5), at most 16 CTAs, a halo
// no wider than a CTA's rows, the shared memory of one CTA.  Then the FP32 DIA
// copy is allocated; otherwise the pipelined kernels stay (clusterCtas = 0).
int prepare_cluster(ciecu_mgcg_s* M, cudaStream_t st) {
    M->clusterCtas = 0;
    if (M->m <= 0) return CIECU_OK;
    const std::vector<int>* offsets = nullptr;
    CIECU_TRY(dia_offsets(M->Ac, &offsets));
    const std::vector<int>& off = *offsets;
    const int nd = static_cast<int>(off.size());
    if (nd != 27 && nd != 9) return CIECU_OK;
    const int h = nd / 2, nt = nd / 3;
    if (off[h] != 0) return CIECU_OK;
    for (int k = 1; k <= h; ++k)
        if (off[h + k] != -off[h - k]) return CIECU_OK;
    const int* up = off.data() + h;  // the h + 1 upper offsets, ascending from 0
    if (up[1] != 1) return CIECU_OK;
    ClusterCoarse a{};
    int last = 1;
    for (int t = 1; t <= nt / 2; ++t) {
        const int* tri = up + 2 + 3 * (t - 1);
        const int c = tri[1];
        if (tri[0] != c - 1 || tri[2] != c + 1 || c - 1 <= last) return CIECU_OK;
        last = c + 1;
        a.center[nt / 2 + t] = c;
        a.center[nt / 2 - t] = -c;
    }
    a.center[nt / 2] = 0;
    const int halo = up[h];
    int dev = 0, maxSmem = 0;
    CIECU_CUDA(cudaGetDevice(&dev));
    CIECU_CUDA(cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int rows = 0, ctas = 0;
    long smem = 0;
    for (int r : {1, 3, 5}) {
        const long c = static_cast<long>(r) * kClusterThreads;
        const long n = (M->m + c - 1) / c;
        if (n > kClusterMaxCtas || (n > 1 && halo > c)) continue;
        smem = cluster_smem_bytes(h + 1, static_cast<int>(c), halo);
        if (smem > maxSmem) break;  // more rows per CTA only need more
        rows = r;
        ctas = static_cast<int>(n);
        break;
    }
    if (!rows) return CIECU_OK;
    const ClusterKernel kern = cluster_kernel(nt, rows);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e == cudaSuccess && ctas > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    int clusters = 0;
    if (e == cudaSuccess) {
        M->clusterCtas = ctas;
        M->clusterSmem = static_cast<size_t>(smem);
        cudaLaunchAttribute attr{};
        const cudaLaunchConfig_t cfg = cluster_config(M, st, &attr);
        e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg);
        M->clusterCtas = 0;
    }
    if (e != cudaSuccess || clusters < 1) {
        cudaGetLastError();  // no such cluster on this device: the pipelined kernels stay
        return CIECU_OK;
    }
    DiaArgs<float> full = dia_shape<float>(M->Ac, off);
    const size_t bytes = sizeof(float) * static_cast<size_t>(full.ndiag) * static_cast<size_t>(full.ld);
    if (cudaMalloc(&M->coarse32, bytes) != cudaSuccess) {
        cudaGetLastError();
        M->coarse32 = nullptr;
        return CIECU_OK;
    }
    CIECU_CUDA(cudaMemsetAsync(M->coarse32, 0, bytes, st));
    full.val = M->coarse32;
    M->coarseDia = full;
    a.upper = M->coarse32 + static_cast<long>(h) * full.ld;
    a.ld = full.ld;
    a.b = M->rc;
    a.dinv = M->dinvc;
    a.x = M->cx;
    a.m = static_cast<int>(M->m);
    a.rowsPerCta = rows * kClusterThreads;
    a.halo = halo;
    a.iterations = M->options.coarseIterations;
    M->cluster = a;
    M->clusterCtas = ctas;
    M->clusterTriples = nt;
    M->clusterRows = rows;
    M->clusterSmem = static_cast<size_t>(smem);
    return CIECU_OK;
}

// At every solve: the coarse values into the FP32 copy, and whether they are
// bitwise symmetric (the cluster kernel reads the upper half only).
int refresh_cluster(ciecu_mgcg_s* M, cudaStream_t st) {
    M->clusterActive = false;
    if (!M->clusterCtas || !M->clusterAllowed) return CIECU_OK;
    CIECU_TRY(dia_fill_f32(M->Ac, M->coarseDia, M->coarse32, nullptr, st));
    bool sym = false;
    CIECU_TRY(dia_symmetric<float>(M->coarseDia, st, reinterpret_cast<unsigned*>(M->Ac->space->d_result), &sym));
    M->clusterActive = sym;
    return CIECU_OK;
}

// ec = C rc: coarseIterations Jacobi-PCG iterations from zero, result in M->cx:
// one cluster launch when the coarse matrix allows it, else the pipelined form
// (one kernel per iteration).
int coarse_solve(ciecu_mgcg_s* M, cudaStream_t st) {
    if (M->clusterActive) {
        cudaLaunchAttribute attr{};
        const cudaLaunchConfig_t cfg = cluster_config(M, st, &attr);
        const cudaError_t e =
            cudaLaunchKernelEx(&cfg, cluster_kernel(M->clusterTriples, M->clusterRows), M->cluster);
        count_launch();
        if (e != cudaSuccess) return cuda_fail(e, "coarse_cluster_kernel launch");
        return CIECU_OK;
    }
    const long m = M->m;
    ciecu_csr_s* Ac = M->Ac;
    const CoarseVectors v{M->cx, M->cr, M->cu, M->cw, M->cz, M->cq, M->cs, M->cp, {M->cm0, M->cm1}};
    coarse_start_kernel<<<grid_of(m), kT, 0, st>>>(m, M->rc, M->dinvc, v);
    count_launch();
    const int grid = csr_grid(Ac, Ac->kernel);
    return with_schedule(Ac->kernel, [&](auto kk) -> int {
        constexpr int K = decltype(kk)::value;
        coarse_first_kernel<K><<<fit_grid(coarse_first_kernel<K>, csr_threads<K>(), grid), csr_threads<K>(), 0,
                                 st>>>(Ac->args<double>(), M->dinvc, v, M->d_s, M->partials, M->counter);
        const int g = fit_grid(coarse_pipe_kernel<K>, csr_threads<K>(), grid);
        for (int it = 0; it < M->options.coarseIterations; ++it)
            coarse_pipe_kernel<K><<<g, csr_threads<K>(), 0, st>>>(Ac->args<double>(), M->dinvc, v, it & 1, M->d_s,
                                                                 M->partials, M->counter);
        count_launch(1 + M->options.coarseIterations);
        return CIECU_OK;
    });
}

// z = cycle(r) (the symmetric two-level cycle).
int cycle(ciecu_mgcg_s* M, cudaStream_t st) {
    const long n = M->n;
    ciecu_csr_s* A = M->A;
    if (!M->S32) {
        CIECU_TRY(chebyshev<double>(M, A, M->dinv, M->r, M->z, false, M->cheb, st));
        CIECU_CUDA(cudaMemcpyAsync(M->t, M->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(ciecu_csr_spmv_f64(A, 1.0, M->z, -1.0, M->t));  // t = r - A z
        CIECU_TRY(ciecu_csr_spmv_f64(M->R, 0.0, M->t, 1.0, M->rc));
        CIECU_TRY(coarse_solve(M, st));
        CIECU_TRY(ciecu_csr_spmv_f64(M->P, 1.0, M->cx, 1.0, M->z));
        CIECU_CUDA(cudaMemcpyAsync(M->t, M->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(ciecu_csr_spmv_f64(A, 1.0, M->z, -1.0, M->t));
        CIECU_TRY(chebyshev<double>(M, A, M->dinv, M->t, M->z, true, M->cheb, st));
    } else {
        ciecu_csr_s* S = M->S32;
        convert_kernel<double, float><<<grid_of(n), kT, 0, st>>>(n, M->r, M->r32, 0);
        count_launch();
        CIECU_TRY(chebyshev<float>(M, S, M->dinv32, M->r32, M->z32, false, M->cheb32, st));
        CIECU_CUDA(cudaMemcpyAsync(M->t32, M->r32, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(residual32(M, M->z32, M->t32, st));  // t = r - A32 z (FP32)
        convert_kernel<float, double><<<grid_of(n), kT, 0, st>>>(n, M->t32, M->t, 0);
        count_launch();
        CIECU_TRY(ciecu_csr_spmv_f64(M->R, 0.0, M->t, 1.0, M->rc));
        CIECU_TRY(coarse_solve(M, st));
        CIECU_TRY(ciecu_csr_spmv_f64(M->P, 0.0, M->cx, 1.0, M->t));  // t = P ec
        convert_kernel<double, float><<<grid_of(n), kT, 0, st>>>(n, M->t, M->z32, 1);
        count_launch();
        CIECU_CUDA(cudaMemcpyAsync(M->t32, M->r32, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(residual32(M, M->z32, M->t32, st));
        CIECU_TRY(chebyshev<float>(M, S, M->dinv32, M->t32, M->z32, true, M->cheb32, st));
        convert_kernel<float, double><<<grid_of(n), kT, 0, st>>>(n, M->z32, M->z, 0);
        count_launch();
    }
    count_cycle_kernel<<<1, 1, 0, st>>>(M->d_s);
    count_launch();
    CIECU_CHECK_LAUNCH("two-level cycle");
    return CIECU_OK;
}

template <bool COND>
int iteration(ciecu_mgcg_s* M, cudaStream_t st, cudaGraphConditionalHandle loop) {
    const long n = M->n;
    ciecu_csr_s* A = M->A;
    const int grid = csr_grid(A, A->kernel);
    CIECU_TRY(with_schedule(A->kernel, [&](auto kk) -> int {
        constexpr int K = decltype(kk)::value;
        mg_spmv_kernel<K, COND><<<fit_grid(mg_spmv_kernel<K, COND>, csr_threads<K>(), grid), csr_threads<K>(), 0,
                                  st>>>(A->args<double>(), M->p, M->q, M->d_s, M->partials, M->counter, loop);
        return CIECU_OK;
    }));
    mg_update_kernel<COND><<<grid_of(n), kT, 0, st>>>(n, M->x, M->r, M->p, M->q, M->d_s, M->partials, M->counter,
                                                      loop);
    count_launch(2);
    CIECU_TRY(cycle(M, st));
    mg_beta_kernel<false><<<grid_of(n), kT, 0, st>>>(n, M->r, M->z, M->zold, M->p, M->d_s, M->partials, M->counter);
    mg_direction_kernel<<<grid_of(n), kT, 0, st>>>(n, M->z, M->p, M->zold, M->d_s);
    count_launch(2);
    CIECU_CHECK_LAUNCH("two-level CG iteration");
    return CIECU_OK;
}

int build_graph(ciecu_mgcg_s* M) {
    if (M->graph) return CIECU_OK;
    cudaStream_t st = M->A->space->stream;
    int status = CIECU_ERR_ARGUMENT;
    if (device_loop_enabled())
        status = build_while_graph(st, [&](cudaGraph_t, cudaGraphConditionalHandle loop) {
            return iteration<true>(M, st, loop);
        }, &M->graph);
    if (status == CIECU_OK) {
        M->deviceLoop = true;
        M->graphCluster = M->clusterActive;
        return CIECU_OK;
    }
    cudaGetLastError();
    M->deviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    status = iteration<false>(M, st, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "two-level CG graph capture");
    e = cudaGraphInstantiate(&M->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "two-level CG graph instantiate");
    M->graphCluster = M->clusterActive;
    return CIECU_OK;
}

__global__ void to_f32_kernel(long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        b[i] = static_cast<float>(a[i]);
}

// 16-bit column offsets of the FP32 smoother matrix when every |col - row| fits,
// and the lanes per row of its kernels (the residual kernel timed, best of
// three, on scratch vectors); otherwise the smoother keeps the int32 columns.
int prepare_offsets16(ciecu_mgcg_s* M, cudaStream_t st) {
    ciecu_csr_s* S = M->S32;
    if (S->nnz <= 0) return CIECU_OK;
    unsigned* d_bad = reinterpret_cast<unsigned*>(S->space->d_result);
    unsigned bad = 0;
    if (cudaMalloc(&M->col16, sizeof(short) * static_cast<size_t>(S->nnz)) != cudaSuccess) {
        cudaGetLastError();  // no room: int32 columns
        M->col16 = nullptr;
        return CIECU_OK;
    }
    CIECU_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), st));
    offsets16_kernel<<<grid_for(M->n, 256, 8), 256, 0, st>>>(static_cast<int>(M->n), S->rowptr, S->col, M->col16,
                                                             d_bad);
    count_launch();
    CIECU_CHECK_LAUNCH("offsets16_kernel");
    CIECU_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (bad) {
        cudaFree(M->col16);
        M->col16 = nullptr;
        return CIECU_OK;
    }
    // t32 / z32 as scratch (the solve overwrites both)
    CIECU_CUDA(cudaMemsetAsync(M->z32, 0, sizeof(float) * M->n, st));
    cudaEvent_t e0, e1;
    CIECU_CUDA(cudaEventCreate(&e0));
    CIECU_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestLanes = 8;
    cudaError_t e = cudaSuccess;
    for (int vs : {4, 8, 16, 32}) {
        M->lanes16 = vs;
        for (int trial = 0; trial < 4 && e == cudaSuccess; ++trial) {
            cudaEventRecord(e0, st);
            residual32(M, M->z32, M->t32, st);
            cudaEventRecord(e1, st);
            e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
            if (trial > 0 && e == cudaSuccess && ms < best) {  // the first run warms up
                best = ms;
                bestLanes = vs;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "mgcg_create: smoother kernel choice");
    M->lanes16 = bestLanes;
    return CIECU_OK;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_mgcg_destroy(ciecu_mgcg M) {
    if (!M) return CIECU_OK;
    if (M->graph) cudaGraphExecDestroy(M->graph);
    for (double* v : {M->x, M->r, M->p, M->q, M->z, M->zold, M->t, M->cheb, M->rc, M->cx, M->cr, M->cz, M->cp, M->cq,
                      M->cu, M->cw, M->cs, M->cm0, M->cm1, M->partials})
        cudaFree(v);
    for (float* v : {M->dinv32, M->r32, M->z32, M->t32, M->cheb32}) cudaFree(v);
    cudaFree(M->col16);
    cudaFree(M->coarse32);
    cudaFree(M->d_s);
    cudaFree(M->counter);
    if (M->h_s) cudaFreeHost(M->h_s);
    delete M;
    return CIECU_OK;
}

int ciecu_mgcg_create(ciecu_csr fine, const double* d_fineInverseDiagonal, ciecu_csr smoother32,
                      ciecu_csr prolongation, ciecu_csr restriction, ciecu_csr coarse,
                      const double* d_coarseInverseDiagonal, ciecu_mg_options options, ciecu_statistics settings,
                      ciecu_mgcg* out) {
    CIECU_REQUIRE(fine && d_fineInverseDiagonal && prolongation && restriction && coarse && d_coarseInverseDiagonal &&
                      out,
                  "mgcg_create: null argument");
    CIECU_REQUIRE(fine->valueType == CIECU_F64 && fine->rows == fine->cols, "mgcg_create: square FP64 fine matrix");
    CIECU_REQUIRE(coarse->valueType == CIECU_F64 && coarse->rows == coarse->cols,
                  "mgcg_create: square FP64 coarse matrix");
    CIECU_REQUIRE(prolongation->valueType == CIECU_F64 && prolongation->rows == fine->rows &&
                      prolongation->cols == coarse->rows,
                  "mgcg_create: prolongation must be FP64, fine rows x coarse rows");
    CIECU_REQUIRE(restriction->valueType == CIECU_F64 && restriction->rows == coarse->rows &&
                      restriction->cols == fine->rows,
                  "mgcg_create: restriction must be FP64, coarse rows x fine rows");
    CIECU_REQUIRE(!smoother32 || (smoother32->valueType == CIECU_F32 && smoother32->rows == fine->rows &&
                                  smoother32->cols == fine->cols),
                  "mgcg_create: the FP32 smoother matrix must be FP32 and of the fine matrix's shape");
    CIECU_REQUIRE(prolongation->space == fine->space && restriction->space == fine->space &&
                      coarse->space == fine->space && (!smoother32 || smoother32->space == fine->space),
                  "mgcg_create: every matrix must belong to the fine matrix's space");
    CIECU_REQUIRE(options.degree >= 1 && options.degree <= 64, "mgcg_create: degree in [1, 64]");
    CIECU_REQUIRE(options.coarseIterations >= 1 && options.coarseIterations <= 1000,
                  "mgcg_create: coarse iterations in [1, 1000]");
    CIECU_REQUIRE(options.ratio > 1.0, "mgcg_create: ratio must exceed 1");
    CIECU_TRY(ensure_tuned(fine));
    CIECU_TRY(ensure_tuned(coarse));
    CIECU_TRY(ensure_tuned(prolongation));
    CIECU_TRY(ensure_tuned(restriction));
    if (smoother32) CIECU_TRY(ensure_tuned(smoother32));
    auto* M = new ciecu_mgcg_s();
    M->A = fine;
    M->S32 = smoother32;
    M->P = prolongation;
    M->R = restriction;
    M->Ac = coarse;
    M->dinv = d_fineInverseDiagonal;
    M->dinvc = d_coarseInverseDiagonal;
    M->options = options;
    M->settings = settings;
    M->n = fine->rows;
    M->m = coarse->rows;
    const size_t n = static_cast<size_t>(std::max<long>(M->n, 1)), m = static_cast<size_t>(std::max<long>(M->m, 1));
    cudaStream_t st = fine->space->stream;
    cudaError_t e = cudaSuccess;
    for (double** v : {&M->x, &M->r, &M->p, &M->q, &M->z, &M->zold, &M->t})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(double) * n);
    for (double** v : {&M->rc, &M->cx, &M->cr, &M->cz, &M->cp, &M->cq, &M->cu, &M->cw, &M->cs, &M->cm0, &M->cm1})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(double) * m);
    if (e == cudaSuccess && !smoother32) e = cudaMalloc(&M->cheb, sizeof(double) * 4 * n);
    if (e == cudaSuccess && smoother32) {
        for (float** v : {&M->dinv32, &M->r32, &M->z32, &M->t32})
            if (e == cudaSuccess) e = cudaMalloc(v, sizeof(float) * n);
        if (e == cudaSuccess) e = cudaMalloc(&M->cheb32, sizeof(float) * 4 * n);
    }
    if (e == cudaSuccess) e = cudaMalloc(&M->partials, sizeof(double) * 2 * kMaxPartials);
    if (e == cudaSuccess) e = cudaMalloc(&M->counter, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->counter, 0, sizeof(unsigned) * 4, st);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_s, sizeof(MgScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&M->h_s, sizeof(MgScalars));
    if (e != cudaSuccess) {
        ciecu_mgcg_destroy(M);
        return cuda_fail(e, "mgcg_create: allocation");
    }
    if (smoother32 && M->n > 0) {
        to_f32_kernel<<<grid_of(M->n), kT, 0, st>>>(M->n, d_fineInverseDiagonal, M->dinv32);
        count_launch();
        const int status = prepare_offsets16(M, st);
        if (status != CIECU_OK) {
            ciecu_mgcg_destroy(M);
            return status;
        }
    }
    {
        const int status = prepare_cluster(M, st);
        if (status != CIECU_OK) {
            ciecu_mgcg_destroy(M);
            return status;
        }
    }
    M->lambdaMax = options.lambdaMax;
    if (!(M->lambdaMax > 0.0) && M->n > 0) {
        double lam = 0.0;
        // 2n doubles of work: the FP64 Chebyshev buffer, or the FP32 one (4n floats)
        double* work = M->cheb ? M->cheb : reinterpret_cast<double*>(M->cheb32);
        const int status = ciecu_power_lambda_max_f64(fine, d_fineInverseDiagonal, 20, 0, work, &lam);
        if (status != CIECU_OK) {
            ciecu_mgcg_destroy(M);
            return status;
        }
        M->lambdaMax = 1.1 * lam;
    }
    M->lambdaMin = M->lambdaMax / options.ratio;
    *out = M;
    return CIECU_OK;
}

int ciecu_mgcg_product(ciecu_mgcg M, double inScale, const double* d_in, double outScale, double* d_out,
                       ciecu_statistics* h_stats) {
    CIECU_REQUIRE(M, "mgcg_product: null solver");
    const long n = M->n;
    CIECU_REQUIRE(n == 0 || (d_in && d_out), "mgcg_product: null vector");
    cudaStream_t st = M->A->space->stream;
    ciecu_statistics stats{0, 1.7976931348623157e308, 1.7976931348623157e308};
    if (n == 0) {
        if (h_stats) *h_stats = ciecu_statistics{0, 0.0, 0.0};
        return CIECU_OK;
    }
    CIECU_CUDA(cudaMemcpyAsync(M->x, d_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    if (M->settings.iterationCount > 0) {
        CIECU_TRY(refresh_cluster(M, st));
        if (M->graph && M->graphCluster != M->clusterActive) {  // the coarse form changed: capture again
            cudaGraphExecDestroy(M->graph);
            M->graph = nullptr;
        }
        MgScalars init{};
        init.maxIter = M->settings.iterationCount;
        init.absTol = M->settings.absoluteResidual;
        init.relTol = M->settings.relativeResidual;
        init.flexible = M->options.flexible ? 1 : 0;
        *M->h_s = init;
        CIECU_CUDA(cudaMemcpyAsync(M->d_s, M->h_s, sizeof(MgScalars), cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaMemcpyAsync(M->r, d_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(ciecu_csr_spmv_f64(M->A, 1.0, M->x, -1.0, M->r));  // r = b - A x
        mg_init_kernel<<<grid_of(n), kT, 0, st>>>(n, M->r, M->d_s, M->partials, M->counter);
        count_launch();
        CIECU_TRY(cycle(M, st));
        mg_beta_kernel<true><<<grid_of(n), kT, 0, st>>>(n, M->r, M->z, M->zold, M->p, M->d_s, M->partials,
                                                        M->counter);
        count_launch();
        CIECU_CHECK_LAUNCH("two-level CG set-up");
        CIECU_TRY(build_graph(M));
        const long long limit = M->deviceLoop ? (1LL << 20) : 1;
        for (;;) {
            CIECU_CUDA(cudaMemcpyAsync(M->h_s, M->d_s, sizeof(MgScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            if (M->h_s->done) break;
            M->h_s->chunkIter = 0;
            M->h_s->chunkLimit = limit;
            CIECU_CUDA(cudaMemcpyAsync(&M->d_s->chunkIter, &M->h_s->chunkIter, 2 * sizeof(long long),
                                       cudaMemcpyHostToDevice, st));
            CIECU_CUDA(cudaGraphLaunch(M->graph, st));
        }
        const MgScalars& s = *M->h_s;
        if (s.error) {
            if (h_stats) *h_stats = ciecu_statistics{s.errorIter, s.absres, s.relres};
            if (s.errorKind == 1)
                return fail(CIECU_ERR_BREAKDOWN, "preconditioned norm vanished in iteration " +
                                                     std::to_string(s.errorIter) + " (r^T @ z <= 0)");
            return fail(CIECU_ERR_BREAKDOWN, "p^T @ A @ p vanished in iteration " + std::to_string(s.errorIter));
        }
        stats = ciecu_statistics{s.iter, s.absres, s.relres};
    }
    mg_output_kernel<<<grid_of(n), kT, 0, st>>>(n, inScale, outScale, M->x, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("mg_output_kernel");
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (h_stats) *h_stats = stats;
    return CIECU_OK;
}

int ciecu_mgcg_smoother_info(ciecu_mgcg M, int* offsets16, int* lanesPerRow) {
    CIECU_REQUIRE(M && offsets16 && lanesPerRow, "mgcg_smoother_info: null argument");
    *offsets16 = M->col16 ? 1 : 0;
    *lanesPerRow = M->col16 ? M->lanes16 : 0;
    return CIECU_OK;
}

int ciecu_mgcg_coarse_apply(ciecu_mgcg M, const double* d_in, double* d_out) {
    CIECU_REQUIRE(M, "mgcg_coarse_apply: null solver");
    CIECU_REQUIRE(M->m == 0 || (d_in && d_out), "mgcg_coarse_apply: null vector");
    if (M->m == 0) return CIECU_OK;
    cudaStream_t st = M->A->space->stream;
    CIECU_TRY(refresh_cluster(M, st));
    CIECU_CUDA(cudaMemcpyAsync(M->rc, d_in, sizeof(double) * M->m, cudaMemcpyDeviceToDevice, st));
    CIECU_TRY(coarse_solve(M, st));
    CIECU_CHECK_LAUNCH("coarse solve");
    CIECU_CUDA(cudaMemcpyAsync(d_out, M->cx, sizeof(double) * M->m, cudaMemcpyDeviceToDevice, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    return CIECU_OK;
}

int ciecu_mgcg_set_coarse_cluster(ciecu_mgcg M, int enable) {
    CIECU_REQUIRE(M, "mgcg_set_coarse_cluster: null solver");
    M->clusterAllowed = enable != 0;
    return CIECU_OK;
}

int ciecu_mgcg_coarse_info(ciecu_mgcg M, int* clusterCtas, int* active) {
    CIECU_REQUIRE(M && clusterCtas && active, "mgcg_coarse_info: null argument");
    *clusterCtas = M->clusterCtas;
    *active = M->clusterActive ? 1 : 0;
    return CIECU_OK;
}

int ciecu_mgcg_info(ciecu_mgcg M, double* h_lambdaMax, int64_t* h_cycles) {
    CIECU_REQUIRE(M, "mgcg_info: null solver");
    if (h_lambdaMax) *h_lambdaMax = M->lambdaMax;
    if (h_cycles) *h_cycles = M->h_s ? M->h_s->cycles : 0;
    return CIECU_OK;
}

}  // extern "C"
