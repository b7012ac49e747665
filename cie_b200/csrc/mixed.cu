// Mixed-precision Jacobi-PCG: FP32 inner iterations, FP64 refinement.
//
// No reference counterpart (the reference solves in one precision,
// ConjugateGradients_impl.hpp:49-201); the inner iteration is that algorithm in
// FP32 and the FP64 part is defect correction:
//
//   FP64 (kept on the GPU only here): the solution x64, the residual
//        r = b - A64 x64 recomputed with the FP64 matrix, and every dot-product
//        accumulator (the FP32 vectors are reduced in double).
//   FP32: the matrix values (a converted copy), the vectors r, p, q, x-increment
//        and the inverse diagonal.  Column indices are stored as 16-bit offsets
//        from the row (col - row) when the matrix bandwidth allows -- a lossless,
//        checked re-encoding of the int32 CSR that halves the index bytes.
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
// M3 direction); the two refinement kernels (R1 fold, R2 FP64 residual) are in
// the same CUDA graph and return at once unless M2 asked for a replacement.
#include "ciecu_mixed.h"
#include "pcg.cuh"

#include <string>

namespace ciecu {
namespace {

constexpr int kT = 256;

struct MixedScalars {
    double rz, pq, alpha, beta, rzPending;
    double r0, absres, relres, rnorm;  // true residual norms
    double sloppy;                      // FP32 residual norm of the last iteration
    double maxrx, maxrr, cycleStart;
    double absTol, relTol, delta;
    long long iter, maxIter, refinements;
    int done, error, update, updateX, mode, pad;
};

// ---- compressed FP32 matrix ---------------------------------------------------

__global__ void compress_kernel(int nrows, const int* __restrict__ rowptr, const int* __restrict__ col,
                                const double* __restrict__ val, float* __restrict__ val32,
                                short* __restrict__ col16, unsigned* tooFar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
        for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            val32[k] = static_cast<float>(val[k]);
            const int off = col[k] - r;
            if (col16) {
                if (off < -32768 || off > 32767) atomicOr(tooFar, 1u);
                col16[k] = static_cast<short>(off);
            }
        }
    }
}

// Row sums over the FP32 matrix, VS lanes per row, UNROLL strided entries per
// lane loaded before the FMA chain.  IDX16: columns are 16-bit row offsets.
template <int VS, bool IDX16, typename Op>
__device__ __forceinline__ void f32_rows(int nrows, const int* __restrict__ rowptr, const void* __restrict__ colv,
                                         const float* __restrict__ val, const float* __restrict__ x, Op& op) {
    constexpr int ROWS_PER_WARP = 32 / VS;
    constexpr int UNROLL = VS <= 4 ? 8 : 4;
    const int lane = threadIdx.x & 31;
    const int sub = lane % VS;
    const long warpGlobal = (static_cast<long>(blockIdx.x) * kT + threadIdx.x) >> 5;
    const long warps = (static_cast<long>(gridDim.x) * kT) >> 5;
    const long groups = (nrows + ROWS_PER_WARP - 1) / ROWS_PER_WARP;
    const short* col16 = static_cast<const short*>(colv);
    const int* col32 = static_cast<const int*>(colv);
    for (long g = warpGlobal; g < groups; g += warps) {
        const long rowL = g * ROWS_PER_WARP + lane / VS;
        const bool valid = rowL < nrows;
        const int r = valid ? static_cast<int>(rowL) : 0;
        float sum = 0.0f;
        if (valid) {
            const int k1 = rowptr[r + 1];
            for (int k = rowptr[r] + sub; k < k1; k += UNROLL * VS) {
                float v[UNROLL];
                int c[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) {
                    const int kk = k + u * VS;
                    const bool in = kk < k1;
                    v[u] = in ? __ldg(val + kk) : 0.0f;
                    if (IDX16) c[u] = in ? r + static_cast<int>(__ldg(col16 + kk)) : -1;
                    else c[u] = in ? __ldg(col32 + kk) : -1;
                }
                float xv[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : 0.0f;
#pragma unroll
                for (int u = 0; u < UNROLL; ++u) sum = fmaf(v[u], xv[u], sum);
            }
        }
#pragma unroll
        for (int offset = VS / 2; offset > 0; offset >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, offset, VS);
        if (valid && sub == 0) op(r, sum);
    }
}

// out = A32 in (the inner operator on its own).
template <int VS, bool IDX16>
__global__ void __launch_bounds__(kT) mixed_apply_kernel(int nrows, const int* __restrict__ rowptr,
                                                         const void* __restrict__ col, const float* __restrict__ val,
                                                         const float* __restrict__ x, float* __restrict__ y) {
    auto op = [&](int r, float sum) { y[r] = sum; };
    f32_rows<VS, IDX16>(nrows, rowptr, col, val, x, op);
}

// M1: q = A32 p, p^T q (FP64 accumulation), alpha.
template <int VS, bool IDX16>
__global__ void __launch_bounds__(kT) mixed_spmv_kernel(int nrows, const int* __restrict__ rowptr,
                                                        const void* __restrict__ col, const float* __restrict__ val,
                                                        const float* __restrict__ p, float* __restrict__ q,
                                                        MixedScalars* s, double* partials, unsigned* counter) {
    if (*reinterpret_cast<volatile int*>(&s->done)) return;
    double acc = 0.0;
    auto op = [&](int r, float sum) {
        q[r] = sum;
        acc = fma(static_cast<double>(p[r]), static_cast<double>(sum), acc);
    };
    f32_rows<VS, IDX16>(nrows, rowptr, col, val, p, op);
    double mine[1] = {acc}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (!(0.0 < tot[0])) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// M2: x32 += alpha p; r32 -= alpha q; rr, rz in FP64; replacement decision.
__global__ void __launch_bounds__(kT) mixed_update_kernel(long n, float* __restrict__ x, float* __restrict__ r,
                                                          const float* __restrict__ p, const float* __restrict__ q,
                                                          const float* __restrict__ dinv, MixedScalars* s,
                                                          double* partials, unsigned* counter) {
    if (*reinterpret_cast<volatile int*>(&s->done)) return;
    const float alpha = static_cast<float>(s->alpha);
    double rr = 0.0, rz = 0.0;
    const long quads = n >> 2;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long j = static_cast<long>(blockIdx.x) * kT + threadIdx.x; j < quads; j += stride) {
        const float4 pj = reinterpret_cast<const float4*>(p)[j];
        const float4 qj = reinterpret_cast<const float4*>(q)[j];
        const float4 dj = reinterpret_cast<const float4*>(dinv)[j];
        float4 xj = reinterpret_cast<const float4*>(x)[j];
        float4 rj = reinterpret_cast<const float4*>(r)[j];
        xj.x = fmaf(alpha, pj.x, xj.x); xj.y = fmaf(alpha, pj.y, xj.y);
        xj.z = fmaf(alpha, pj.z, xj.z); xj.w = fmaf(alpha, pj.w, xj.w);
        rj.x = fmaf(-alpha, qj.x, rj.x); rj.y = fmaf(-alpha, qj.y, rj.y);
        rj.z = fmaf(-alpha, qj.z, rj.z); rj.w = fmaf(-alpha, qj.w, rj.w);
        reinterpret_cast<float4*>(x)[j] = xj;
        reinterpret_cast<float4*>(r)[j] = rj;
        rr = fma(double(rj.x), double(rj.x), rr); rr = fma(double(rj.y), double(rj.y), rr);
        rr = fma(double(rj.z), double(rj.z), rr); rr = fma(double(rj.w), double(rj.w), rr);
        rz = fma(double(rj.x), double(rj.x * dj.x), rz); rz = fma(double(rj.y), double(rj.y * dj.y), rz);
        rz = fma(double(rj.z), double(rj.z * dj.z), rz); rz = fma(double(rj.w), double(rj.w * dj.w), rz);
    }
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
        const long i = (quads << 2) + threadIdx.x;
        x[i] = fmaf(alpha, p[i], x[i]);
        const float ri = fmaf(-alpha, q[i], r[i]);
        r[i] = ri;
        rr = fma(double(ri), double(ri), rr);
        rz = fma(double(ri), double(ri * dinv[i]), rz);
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
        update = update || rnorm < s->relTol * s->r0 || rnorm < s->absTol || s->iter >= s->maxIter;
        if (update) {
            s->rzPending = tot[1];
            s->update = 1;
        } else {
            s->beta = tot[1] / s->rz;
            s->rz = tot[1];
        }
    }
}

// R1: x64 += x32; x32 = 0 (only when a replacement was requested).
__global__ void __launch_bounds__(kT) mixed_fold_kernel(long n, double* __restrict__ x64, float* __restrict__ x32,
                                                        const MixedScalars* s) {
    if (!*reinterpret_cast<const volatile int*>(&s->update)) return;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long i = static_cast<long>(blockIdx.x) * kT + threadIdx.x; i < n; i += stride) {
        x64[i] += static_cast<double>(x32[i]);
        x32[i] = 0.0f;
    }
}

// R2 (and set-up): r = b - A64 x64 in FP64; r32 = float(r); ||r||^2 and r32^T z32
// in FP64.  INIT: first residual of a solve.
template <int KERNEL, bool INIT>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    mixed_residual_kernel(CsrArgs<double> A, const double* __restrict__ b, const double* __restrict__ x64,
                          const float* __restrict__ dinv, float* __restrict__ r32, MixedScalars* s,
                          double* partials, unsigned* counter) {
    if (!INIT && !*reinterpret_cast<volatile int*>(&s->update)) return;
    constexpr int T = csr_threads<KERNEL>();
    double rr = 0.0, rz = 0.0;
    auto op = [&](int row, double sum) {
        const double ri = b[row] - sum;
        const float rf = static_cast<float>(ri);
        r32[row] = rf;
        rr = fma(ri, ri, rr);
        rz = fma(double(rf), double(rf * dinv[row]), rz);
    };
    csr_rows<KERNEL, double, double, false>(A, x64, op);
    double mine[2] = {rr, rz}, tot[2];
    if (grid_reduce_last<2, T>(mine, partials, counter, tot) && threadIdx.x == 0) {
        const double rnorm = sqrt(tot[0]);
        s->rnorm = rnorm;
        if (INIT) {
            s->r0 = rnorm;
            s->absres = rnorm;
            s->relres = 1.0;
            s->maxrx = s->maxrr = s->cycleStart = rnorm;
            s->iter = 0;
            s->refinements = 0;
            s->update = 0;
            s->done = 0;
            s->error = 0;
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
                s->maxrr = rnorm;
                if (s->updateX) s->maxrx = rnorm;
                s->beta = tot[1] / s->rz;
            } else {
                s->cycleStart = rnorm;
                s->beta = 0.0;  // restart the inner CG: p = z
            }
            s->rz = tot[1];
        }
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
    int vs = 4;
    bool idx16 = false;
    float* val32 = nullptr;
    void* col32or16 = nullptr;
    float* dinv32 = nullptr;
    float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
    double* x64 = nullptr;
    const double* b = nullptr;
    ciecu::MixedScalars* d_s = nullptr;
    ciecu::MixedScalars* h_s = nullptr;
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* graphB = nullptr;
    int chunk = 16;
};

namespace ciecu {
namespace {

template <typename F>
int with_vs(int vs, F&& f) {
    switch (vs) {
        case 2: return f(std::integral_constant<int, 2>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 16: return f(std::integral_constant<int, 16>{});
        case 32: return f(std::integral_constant<int, 32>{});
        default: return f(std::integral_constant<int, 4>{});
    }
}

int f32_grid(const ciecu_mixed_s* M) {
    const long rowsPerCta = static_cast<long>(kT / 32) * (32 / M->vs);
    const long need = (M->n + rowsPerCta - 1) / rowsPerCta;
    return static_cast<int>(std::max(1L, std::min(need, static_cast<long>(sm_count()) * 8)));
}

int launch_inner(ciecu_mixed_s* M, cudaStream_t st) {
    const int gridA = f32_grid(M);
    const int gridV = grid_for((M->n + 3) / 4, kT, 8);
    ciecu_csr_s* A = M->A;
    CIECU_TRY(with_vs(M->vs, [&](auto v) -> int {
        constexpr int VS = decltype(v)::value;
        if (M->idx16)
            mixed_spmv_kernel<VS, true><<<gridA, kT, 0, st>>>(static_cast<int>(M->n), A->rowptr, M->col32or16,
                                                              M->val32, M->p32, M->q32, M->d_s, M->d_partials,
                                                              M->d_counter);
        else
            mixed_spmv_kernel<VS, false><<<gridA, kT, 0, st>>>(static_cast<int>(M->n), A->rowptr, M->col32or16,
                                                               M->val32, M->p32, M->q32, M->d_s, M->d_partials,
                                                               M->d_counter);
        return CIECU_OK;
    }));
    mixed_update_kernel<<<gridV, kT, 0, st>>>(M->n, M->x32, M->r32, M->p32, M->q32, M->dinv32, M->d_s, M->d_partials,
                                              M->d_counter);
    mixed_fold_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, M->x64, M->x32, M->d_s);
    const int gridR = csr_grid(A, A->kernel);
    CIECU_TRY(with_schedule(A->kernel, [&](auto k) -> int {
        constexpr int K = decltype(k)::value;
        mixed_residual_kernel<K, false><<<gridR, csr_threads<K>(), 0, st>>>(
            A->args<double>(), M->b, M->x64, M->dinv32, M->r32, M->d_s, M->d_partials, M->d_counter);
        return CIECU_OK;
    }));
    mixed_direction_kernel<<<gridV, kT, 0, st>>>(M->n, M->p32, M->r32, M->dinv32, M->d_s);
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
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int status = CIECU_OK;
    for (int i = 0; i < M->chunk && status == CIECU_OK; ++i) status = launch_inner(M, st);
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

extern "C" {

int ciecu_mixed_create(ciecu_csr lhs, const double* d_inverseDiagonal, ciecu_statistics settings,
                       ciecu_mixed_options options, ciecu_mixed* out) {
    CIECU_REQUIRE(lhs && out && d_inverseDiagonal, "mixed_create: null argument");
    CIECU_REQUIRE(lhs->valueType == CIECU_F64 && lhs->rows == lhs->cols, "mixed_create: square FP64 matrix expected");
    CIECU_REQUIRE(options.mode == 0 || options.mode == 1, "mixed_create: mode must be 0 or 1");
    CIECU_REQUIRE(options.delta > 0.0 && options.delta < 1.0, "mixed_create: delta must be in (0, 1)");
    CIECU_TRY(ensure_tuned(lhs));
    auto* M = new ciecu_mixed_s();
    M->A = lhs;
    M->dinv64 = d_inverseDiagonal;
    M->settings = settings;
    M->options = options;
    M->n = lhs->rows;
    M->vs = lhs->avgRow > 12 ? 4 : 2;
    cudaStream_t st = lhs->space->stream;
    const size_t n = static_cast<size_t>(std::max<long>(M->n, 1)) + 4;
    const size_t nnz = static_cast<size_t>(std::max<long>(lhs->nnz, 1));
    cudaError_t e = cudaMalloc(&M->val32, sizeof(float) * nnz);
    const bool try16 = options.compressColumns != 0;
    if (e == cudaSuccess) e = cudaMalloc(&M->col32or16, (try16 ? sizeof(short) : sizeof(int)) * nnz);
    for (float** v : {&M->dinv32, &M->x32, &M->r32, &M->p32, &M->q32})
        if (e == cudaSuccess) e = cudaMalloc(v, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&M->x64, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_s, sizeof(MixedScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&M->h_s, sizeof(MixedScalars));
    if (e == cudaSuccess) e = cudaMalloc(&M->d_partials, sizeof(double) * kMaxPartials * 2);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_counter, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_counter, 0, sizeof(unsigned) * 4, st);
    if (e != cudaSuccess) {
        ciecu_mixed_destroy(M);
        return cuda_fail(e, "mixed_create: allocation");
    }
    unsigned* d_far = reinterpret_cast<unsigned*>(lhs->space->d_result);
    unsigned far = 0;
    e = cudaMemsetAsync(d_far, 0, sizeof(unsigned), st);
    if (M->n > 0) {
        compress_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(
            static_cast<int>(M->n), lhs->rowptr, lhs->col, static_cast<const double*>(lhs->val), M->val32,
            try16 ? static_cast<short*>(M->col32or16) : nullptr, d_far);
        to_f32_kernel<<<grid_for(M->n, kT, 8), kT, 0, st>>>(M->n, d_inverseDiagonal, M->dinv32);
        count_launch(2);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&far, d_far, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ciecu_mixed_destroy(M);
        return cuda_fail(e, "mixed_create: conversion");
    }
    M->idx16 = try16 && !far;
    if (!M->idx16) {
        // bandwidth too large for 16-bit offsets (or not requested): int32 columns
        cudaFree(M->col32or16);
        M->col32or16 = nullptr;
        e = cudaMalloc(&M->col32or16, sizeof(int) * nnz);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(M->col32or16, lhs->col, sizeof(int) * lhs->nnz, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            ciecu_mixed_destroy(M);
            return cuda_fail(e, "mixed_create: int32 columns");
        }
    }
    *out = M;
    return CIECU_OK;
}

int ciecu_mixed_destroy(ciecu_mixed M) {
    if (!M) return CIECU_OK;
    if (M->A && M->A->space) cudaStreamSynchronize(M->A->space->stream);
    if (M->graph) cudaGraphExecDestroy(M->graph);
    cudaFree(M->val32);
    cudaFree(M->col32or16);
    cudaFree(M->dinv32);
    cudaFree(M->x32);
    cudaFree(M->r32);
    cudaFree(M->p32);
    cudaFree(M->q32);
    cudaFree(M->x64);
    cudaFree(M->d_s);
    if (M->h_s) cudaFreeHost(M->h_s);
    cudaFree(M->d_partials);
    cudaFree(M->d_counter);
    delete M;
    return CIECU_OK;
}

int ciecu_mixed_info(ciecu_mixed M, int* compressedColumns, int* lanesPerRow) {
    CIECU_REQUIRE(M, "mixed_info: null solver");
    if (compressedColumns) *compressedColumns = M->idx16 ? 1 : 0;
    if (lanesPerRow) *lanesPerRow = M->vs;
    return CIECU_OK;
}

int ciecu_mixed_apply_f32(ciecu_mixed M, const float* d_in, float* d_out) {
    CIECU_REQUIRE(M && (M->n == 0 || (d_in && d_out)), "mixed_apply_f32: null argument");
    if (M->n == 0) return CIECU_OK;
    cudaStream_t st = M->A->space->stream;
    const int grid = f32_grid(M);
    CIECU_TRY(with_vs(M->vs, [&](auto v) -> int {
        constexpr int VS = decltype(v)::value;
        if (M->idx16)
            mixed_apply_kernel<VS, true><<<grid, kT, 0, st>>>(static_cast<int>(M->n), M->A->rowptr, M->col32or16,
                                                              M->val32, d_in, d_out);
        else
            mixed_apply_kernel<VS, false><<<grid, kT, 0, st>>>(static_cast<int>(M->n), M->A->rowptr, M->col32or16,
                                                               M->val32, d_in, d_out);
        return CIECU_OK;
    }));
    count_launch();
    CIECU_CHECK_LAUNCH("mixed_apply_kernel");
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
        *M->h_s = init;
        CIECU_CUDA(cudaMemcpyAsync(M->d_s, M->h_s, sizeof(MixedScalars), cudaMemcpyHostToDevice, st));
        CIECU_CUDA(cudaMemsetAsync(M->x32, 0, sizeof(float) * n, st));
        CIECU_CUDA(cudaMemsetAsync(M->p32, 0, sizeof(float) * n, st));
        const int gridR = csr_grid(A, A->kernel);
        CIECU_TRY(with_schedule(A->kernel, [&](auto k) -> int {
            constexpr int K = decltype(k)::value;
            mixed_residual_kernel<K, true><<<gridR, csr_threads<K>(), 0, st>>>(
                A->args<double>(), d_in, M->x64, M->dinv32, M->r32, M->d_s, M->d_partials, M->d_counter);
            return CIECU_OK;
        }));
        mixed_direction_kernel<<<grid_for((n + 3) / 4, kT, 8), kT, 0, st>>>(n, M->p32, M->r32, M->dinv32, M->d_s);
        count_launch(2);
        CIECU_CHECK_LAUNCH("mixed set-up");
        CIECU_TRY(build_mixed_graph(M));
        for (;;) {
            CIECU_CUDA(cudaMemcpyAsync(M->h_s, M->d_s, sizeof(MixedScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            if (M->h_s->done) break;
            CIECU_CUDA(cudaGraphLaunch(M->graph, st));
            count_launch(5LL * M->chunk);
        }
        const MixedScalars& s = *M->h_s;
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
