// Jacobi-preconditioned conjugate gradients, FP64:
// ConjugateGradients<TSpace>::product (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201)
// with DiagonalOperator (DiagonalOperator.cpp:37-53) as preconditioner.
//
// One iteration = three kernels over HBM, with the solver scalars on the device:
//   K1  q = A p (CSR row pass) and p^T q in the same pass; the last CTA forms
//       alpha = rz / p^T q and flags the p^T A p <= 0 breakdown.
//   K2  x += alpha p; r -= alpha q; z = D^-1 r; r^T r and r^T z in the same pass;
//       the last CTA forms beta, the residual norms and the stopping decision.
//   K3  p = beta p + z (z recomputed from r and D^-1; same rounding as
//       space.scale(search, beta) followed by space.add(search, z, 1)).
// Every kernel returns at once when the done flag is set, so a CUDA graph of a
// fixed number of iterations can be replayed until the host sees the flag.
#include "graph.cuh"
#include "pcg.cuh"

#include <string>

namespace ciecu {

namespace {

constexpr int kT = 256;

// r = b - A x (x = initial guess) is formed with the CSR kernel in the host code;
// this kernel does the rest of the set-up (:100-132): rr, early exit, z, rz, p.
template <bool PRECOND>
__global__ void __launch_bounds__(kT) pcg_init_kernel(long n, const double* __restrict__ r,
                                                      const double* __restrict__ dinv, double* __restrict__ p,
                                                      PcgScalars* s, double* partials, unsigned* counter) {
    double rr = 0.0, rz = 0.0;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long i = static_cast<long>(blockIdx.x) * kT + threadIdx.x; i < n; i += stride) {
        const double ri = r[i];
        const double zi = PRECOND ? ri * dinv[i] : ri;
        p[i] = zi;
        rr = fma(ri, ri, rr);
        rz = fma(ri, zi, rz);
    }
    double mine[2] = {rr, rz}, tot[2];
    if (grid_reduce_last<2, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->rr = tot[0];
        s->r0 = sqrt(tot[0]);
        s->absres = s->r0;
        s->relres = 1.0;
        s->iter = 0;
        s->done = 0;
        s->error = 0;
        if (float_less(s->absres, s->absTol) || float_less(s->relres, s->relTol)) {
            s->done = 1;
        } else {
            s->rz = PRECOND ? tot[1] : tot[0];
            if (!(0.0 < s->rz)) {
                s->done = 3;
                s->error = CIECU_ERR_BREAKDOWN;
                s->errorKind = 1;
                s->errorIter = 0;
            } else if (s->maxIter <= 0) {
                s->done = 2;
            }
        }
    }
}

// K1: q = A p, p^T q, alpha.
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

// Ends the device-side loop (graph WHILE node).  COND is a template parameter so
// that the instantiation used by the plain captured graphs contains no
// conditional-node call at all (profilers skip kernels that have one).
template <bool COND>
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle cond, unsigned value) {
    if constexpr (COND) cudaGraphSetConditional(cond, value);
}

template <int KERNEL, bool COND>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    pcg_spmv_kernel(CsrArgs<double> A, const double* __restrict__ p, double* __restrict__ q, PcgScalars* s,
                    double* partials, unsigned* counter, cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    constexpr int T = csr_threads<KERNEL>();
    PqOp op{p, q, 0.0};
    csr_rows<KERNEL, double, double, false>(A, p, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, T>(mine, partials, counter, tot) && threadIdx.x == 0) {
        s->pq = tot[0];
        if (!(0.0 < tot[0])) {
            s->done = 3;
            s->error = CIECU_ERR_BREAKDOWN;
            s->errorKind = 2;
            s->errorIter = s->iter;
            set_loop<COND>(cond, 0);
        } else {
            s->alpha = s->rz / tot[0];
        }
    }
}

// K2: x, r update; z; rr, rz; beta and the stopping test (:154-185).
// Two elements per thread with 16-byte loads (all operands 16-byte aligned).
template <bool PRECOND, bool COND>
__global__ void __launch_bounds__(kT) pcg_update_kernel(long n, double* __restrict__ x, double* __restrict__ r,
                                                        const double* __restrict__ p, const double* __restrict__ q,
                                                        const double* __restrict__ dinv, PcgScalars* s,
                                                        double* partials, unsigned* counter,
                                                        cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    const double alpha = s->alpha;
    const double malpha = -alpha;
    double rr = 0.0, rz = 0.0;
    const long pairs = n >> 1;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long j = static_cast<long>(blockIdx.x) * kT + threadIdx.x; j < pairs; j += stride) {
        const double2 pj = reinterpret_cast<const double2*>(p)[j];
        const double2 qj = reinterpret_cast<const double2*>(q)[j];
        double2 xj = reinterpret_cast<const double2*>(x)[j];
        double2 rj = reinterpret_cast<const double2*>(r)[j];
        xj.x = fma(alpha, pj.x, xj.x);
        xj.y = fma(alpha, pj.y, xj.y);
        rj.x = fma(malpha, qj.x, rj.x);
        rj.y = fma(malpha, qj.y, rj.y);
        reinterpret_cast<double2*>(x)[j] = xj;
        reinterpret_cast<double2*>(r)[j] = rj;
        rr = fma(rj.x, rj.x, rr);
        rr = fma(rj.y, rj.y, rr);
        if (PRECOND) {
            const double2 dj = reinterpret_cast<const double2*>(dinv)[j];
            rz = fma(rj.x, rj.x * dj.x, rz);
            rz = fma(rj.y, rj.y * dj.y, rz);
        }
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long i = n - 1;
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(malpha, q[i], r[i]);
        r[i] = ri;
        rr = fma(ri, ri, rr);
        if (PRECOND) rz = fma(ri, ri * dinv[i], rz);
    }
    double mine[2] = {rr, rz}, tot[2];
    if (grid_reduce_last<2, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
        const double rzNew = PRECOND ? tot[1] : tot[0];
        s->rr = tot[0];
        s->beta = rzNew / s->rz;
        s->rz = rzNew;
        s->absres = sqrt(tot[0]);
        s->relres = s->absres / s->r0;
        if (float_less(s->absres, s->absTol) || float_less(s->relres, s->relTol)) {
            s->done = 1;
        } else {
            s->iter += 1;
            if (s->iter >= s->maxIter) s->done = 2;
        }
        s->chunkIter += 1;
        set_loop<COND>(cond, (s->done == 0 && s->chunkIter < s->chunkLimit) ? 1u : 0u);
    }
}

// K3: p = beta p + z.  Runs after K2 decided to continue; a converged solve
// does not need the new search direction.
template <bool PRECOND>
__global__ void __launch_bounds__(kT) pcg_direction_kernel(long n, double* __restrict__ p,
                                                           const double* __restrict__ r,
                                                           const double* __restrict__ dinv, const PcgScalars* s) {
    if (*reinterpret_cast<const volatile int*>(&s->done)) return;
    const double beta = s->beta;
    const long pairs = n >> 1;
    const long stride = static_cast<long>(gridDim.x) * kT;
    for (long j = static_cast<long>(blockIdx.x) * kT + threadIdx.x; j < pairs; j += stride) {
        const double2 rj = reinterpret_cast<const double2*>(r)[j];
        double2 pj = reinterpret_cast<const double2*>(p)[j];
        double2 zj = rj;
        if (PRECOND) {
            const double2 dj = reinterpret_cast<const double2*>(dinv)[j];
            zj.x = __dmul_rn(rj.x, dj.x);
            zj.y = __dmul_rn(rj.y, dj.y);
        }
        pj.x = __dadd_rn(__dmul_rn(pj.x, beta), zj.x);
        pj.y = __dadd_rn(__dmul_rn(pj.y, beta), zj.y);
        reinterpret_cast<double2*>(p)[j] = pj;
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long i = n - 1;
        const double zi = PRECOND ? __dmul_rn(r[i], dinv[i]) : r[i];
        p[i] = __dadd_rn(__dmul_rn(p[i], beta), zi);
    }
}

__global__ void fill_ones_kernel(long n, double* __restrict__ v) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) v[i] = 1.0;
}

// out = inScale*out + outScale*x with the space ops of :190-198.
__global__ void pcg_output_kernel(long n, double inScale, double outScale, const double* __restrict__ x,
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

struct ciecu_pcg_s {
    ciecu_csr_s* A = nullptr;
    const double* dinv = nullptr;
    ciecu_statistics settings{};
    int verbosity = 0;
    long n = 0;
    double* x = nullptr;
    double* r = nullptr;
    double* p = nullptr;
    double* q = nullptr;
    ciecu::PcgScalars* d_s = nullptr;
    ciecu::PcgScalars* h_s = nullptr;
    double* d_partials = nullptr;
    unsigned* d_counter = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graphKernel = -1;
    bool deviceLoop = false;  // graph = WHILE loop (else `chunk` unrolled iterations)
    int kernel = 0;           // K1 schedule, autotuned on the fused SpMV kernel itself
    int chunk = 16;
};

namespace ciecu {
namespace {

template <bool COND>
int launch_iteration(ciecu_pcg_s* S, cudaStream_t st, cudaGraphConditionalHandle cond) {
    ciecu_csr_s* A = S->A;
    const int needA = csr_grid(A, S->kernel);
    const long needV = ((S->n + 1) / 2 + kT - 1) / kT;
    const bool pre = S->dinv != nullptr;
    CIECU_TRY(with_schedule(S->kernel, [&](auto k) -> int {
        constexpr int K = decltype(k)::value;
        pcg_spmv_kernel<K, COND><<<fit_grid(pcg_spmv_kernel<K, COND>, csr_threads<K>(), needA), csr_threads<K>(), 0,
                                   st>>>(A->args<double>(), S->p, S->q, S->d_s, S->d_partials, S->d_counter, cond);
        return CIECU_OK;
    }));
    if (pre) {
        pcg_update_kernel<true, COND><<<fit_grid(pcg_update_kernel<true, COND>, kT, needV), kT, 0, st>>>(
            S->n, S->x, S->r, S->p, S->q, S->dinv, S->d_s, S->d_partials, S->d_counter, cond);
        pcg_direction_kernel<true><<<fit_grid(pcg_direction_kernel<true>, kT, needV), kT, 0, st>>>(S->n, S->p, S->r,
                                                                                                   S->dinv, S->d_s);
    } else {
        pcg_update_kernel<false, COND><<<fit_grid(pcg_update_kernel<false, COND>, kT, needV), kT, 0, st>>>(
            S->n, S->x, S->r, S->p, S->q, S->dinv, S->d_s, S->d_partials, S->d_counter, cond);
        pcg_direction_kernel<false><<<fit_grid(pcg_direction_kernel<false>, kT, needV), kT, 0, st>>>(S->n, S->p, S->r,
                                                                                                    S->dinv, S->d_s);
    }
    CIECU_CHECK_LAUNCH("pcg iteration");
    return CIECU_OK;
}

// Picks the K1 schedule by timing the fused SpMV + p^T q kernel itself on the
// solver's buffers (p = 0 -> q); its register use, and so the best schedule,
// differs from the plain operator's.
int tune_solver_spmv(ciecu_pcg_s* S) {
    if (S->kernel != 0) return CIECU_OK;
    ciecu_csr_s* A = S->A;
    cudaStream_t st = A->space->stream;
    // p = D^-1 (or 1): positive, so p^T A p > 0 for an SPD matrix and the timed
    // kernel never trips the breakdown flag (which would make later candidates
    // return at once and win).
    PcgScalars scratch{};
    scratch.rz = 1.0;
    CIECU_CUDA(cudaMemcpyAsync(S->d_s, &scratch, sizeof(PcgScalars), cudaMemcpyHostToDevice, st));
    if (S->dinv)
        CIECU_CUDA(cudaMemcpyAsync(S->p, S->dinv, sizeof(double) * S->n, cudaMemcpyDeviceToDevice, st));
    else
        fill_ones_kernel<<<grid_for(S->n, kT, 8), kT, 0, st>>>(S->n, S->p);
    cudaEvent_t e0, e1;
    CIECU_CUDA(cudaEventCreate(&e0));
    CIECU_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestK = A->kernel;
    cudaError_t e = cudaSuccess;
    for (int k : {1, 2, 4, 8, 16, 32}) {
        if (k >= 16 && A->avgRow < k) continue;
        auto launch = [&]() {
            with_schedule(k, [&](auto kk) -> int {
                constexpr int K = decltype(kk)::value;
                pcg_spmv_kernel<K, false><<<fit_grid(pcg_spmv_kernel<K, false>, csr_threads<K>(), csr_grid(A, k)),
                                            csr_threads<K>(), 0, st>>>(A->args<double>(), S->p, S->q, S->d_s,
                                                                       S->d_partials, S->d_counter, 0);
                return CIECU_OK;
            });
        };
        for (int rep = 0; rep < 2; ++rep) launch();
        for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {  // best of three: robust to noise
            cudaEventRecord(e0, st);
            for (int rep = 0; rep < 3; ++rep) launch();
            cudaEventRecord(e1, st);
            count_launch(3);
            e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                bestK = k;
            }
        }
        count_launch(2);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pcg: K1 autotune");
    // A breakdown during tuning (matrix not SPD) invalidates the timings: keep
    // the operator's own schedule.
    int flag = 0;
    CIECU_CUDA(cudaMemcpyAsync(&flag, &S->d_s->done, sizeof(int), cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    S->kernel = flag ? A->kernel : bestK;
    return CIECU_OK;
}

// The solve loop as a graph: a device-side WHILE loop over one iteration when the
// driver supports conditional nodes, else `chunk` captured iterations that the
// host replays until the done flag is set.
int build_graph(ciecu_pcg_s* S) {
    cudaStream_t st = S->A->space->stream;
    if (S->graph && S->graphKernel == S->kernel) return CIECU_OK;
    if (S->graph) {
        cudaGraphExecDestroy(S->graph);
        S->graph = nullptr;
    }
    int status = CIECU_ERR_ARGUMENT;
    if (device_loop_enabled())
        status = build_while_graph(st, [&](cudaGraph_t, cudaGraphConditionalHandle cond) {
        return launch_iteration<true>(S, st, cond);
    }, &S->graph);
    if (status == CIECU_OK) {
        S->deviceLoop = true;
        S->graphKernel = S->kernel;
        return CIECU_OK;
    }
    cudaGetLastError();  // clear a sticky launch error of the failed attempt
    S->deviceLoop = false;
    cudaGraph_t g = nullptr;
    CIECU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    status = CIECU_OK;
    for (int i = 0; i < S->chunk && status == CIECU_OK; ++i) status = launch_iteration<false>(S, st, 0);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (status != CIECU_OK) {
        if (g) cudaGraphDestroy(g);
        return status;
    }
    if (e != cudaSuccess) return cuda_fail(e, "pcg graph capture");
    e = cudaGraphInstantiate(&S->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "pcg graph instantiate");
    S->graphKernel = S->kernel;
    return CIECU_OK;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_pcg_create(ciecu_csr lhs, const double* d_inverseDiagonal, ciecu_statistics settings, int verbosity,
                     ciecu_pcg* out) {
    CIECU_REQUIRE(lhs && out, "pcg_create: null matrix or output");
    CIECU_REQUIRE(lhs->valueType == CIECU_F64, "pcg_create: the FP64 solver needs an FP64 matrix");
    CIECU_REQUIRE(lhs->rows == lhs->cols, "pcg_create: the system matrix must be square");
    CIECU_REQUIRE(reinterpret_cast<uintptr_t>(d_inverseDiagonal) % 16 == 0,
                  "pcg_create: the inverse diagonal must be 16-byte aligned");
    auto* S = new ciecu_pcg_s();
    S->A = lhs;
    S->dinv = d_inverseDiagonal;
    S->settings = settings;
    S->verbosity = verbosity;
    S->n = lhs->rows;
    const size_t bytes = sizeof(double) * static_cast<size_t>(std::max<long>(S->n, 1));
    cudaError_t e = cudaSuccess;
    for (double** v : {&S->x, &S->r, &S->p, &S->q})
        if (e == cudaSuccess) e = cudaMalloc(v, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&S->d_s, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_s, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMalloc(&S->d_partials, sizeof(double) * kMaxPartials * 2);
    if (e == cudaSuccess) e = cudaMalloc(&S->d_counter, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->d_counter, 0, sizeof(unsigned) * 4, lhs->space->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->q, 0, bytes, lhs->space->stream);
    if (e != cudaSuccess) {
        ciecu_pcg_destroy(S);
        return cuda_fail(e, "pcg_create: allocation");
    }
    *out = S;
    return CIECU_OK;
}

int ciecu_pcg_destroy(ciecu_pcg S) {
    if (!S) return CIECU_OK;
    // No access to S->A: the matrix handle may already be gone.  cudaFree
    // synchronises the device before releasing memory.
    if (S->graph) cudaGraphExecDestroy(S->graph);
    cudaFree(S->x);
    cudaFree(S->r);
    cudaFree(S->p);
    cudaFree(S->q);
    cudaFree(S->d_s);
    if (S->h_s) cudaFreeHost(S->h_s);
    cudaFree(S->d_partials);
    cudaFree(S->d_counter);
    delete S;
    return CIECU_OK;
}

int ciecu_pcg_info(ciecu_pcg S, int* spmvSchedule, int* deviceLoop) {
    CIECU_REQUIRE(S, "pcg_info: null solver");
    if (spmvSchedule) *spmvSchedule = S->kernel;
    if (deviceLoop) *deviceLoop = S->deviceLoop ? 1 : 0;
    return CIECU_OK;
}

int ciecu_pcg_set_graph_chunk(ciecu_pcg S, int iterations) {
    CIECU_REQUIRE(S && iterations >= 1 && iterations <= 4096, "pcg_set_graph_chunk: chunk must be in [1, 4096]");
    if (S->chunk != iterations && S->graph) {
        cudaGraphExecDestroy(S->graph);
        S->graph = nullptr;
    }
    S->chunk = iterations;
    return CIECU_OK;
}

int ciecu_pcg_set_schedule(ciecu_pcg S, int schedule) {
    CIECU_REQUIRE(S, "pcg_set_schedule: null solver");
    CIECU_REQUIRE(schedule == 0 || schedule == 1 || schedule == 2 || schedule == 4 || schedule == 8 ||
                      schedule == 16 || schedule == 32,
                  "pcg_set_schedule: schedule must be 0 (autotune), 1, 2, 4, 8, 16 or 32");
    S->kernel = schedule;  // the graph is rebuilt when it was built for another schedule
    return CIECU_OK;
}

int ciecu_pcg_product(ciecu_pcg S, double inScale, const double* d_in, double outScale, double* d_out,
                      ciecu_statistics* h_stats) {
    CIECU_REQUIRE(S, "pcg_product: null solver");
    const long n = S->n;
    CIECU_REQUIRE(n == 0 || (d_in && d_out), "pcg_product: null vector");
    ciecu_csr_s* A = S->A;
    cudaStream_t st = A->space->stream;
    ciecu_statistics stats{0, 1.7976931348623157e308, 1.7976931348623157e308};
    if (n == 0) {
        if (h_stats) *h_stats = ciecu_statistics{0, 0.0, 0.0};
        return CIECU_OK;
    }
    CIECU_TRY(ensure_tuned(A));
    CIECU_TRY(tune_solver_spmv(S));
    // solution <- out (initial guess)
    CIECU_CUDA(cudaMemcpyAsync(S->x, d_out, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    if (S->settings.iterationCount > 0) {
        PcgScalars init{};
        init.maxIter = S->settings.iterationCount;
        init.absTol = S->settings.absoluteResidual;
        init.relTol = S->settings.relativeResidual;
        *S->h_s = init;
        CIECU_CUDA(cudaMemcpyAsync(S->d_s, S->h_s, sizeof(PcgScalars), cudaMemcpyHostToDevice, st));
        // r = b - A x
        CIECU_CUDA(cudaMemcpyAsync(S->r, d_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        CIECU_TRY(ciecu_csr_spmv_f64(A, 1.0, S->x, -1.0, S->r));
        const long needV = (n + kT - 1) / kT;
        if (S->dinv)
            pcg_init_kernel<true><<<fit_grid(pcg_init_kernel<true>, kT, needV), kT, 0, st>>>(
                n, S->r, S->dinv, S->p, S->d_s, S->d_partials, S->d_counter);
        else
            pcg_init_kernel<false><<<fit_grid(pcg_init_kernel<false>, kT, needV), kT, 0, st>>>(
                n, S->r, S->dinv, S->p, S->d_s, S->d_partials, S->d_counter);
        count_launch();
        CIECU_CHECK_LAUNCH("pcg_init_kernel");
        CIECU_TRY(build_graph(S));
        // Replay graph chunks until the device reports done.  The scalars are read
        // back after each chunk; the kernels of a finished solve return at once.
        // Device loop: one launch runs up to chunkLimit iterations; the host only
        // looks at the scalars between launches.
        const long long limit = S->deviceLoop ? 4096 : S->chunk;
        for (;;) {
            CIECU_CUDA(cudaMemcpyAsync(S->h_s, S->d_s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            if (S->h_s->done) break;
            const long long before = S->h_s->iter;
            S->h_s->chunkIter = 0;
            S->h_s->chunkLimit = limit;
            CIECU_CUDA(cudaMemcpyAsync(&S->d_s->chunkIter, &S->h_s->chunkIter, 2 * sizeof(long long),
                                       cudaMemcpyHostToDevice, st));
            CIECU_CUDA(cudaGraphLaunch(S->graph, st));
            CIECU_CUDA(cudaMemcpyAsync(S->h_s, S->d_s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            count_launch(3LL * std::max<long long>(1, S->deviceLoop ? S->h_s->iter - before + 1 : S->chunk));
            if (S->h_s->done) break;
        }
        const PcgScalars& s = *S->h_s;
        if (s.error) {
            if (h_stats) *h_stats = ciecu_statistics{s.errorIter, s.absres, s.relres};
            if (s.errorKind == 1)
                return fail(CIECU_ERR_BREAKDOWN, "preconditioned norm vanished in iteration 0 (r^T @ z = 0)");
            return fail(CIECU_ERR_BREAKDOWN, "p^T @ A @ p vanished in iteration " + std::to_string(s.errorIter));
        }
        stats.iterationCount = s.iter;
        stats.absoluteResidual = s.absres;
        stats.relativeResidual = s.relres;
    }
    pcg_output_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, inScale, outScale, S->x, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("pcg_output_kernel");
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (h_stats) *h_stats = stats;
    return CIECU_OK;
}

}  // extern "C"
