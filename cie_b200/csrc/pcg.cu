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
#include "dia.cuh"
#include "pcg.cuh"

#include <string>
#include <tuple>
#include <mutex>
#include <map>
#include <vector>

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

// K1 over the upper half of the DIA copy of a bitwise symmetric matrix: half the
// matrix bytes, the same row sums (dia_rows_sym).
template <bool COND>
__global__ void __launch_bounds__(kT) pcg_spmv_dia_sym_kernel(DiaArgs<double> U, const double* __restrict__ p,
                                                             double* __restrict__ q, PcgScalars* s, double* partials,
                                                             unsigned* counter, cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp op{p, q, 0.0};
    dia_rows_sym<0, double, double>(U, p, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
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

// K1 over the DIA copy of a few-diagonal matrix (dia.cuh): no column indices,
// 8 bytes per stored entry.
template <int ND, bool COND>
__global__ void __launch_bounds__(kT) pcg_spmv_dia_kernel(DiaArgs<double> A, const double* __restrict__ p,
                                                         double* __restrict__ q, PcgScalars* s, double* partials,
                                                         unsigned* counter, cudaGraphConditionalHandle cond) {
    if (*reinterpret_cast<volatile int*>(&s->done)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_loop<COND>(cond, 0);
        return;
    }
    PqOp op{p, q, 0.0};
    dia_rows<ND, double, double>(A, p, op);
    double mine[1] = {op.acc}, tot[1];
    if (grid_reduce_last<1, kT>(mine, partials, counter, tot) && threadIdx.x == 0) {
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

// ---- single-launch solve -----------------------------------------------------
// For a system whose matrix fits in the shared memory of the whole chip, the three
// launches per iteration cost more than their work.  Here one cooperative launch
// (every block resident, one per SM) runs the iterations.  Each block owns one
// contiguous row range (balanced by nonzeros) and keeps its rows of the matrix
// and its own x, r, D^-1, q, p and z in shared memory for the whole launch.  An
// iteration has two grid-wide exchanges:
//   S  q = A p_k with p_k = beta p_{k-1} + z_k formed on the fly for each gathered
//      column (p is double-buffered in global memory, so no block overwrites a
//      p_{k-1} another block still reads); the owner of row i stores p_k,i;
//      partial p^T q.  -> exchange 1: alpha = rz / p^T q in every block.
//   U  x += alpha p_k, r -= alpha q, z = D^-1 r on the own rows (z also to global
//      memory for the other blocks' gathers); partial r^T r, r^T z.
//      -> exchange 2: beta, norms and the stopping test.
// An exchange publishes the block's partial sums with a release store of an
// epoch number; every block then reads all blocks' epochs (relaxed loads and one
// acquire fence) and sums the partials in block order, so all blocks hold
// bit-identical scalars and take the same branches.  Global vectors written
// during the launch are read with ld.global.cg (L2), never through the
// non-coherent L1 or texture paths.  Every wait is bounded in time (2 s of the
// GPU's global timer by default); a wait that gives up sets the abort flag, every
// block leaves, and the host reports CIECU_ERR_TIMEOUT.  One exchange costs about
// 5 us on B200 (148 blocks), about a quarter of what three launches per
// iteration cost together.
constexpr int kPT = 1024;

struct alignas(32) ExchangeSlot {
    double v[2];
    unsigned long long epoch;
    unsigned long long pad;
};

struct PersistentArgs {
    CsrArgs<double> A;
    const int2* __restrict__ split;  // (first row, its first entry) of each block; grid + 1 entries
    const double* __restrict__ dinv;
    double* x;
    double* r;
    double* z;
    double* p0;  // p_k for even k
    double* p1;  // p_k for odd k
    ExchangeSlot* slotsS;
    ExchangeSlot* slotsU;
    int* abortFlag;
    PcgScalars* s;
    unsigned long long epoch0;
    long long waitNs;                   // bound of one exchange wait
    unsigned long long withholdEpoch;   // test hook: the last block never publishes this epoch (0: none)
};

// Shared memory of a block with ne entries and nr rows: doubles (values, then x,
// r, D^-1, q, p, z of the own rows) followed by ints (columns, local row offsets).
__host__ __device__ inline size_t persistent_smem(long ne, long nr) {
    return static_cast<size_t>(8 * (ne + 6 * nr) + 4 * (ne + nr + 1));
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Publishes the block's K partial sums under `epoch` and returns in `out` the
// grid-wide sums (blocks in index order, identical in every block).  False when a
// wait gave up or another block aborted; the block then leaves the launch.
template <int K>
__device__ bool grid_exchange(const double (&mine)[K], ExchangeSlot* slots, unsigned long long epoch,
                              const PersistentArgs& P, double (&out)[K], double* s_red) {
    int* abortFlag = P.abortFlag;
    double sums[K];
#pragma unroll
    for (int k = 0; k < K; ++k) sums[k] = block_sum<double, kPT>(mine[k], s_red);  // orders the block's stores
    if (threadIdx.x == 0 && !(epoch == P.withholdEpoch && blockIdx.x == gridDim.x - 1)) {
        ExchangeSlot* m = slots + blockIdx.x;
#pragma unroll
        for (int k = 0; k < K; ++k) m->v[k] = sums[k];
        st_release_u64(&m->epoch, epoch);  // cumulative: also releases the block's stores before the barrier
    }
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    bool ok = true;
    for (unsigned b = threadIdx.x; b < gridDim.x && ok; b += kPT) {
        const ExchangeSlot* o = slots + b;
        const unsigned long long t0 = global_ns();
        unsigned spin = 0;
        while (ld_relaxed_u64(&o->epoch) != epoch) {
            __nanosleep(20);
            if ((++spin & 63u) == 0u &&
                (*reinterpret_cast<volatile int*>(abortFlag) ||
                 global_ns() - t0 > static_cast<unsigned long long>(P.waitNs))) {
                atomicExch(abortFlag, 1);
                ok = false;
                break;
            }
        }
        if (ok) {
            fence_acq_rel_gpu();  // acquire: the partials and the block's vector stores are visible
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += __ldcg(&o->v[k]);
        }
    }
    if (!__syncthreads_and(ok)) return false;
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = block_sum<double, kPT>(acc[k], s_red);
    return true;
}

// First row of block b when the rows are split into `blocks` ranges of about equal
// nonzero count; entry b of `out` = (first row, its first entry).
__global__ void persistent_split_kernel(const int* __restrict__ rowptr, int n, long nnz, int blocks,
                                        int2* __restrict__ out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > blocks) return;
    int row;
    if (b == 0) {
        row = 0;
    } else if (b == blocks) {
        row = n;
    } else {
        const long target = nnz * b / blocks;
        int lo = 0, hi = n;  // first row with rowptr[row] >= target
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (rowptr[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        row = lo;
    }
    out[b] = make_int2(row, rowptr[row]);
}

template <int VS, bool PRECOND>
__global__ void __launch_bounds__(kPT, 1) pcg_persistent_kernel(PersistentArgs P) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_red[32];
    const CsrArgs<double>& A = P.A;
    PcgScalars* s = P.s;
    const int2 lo = P.split[blockIdx.x], hi = P.split[blockIdx.x + 1];
    const int rb = lo.x, nr = hi.x - lo.x;
    const int eb = lo.y, ne = hi.y - lo.y;
    double* s_val = reinterpret_cast<double*>(smem);
    double* s_x = s_val + ne;
    double* s_r = s_x + nr;
    double* s_d = s_r + nr;
    double* s_q = s_d + nr;
    double* s_p = s_q + nr;
    double* s_z = s_p + nr;
    int* s_col = reinterpret_cast<int*>(s_z + nr);
    int* s_rp = s_col + ne;
    // Scalars of the iteration, identical in every block.  All reads of *s happen
    // before this block's first exchange, and block 0 writes *s back only after the
    // last one, so no block reads a scalar block 0 has already overwritten.
    long long iter = s->iter;
    const long long maxIter = s->maxIter;
    const long long chunkLimit = s->chunkLimit;
    long long chunkIter = 0;
    const double absTol = s->absTol, relTol = s->relTol, r0 = s->r0;
    double rz = s->rz, beta = s->beta, pq = s->pq, alpha = s->alpha, rr = s->rr;
    double absres = s->absres, relres = s->relres;
    int done = s->done, error = 0, errorKind = 0;
    long long errorIter = 0;
    // Stage the block's matrix rows and own vectors.
    {
        const double* pprev = (iter & 1) ? P.p0 : P.p1;
        for (int e = threadIdx.x; e < ne; e += kPT) {
            s_val[e] = __ldg(A.val + eb + e);
            s_col[e] = __ldg(A.col + eb + e);
        }
        for (int i = threadIdx.x; i <= nr; i += kPT) s_rp[i] = A.rowptr[rb + i] - eb;
        for (int i = threadIdx.x; i < nr; i += kPT) {
            s_x[i] = P.x[rb + i];
            s_r[i] = P.r[rb + i];
            s_d[i] = PRECOND ? P.dinv[rb + i] : 1.0;
            s_z[i] = P.z[rb + i];
            s_p[i] = iter > 0 ? pprev[rb + i] : 0.0;
        }
        __syncthreads();
    }
    unsigned long long epoch = P.epoch0;
    const int lane = threadIdx.x % VS;
    const int group = threadIdx.x / VS;
    constexpr int kGroups = kPT / VS;
    bool aborted = false;
    while (done == 0) {
        // ---- S: q = A p_k; p_k of the own rows to shared and global memory -----
        const bool first = iter == 0;
        const double* pprev = (iter & 1) ? P.p0 : P.p1;
        double* pcur = (iter & 1) ? P.p1 : P.p0;
        double pqPart = 0.0;
        for (int base = 0; base < nr; base += kGroups) {  // warp-uniform trip count
            const int row = base + group;
            double sum = 0.0;
            if (row < nr) {
                const int e1 = s_rp[row + 1];
#pragma unroll 4
                for (int e = s_rp[row] + lane; e < e1; e += VS) {
                    const int c = s_col[e];
                    const double zc = __ldcg(P.z + c);
                    const double pc = first ? zc : __dadd_rn(__dmul_rn(__ldcg(pprev + c), beta), zc);
                    sum = fma(s_val[e], pc, sum);
                }
            }
#pragma unroll
            for (int off = VS / 2; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off, VS);
            if (row < nr && lane == 0) {
                const double zi = s_z[row];
                const double pi = first ? zi : __dadd_rn(__dmul_rn(s_p[row], beta), zi);
                s_p[row] = pi;
                pcur[rb + row] = pi;
                s_q[row] = sum;
                pqPart = fma(pi, sum, pqPart);
            }
        }
        {
            double mine[1] = {pqPart}, tot[1];
            if (!grid_exchange<1>(mine, P.slotsS, ++epoch, P, tot, s_red)) {
                aborted = true;
                break;
            }
            pq = tot[0];
        }
        if (!(0.0 < pq)) {
            done = 3;
            error = CIECU_ERR_BREAKDOWN;
            errorKind = 2;
            errorIter = iter;
            break;
        }
        alpha = rz / pq;
        // ---- U: x, r, z on the own rows ----------------------------------------
        const double malpha = -alpha;
        double rrPart = 0.0, rzPart = 0.0;
        for (int i = threadIdx.x; i < nr; i += kPT) {
            s_x[i] = fma(alpha, s_p[i], s_x[i]);
            const double ri = fma(malpha, s_q[i], s_r[i]);
            s_r[i] = ri;
            rrPart = fma(ri, ri, rrPart);
            double zi = ri;
            if (PRECOND) {
                zi = __dmul_rn(ri, s_d[i]);
                rzPart = fma(ri, zi, rzPart);
            }
            s_z[i] = zi;
            P.z[rb + i] = zi;
        }
        {
            double mine[2] = {rrPart, rzPart}, tot[2];
            if (!grid_exchange<2>(mine, P.slotsU, ++epoch, P, tot, s_red)) {
                aborted = true;
                break;
            }
            const double rzNew = PRECOND ? tot[1] : tot[0];
            rr = tot[0];
            beta = rzNew / rz;
            rz = rzNew;
            absres = sqrt(tot[0]);
            relres = absres / r0;
        }
        if (float_less(absres, absTol) || float_less(relres, relTol)) {
            done = 1;
        } else {
            iter += 1;
            if (iter >= maxIter) done = 2;
        }
        chunkIter += 1;
        if (chunkIter >= chunkLimit) break;
    }
    if (aborted) return;
    for (int i = threadIdx.x; i < nr; i += kPT) {
        P.x[rb + i] = s_x[i];
        P.r[rb + i] = s_r[i];
    }
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    s->iter = iter;
    s->chunkIter = chunkIter;
    s->rz = rz;
    s->beta = beta;
    s->pq = pq;
    s->alpha = alpha;
    s->rr = rr;
    s->absres = absres;
    s->relres = relres;
    s->done = done;
    if (error) {
        s->error = error;
        s->errorKind = errorKind;
        s->errorIter = errorIter;
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
    bool graphSym = false;  // the graph's K1 reads the upper half of the DIA copy
    bool deviceLoop = false;  // graph = WHILE loop (else `chunk` unrolled iterations)
    int kernel = 0;           // K1 schedule, autotuned on the fused SpMV kernel itself
    int chunk = 16;
    // DIA copy of a few-diagonal matrix (K1 schedule kDiaSchedule), refilled from
    // the CSR values at every solve.
    bool diaChecked = false;
    double* diaBuf = nullptr;
    ciecu::DiaArgs<double> dia{};
    bool diaSym = false;           // the copy is bitwise symmetric: K1 reads diaU, its upper half
    ciecu::DiaArgs<double> diaU{};
    // Single-launch solve (allocated at its first use).
    int loopMode = 0;     // 0 auto (single launch when the system fits in L2), 1 graph, 2 single launch
    bool persistent = false;  // the last solve ran as a single launch
    bool planned = false;     // row split and shared-memory size computed
    bool fits = false;        // every block's rows fit in shared memory
    size_t smem = 0;          // dynamic shared memory of the single launch
    int maxRows = 0;          // rows of the largest block
    int grid = 0;             // blocks of the single launch
    int2* split = nullptr;
    double* z = nullptr;
    double* p2 = nullptr;
    void* slots = nullptr;  // 2 x SMs exchange slots
    int* abortFlag = nullptr;
    unsigned long long epoch = 1;
    long long waitNs = 2000000000LL;  // bound of one grid-wide exchange wait (global timer)
    long long withholdExchange = 0;   // test hook of the timeout path (ciecu_pcg_debug_exchange)
    bool pinned = false;              // K1 schedule pinned by ciecu_pcg_set_schedule
};

namespace ciecu {
namespace {

// K1 schedules: 1 (row-block stream kernel), 2..32 (lanes per row) and
// kDiaSchedule (the DIA copy).
constexpr int kDiaSchedule = 64;

template <bool COND>
int launch_k1(ciecu_pcg_s* S, cudaStream_t st, int schedule, cudaGraphConditionalHandle cond) {
    ciecu_csr_s* A = S->A;
    if (schedule == kDiaSchedule) {
        if (!S->diaBuf) return fail(CIECU_ERR_ARGUMENT, "pcg: the DIA schedule needs a matrix of at most 32 diagonals");
        // Runtime diagonal count (9 loads in flight per row): a fully unrolled
        // 27-diagonal FP64 row needs 64 registers and halves the occupancy, which
        // measured 20 % slower at 128^3.
        if (S->diaSym)
            pcg_spmv_dia_sym_kernel<COND><<<fit_grid(pcg_spmv_dia_sym_kernel<COND>, kT, (S->n + kT - 1) / kT), kT, 0,
                                            st>>>(S->diaU, S->p, S->q, S->d_s, S->d_partials, S->d_counter, cond);
        else
            pcg_spmv_dia_kernel<0, COND><<<fit_grid(pcg_spmv_dia_kernel<0, COND>, kT, (S->n + kT - 1) / kT), kT, 0,
                                           st>>>(S->dia, S->p, S->q, S->d_s, S->d_partials, S->d_counter, cond);
        return CIECU_OK;
    }
    const int needA = csr_grid(A, schedule);
    return with_schedule(schedule, [&](auto k) -> int {
        constexpr int K = decltype(k)::value;
        pcg_spmv_kernel<K, COND><<<fit_grid(pcg_spmv_kernel<K, COND>, csr_threads<K>(), needA), csr_threads<K>(), 0,
                                   st>>>(A->args<double>(), S->p, S->q, S->d_s, S->d_partials, S->d_counter, cond);
        return CIECU_OK;
    });
}

// Finds the diagonals once per solver and refills the DIA copy from the CSR
// values (which the caller may have changed since the last solve).
int refresh_dia(ciecu_pcg_s* S, cudaStream_t st) {
    if (!S->diaChecked) {
        S->diaChecked = true;
        const std::vector<int>* offsets = nullptr;
        CIECU_TRY(dia_offsets(S->A, &offsets));
        if (!offsets->empty()) {
            DiaArgs<double> a = dia_shape<double>(S->A, *offsets);
            const size_t bytes = sizeof(double) * static_cast<size_t>(a.ndiag) * static_cast<size_t>(a.ld);
            double* buf = nullptr;
            if (pool_alloc(&buf, bytes, st) != cudaSuccess) {
                cudaGetLastError();  // no room for the copy: the CSR schedules stay
                return CIECU_OK;
            }
            CIECU_CUDA(cudaMemsetAsync(buf, 0, bytes, st));
            a.val = buf;
            S->dia = a;
            S->diaBuf = buf;
        }
    }
    if (S->diaBuf) {
        CIECU_TRY(dia_fill_f64(S->A, S->dia, S->diaBuf, st));
        // a bitwise symmetric matrix (checked at every solve: the values may have
        // changed) is read through the upper half of the copy only
        bool sym = false;
        if (dia_symmetric_enabled())
            CIECU_TRY(dia_symmetric(S->dia, st, reinterpret_cast<unsigned*>(S->A->space->d_result), &sym));
        S->diaSym = sym;
        if (sym) S->diaU = dia_upper_view(S->dia);
    }
    return CIECU_OK;
}

template <bool COND>
int launch_iteration(ciecu_pcg_s* S, cudaStream_t st, cudaGraphConditionalHandle cond) {
    const long needV = ((S->n + 1) / 2 + kT - 1) / kT;
    const bool pre = S->dinv != nullptr;
    CIECU_TRY(launch_k1<COND>(S, st, S->kernel, cond));
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

// Splits the rows into G ranges (balanced by nonzeros) and sizes the shared
// memory of the single launch from the largest range.  G is the smallest of
// SMs/4, SMs/2 and SMs whose ranges fit in shared memory: a grid-wide exchange
// costs less with fewer blocks (measured on B200 per iteration of 2D Q1 128^2:
// 10.8 us with 37 blocks, 13.2 us with 74; 2D Q1 256^2: 13.4 us with 74 blocks,
// 14.6 us with 148).
int plan_persistent(ciecu_pcg_s* S) {
    if (S->planned) return CIECU_OK;
    ciecu_csr_s* A = S->A;
    cudaStream_t st = A->space->stream;
    int device = 0, optin = 0;
    CIECU_CUDA(cudaGetDevice(&device));
    CIECU_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    const int sms = sm_count();
    if (!S->split) CIECU_CUDA(pool_alloc(&S->split, sizeof(int2) * (sms + 1), st));
    S->fits = false;
    for (int G : {std::max(1, sms / 4), std::max(1, sms / 2), sms}) {
        persistent_split_kernel<<<(G + 1 + 127) / 128, 128, 0, st>>>(A->rowptr, A->rows, A->nnz, G, S->split);
        count_launch();
        CIECU_CHECK_LAUNCH("persistent_split_kernel");
        std::vector<int2> h(G + 1);
        CIECU_CUDA(cudaMemcpyAsync(h.data(), S->split, sizeof(int2) * (G + 1), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        size_t smem = 0;
        int maxRows = 0;
        for (int b = 0; b < G; ++b) {
            const long nr = h[b + 1].x - h[b].x, ne = static_cast<long>(h[b + 1].y) - h[b].y;
            smem = std::max(smem, persistent_smem(ne, nr));
            maxRows = std::max<int>(maxRows, static_cast<int>(nr));
        }
        S->smem = std::max<size_t>(smem, 16);
        S->maxRows = maxRows;
        S->grid = G;
        S->fits = S->smem + 1024 <= static_cast<size_t>(optin);  // 1 KB for the static reduction scratch
        if (S->fits) break;  // S->split holds this G's ranges
    }
    S->planned = true;
    return CIECU_OK;
}

int use_persistent(ciecu_pcg_s* S, bool* out) {
    *out = false;
    if (S->loopMode == 1) return CIECU_OK;
    // A pinned K1 schedule names a kernel of the graph loop: in the automatic mode
    // it selects that loop, so the pin takes effect.
    if (S->loopMode == 0 && S->pinned) return CIECU_OK;
    CIECU_TRY(plan_persistent(S));
    if (S->loopMode == 2 && !S->fits)
        return fail(CIECU_ERR_ARGUMENT, "pcg: the single-launch solve needs each SM's rows of the matrix in shared "
                                        "memory; this matrix is too large for it");
    *out = S->fits;
    return CIECU_OK;
}

int ensure_persistent_buffers(ciecu_pcg_s* S) {
    if (S->slots) return CIECU_OK;
    const size_t bytes = sizeof(double) * static_cast<size_t>(std::max<long>(S->n, 1));
    const size_t slotBytes = sizeof(ExchangeSlot) * 2 * static_cast<size_t>(sm_count());
    cudaStream_t st = S->A->space->stream;
    cudaError_t e = pool_alloc(&S->z, bytes, st);
    if (e == cudaSuccess) e = pool_alloc(&S->p2, bytes, st);
    if (e == cudaSuccess) e = pool_alloc(&S->slots, slotBytes, st);
    if (e == cudaSuccess) e = pool_alloc(&S->abortFlag, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->slots, 0, slotBytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->abortFlag, 0, sizeof(int), st);
    if (e != cudaSuccess) {
        pool_release({S->z, S->p2, S->slots, S->abortFlag});
        S->z = S->p2 = nullptr;
        S->slots = nullptr;
        S->abortFlag = nullptr;
        return cuda_fail(e, "pcg: single-launch buffers");
    }
    S->epoch = 1;
    return CIECU_OK;
}

template <int VS, bool PRE>
int launch_persistent(ciecu_pcg_s* S, cudaStream_t st) {
    auto kernel = pcg_persistent_kernel<VS, PRE>;
    CIECU_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S->smem)));
    int occ = 0;
    CIECU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kPT, S->smem));
    if (occ < 1) return fail(CIECU_ERR_CUDA, "pcg: the single-launch kernel does not fit on an SM");
    const int G = S->grid;
    ExchangeSlot* slots = static_cast<ExchangeSlot*>(S->slots);
    PersistentArgs args{S->A->args<double>(), S->split, S->dinv, S->x, S->r, S->z, S->p, S->p2,
                        slots, slots + G, S->abortFlag, S->d_s, S->epoch, S->waitNs,
                        S->withholdExchange > 0 ? S->epoch + static_cast<unsigned long long>(S->withholdExchange)
                                                : 0ULL};
    void* params[] = {&args};
    CIECU_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(G), dim3(kPT), params,
                                           S->smem, st));
    count_launch();
    return CIECU_OK;
}

// Lanes per row: as many as leave one lane group per row of the largest block,
// and no more than the average row needs.
template <bool PRE>
int launch_persistent_rows(ciecu_pcg_s* S, cudaStream_t st) {
    int vs = 32;
    while (vs > 1 && (kPT / vs < S->maxRows || vs / 2 >= S->A->avgRow)) vs >>= 1;
    switch (vs) {
        case 32: return launch_persistent<32, PRE>(S, st);
        case 16: return launch_persistent<16, PRE>(S, st);
        case 8: return launch_persistent<8, PRE>(S, st);
        case 4: return launch_persistent<4, PRE>(S, st);
        case 2: return launch_persistent<2, PRE>(S, st);
        default: return launch_persistent<1, PRE>(S, st);
    }
}

int launch_persistent_any(ciecu_pcg_s* S, cudaStream_t st) {
    return S->dinv ? launch_persistent_rows<true>(S, st) : launch_persistent_rows<false>(S, st);
}

// Runs the iterations as single launches of up to 2^16 iterations each until the
// device reports done.  On entry z holds z_0 (written by the init kernel).
int run_persistent(ciecu_pcg_s* S, cudaStream_t st) {
    constexpr long long kLimit = 1LL << 16;
    for (;;) {
        CIECU_CUDA(cudaMemcpyAsync(S->h_s, S->d_s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (S->h_s->done) return CIECU_OK;
        S->h_s->chunkIter = 0;
        S->h_s->chunkLimit = kLimit;
        CIECU_CUDA(cudaMemcpyAsync(&S->d_s->chunkIter, &S->h_s->chunkIter, 2 * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
        CIECU_TRY(launch_persistent_any(S, st));
        S->epoch += 2 * kLimit + 2;  // exchanges of one launch never reuse an epoch
        int aborted = 0;
        CIECU_CUDA(cudaMemcpyAsync(&aborted, S->abortFlag, sizeof(int), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaStreamSynchronize(st));
        if (aborted) {
            CIECU_CUDA(cudaMemsetAsync(S->abortFlag, 0, sizeof(int), st));
            CIECU_CUDA(cudaStreamSynchronize(st));
            return fail(CIECU_ERR_TIMEOUT, "pcg: a grid-wide exchange of the single-launch solve gave up waiting");
        }
    }
}

// Picks the K1 schedule by timing the fused SpMV + p^T q kernel itself on the
// solver's buffers (p = 0 -> q); its register use, and so the best schedule,
// differs from the plain operator's.
// K1 schedule chosen per matrix shape (rows, nonzeros, diagonals of the DIA
// copy, preconditioned, 16-byte aligned arrays): later solvers of the same shape
// skip the timing.
std::mutex g_k1Mutex;
std::map<std::tuple<int, long, int, int, int>, int> g_k1Choice;

int tune_solver_spmv(ciecu_pcg_s* S) {
    if (S->kernel != 0) return CIECU_OK;
    ciecu_csr_s* A = S->A;
    const auto key = std::make_tuple(A->rows, A->nnz, S->diaBuf ? S->dia.ndiag : 0, S->dinv ? 1 : 0,
                                     static_cast<int>(A->aligned16));
    {
        std::lock_guard<std::mutex> lock(g_k1Mutex);
        auto it = g_k1Choice.find(key);
        if (it != g_k1Choice.end()) {
            S->kernel = it->second;
            return CIECU_OK;
        }
    }
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
    for (int k : {1, 2, 4, 8, 16, 32, kDiaSchedule}) {
        if (k >= 16 && k <= 32 && A->avgRow < k) continue;
        if (k == kDiaSchedule && !S->diaBuf) continue;
        auto launch = [&]() { launch_k1<false>(S, st, k, 0); };
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
    if (!flag) {
        std::lock_guard<std::mutex> lock(g_k1Mutex);
        g_k1Choice[key] = S->kernel;
    }
    return CIECU_OK;
}

// The solve loop as a graph: a device-side WHILE loop over one iteration when the
// driver supports conditional nodes, else `chunk` captured iterations that the
// host replays until the done flag is set.
int build_graph(ciecu_pcg_s* S) {
    cudaStream_t st = S->A->space->stream;
    if (S->graph && S->graphKernel == S->kernel && S->graphSym == S->diaSym) return CIECU_OK;
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
        S->graphSym = S->diaSym;
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
    S->graphSym = S->diaSym;
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
    cudaStream_t st = lhs->space->stream;
    // buffers from the library's stream-ordered pool (pool_alloc)
    for (double** v : {&S->x, &S->r, &S->p, &S->q})
        if (e == cudaSuccess) e = pool_alloc(v, bytes, st);
    if (e == cudaSuccess) e = pool_alloc(&S->d_s, sizeof(PcgScalars), st);
    S->h_s = new PcgScalars();  // read back once per graph launch: pageable is enough
    if (e == cudaSuccess) e = pool_alloc(&S->d_partials, sizeof(double) * kMaxPartials * 2, st);
    if (e == cudaSuccess) e = pool_alloc(&S->d_counter, sizeof(unsigned) * 4, st);
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
    // No access to S->A: the matrix handle may already be gone.  pool_release
    // synchronises the device before releasing memory.
    if (S->graph) cudaGraphExecDestroy(S->graph);
    pool_release({S->x, S->r, S->p, S->q, S->d_s, S->d_partials, S->d_counter, S->diaBuf, S->z, S->p2, S->slots,
                  S->abortFlag, S->split});
    delete S->h_s;
    delete S;
    return CIECU_OK;
}

int ciecu_pcg_info(ciecu_pcg S, int* spmvSchedule, int* deviceLoop) {
    CIECU_REQUIRE(S, "pcg_info: null solver");
    if (spmvSchedule) *spmvSchedule = S->kernel;
    if (deviceLoop) *deviceLoop = S->persistent ? 2 : (S->deviceLoop ? 1 : 0);
    return CIECU_OK;
}

int ciecu_pcg_dia_info(ciecu_pcg S, int* storedDiagonals, int* symmetric) {
    CIECU_REQUIRE(S && storedDiagonals && symmetric, "pcg_dia_info: null argument");
    *storedDiagonals = S->diaBuf ? (S->diaSym ? S->diaU.ndiag : S->dia.ndiag) : 0;
    *symmetric = S->diaSym ? 1 : 0;
    return CIECU_OK;
}

int ciecu_pcg_set_loop(ciecu_pcg S, int mode) {
    CIECU_REQUIRE(S, "pcg_set_loop: null solver");
    CIECU_REQUIRE(mode >= 0 && mode <= 2, "pcg_set_loop: mode must be 0 (auto), 1 (graph) or 2 (single launch)");
    S->loopMode = mode;
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
                      schedule == 16 || schedule == 32 || schedule == kDiaSchedule,
                  "pcg_set_schedule: schedule must be 0 (autotune), 1, 2, 4, 8, 16, 32 or 64 (DIA)");
    S->kernel = schedule;  // the graph is rebuilt when it was built for another schedule
    S->pinned = schedule != 0;
    return CIECU_OK;
}

int ciecu_pcg_debug_exchange(ciecu_pcg S, int64_t waitNanoseconds, int64_t withholdExchange) {
    CIECU_REQUIRE(S, "pcg_debug_exchange: null solver");
    CIECU_REQUIRE(waitNanoseconds >= 1000 && waitNanoseconds <= 60000000000LL,
                  "pcg_debug_exchange: the wait limit must be in [1 us, 60 s]");
    CIECU_REQUIRE(withholdExchange >= 0, "pcg_debug_exchange: negative exchange index");
    S->waitNs = waitNanoseconds;
    S->withholdExchange = withholdExchange;
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
    bool persistent = false;
    CIECU_TRY(use_persistent(S, &persistent));
    if (persistent) {
        CIECU_TRY(ensure_persistent_buffers(S));
    } else {
        CIECU_TRY(refresh_dia(S, st));
        CIECU_TRY(tune_solver_spmv(S));
    }
    S->persistent = persistent;
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
        double* p0 = persistent ? S->z : S->p;  // the single launch forms p_0 from z_0
        if (S->dinv)
            pcg_init_kernel<true><<<fit_grid(pcg_init_kernel<true>, kT, needV), kT, 0, st>>>(
                n, S->r, S->dinv, p0, S->d_s, S->d_partials, S->d_counter);
        else
            pcg_init_kernel<false><<<fit_grid(pcg_init_kernel<false>, kT, needV), kT, 0, st>>>(
                n, S->r, S->dinv, p0, S->d_s, S->d_partials, S->d_counter);
        count_launch();
        CIECU_CHECK_LAUNCH("pcg_init_kernel");
    }
    if (S->settings.iterationCount > 0 && persistent) {
        CIECU_TRY(run_persistent(S, st));
    } else if (S->settings.iterationCount > 0) {
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
    }
    if (S->settings.iterationCount > 0) {
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
