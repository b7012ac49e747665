/*
 * ciecu -- C-ABI of the B200 (sm_100a) backend for the kelofm/cie linear-solve
 * hot path: CSR operators, the linalg space, Jacobi-preconditioned CG, the
 * smoothers and multigrid pieces built from them, and the per-element stiffness
 * assembly that fills the CSR matrix.
 *
 * Conventions
 *  - Every function returns 0 (CIECU_OK) or a CIECU_ERR_* code; the message of the
 *    last failure on the calling thread is available through ciecu_last_error.
 *    No C++ exception crosses this boundary; the C++ wrapper (cie_cuda/linalg.hpp)
 *    turns a non-zero status into an exception, like CIE_CHECK / CIE_THROW
 *    (cieutils/packages/macros/inc/checks.hpp:17-23).
 *  - Pointers named d_* are device pointers, h_* host pointers.  Sizes are element
 *    counts.  All work is ordered on the stream of the ciecu_space it is issued
 *    through; functions that return a value to the host synchronise that stream.
 *  - Operator products follow LinearOperator::product
 *    (linalg/packages/solvers/inc/LinearOperator.hpp:15-33):
 *        out <- inScale * out + outScale * Op(in).
 */
#ifndef CIECU_H
#define CIECU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ciecu_status {
    CIECU_OK = 0,
    CIECU_ERR_ARGUMENT = 1,   /* invalid argument or size mismatch (CIE_CHECK failures) */
    CIECU_ERR_CUDA = 2,       /* CUDA runtime error */
    CIECU_ERR_BREAKDOWN = 3,  /* CG breakdown: p^T A p <= 0 or r^T z <= 0 */
    CIECU_ERR_DIAGONAL = 4,   /* missing or zero diagonal entry */
    CIECU_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
    CIECU_ERR_PATTERN = 6     /* element entry not present in the CSR pattern */
};

enum ciecu_value_type { CIECU_F64 = 0, CIECU_F32 = 1 };

typedef struct ciecu_space_s* ciecu_space;
typedef struct ciecu_csr_s* ciecu_csr;
typedef struct ciecu_pcg_s* ciecu_pcg;

/* IterativeSolver::Statistics (linalg/packages/solvers/inc/IterativeSolver.hpp:21-25):
 * used both as solver settings (limits) and as reported results. */
typedef struct ciecu_statistics {
    int64_t iterationCount;
    double absoluteResidual;
    double relativeResidual;
} ciecu_statistics;

/* ---- errors / library ------------------------------------------------------- */

/* Copies the last error message of the calling thread; returns its length. */
int ciecu_last_error(char* h_buffer, int size);
/* Number of kernels this library launched since load (instrumentation). */
int64_t ciecu_kernel_launch_count(void);
int ciecu_device_info(int* smCount, int* ccMajor, int* ccMinor);

/* ---- space: SYCLSpace / DefaultSpace counterpart ------------------------------
 * linalg/packages/solvers/inc/LinalgSpace.hpp:10-35 (LinalgSpaceLike),
 * linalg/packages/solvers/inc/SYCLSpace.hpp:66-131 (queue-owning backend).
 * A space owns one CUDA stream (or borrows the given one) and the scratch used
 * by its reductions.  One host thread drives one space, like the reference. */
int ciecu_space_create(void* cudaStream, ciecu_space* out);
int ciecu_space_destroy(ciecu_space space);
int ciecu_space_synchronize(ciecu_space space);
void* ciecu_space_stream(ciecu_space space);

/* SYCLSpace::makeVector / DeviceMemory (cieutils/packages/concurrency/inc/sycl.hpp:33-71) */
int ciecu_alloc(ciecu_space space, size_t bytes, void** d_out);
int ciecu_free(ciecu_space space, void* d_ptr);
/* SYCLSpace::assign(view, span) / assign(span, view) (SYCLSpace.cpp:262-313) */
int ciecu_memcpy_h2d(ciecu_space space, void* d_dst, const void* h_src, size_t bytes);
int ciecu_memcpy_d2h(ciecu_space space, void* h_dst, const void* d_src, size_t bytes);
int ciecu_memcpy_d2d(ciecu_space space, void* d_dst, const void* d_src, size_t bytes);

/* DefaultSpace<double> / SYCLSpace<double> BLAS-1 (DefaultSpace.cpp:50-187,
 * SYCLSpace.cpp:114-343).  Note scale(t, s, alpha) is the ELEMENTWISE product
 * t = alpha * t (.) s (DefaultSpace.cpp:81-106). */
int ciecu_dot_f64(ciecu_space space, int64_t n, const double* d_left, const double* d_right, double* h_result);
int ciecu_scale_elementwise_f64(ciecu_space space, int64_t n, double* d_target, const double* d_source, double alpha);
int ciecu_scale_f64(ciecu_space space, int64_t n, double* d_vector, double alpha);
int ciecu_add_f64(ciecu_space space, int64_t n, double* d_target, const double* d_source, double alpha);
int ciecu_assign_f64(ciecu_space space, int64_t n, double* d_target, const double* d_source);
int ciecu_fill_f64(ciecu_space space, int64_t n, double* d_vector, double value);
/* DefaultSpace<float> / SYCLSpace<float> (FP32 vectors; the dot accumulates in FP64) */
int ciecu_dot_f32(ciecu_space space, int64_t n, const float* d_left, const float* d_right, double* h_result);
int ciecu_scale_elementwise_f32(ciecu_space space, int64_t n, float* d_target, const float* d_source, float alpha);
int ciecu_scale_f32(ciecu_space space, int64_t n, float* d_vector, float alpha);
int ciecu_add_f32(ciecu_space space, int64_t n, float* d_target, const float* d_source, float alpha);
int ciecu_assign_f32(ciecu_space space, int64_t n, float* d_target, const float* d_source);
int ciecu_fill_f32(ciecu_space space, int64_t n, float* d_vector, float value);
int ciecu_convert_f64_to_f32(ciecu_space space, int64_t n, float* d_target, const double* d_source);
int ciecu_convert_f32_to_f64(ciecu_space space, int64_t n, double* d_target, const float* d_source);

/* ---- CSR operator -----------------------------------------------------------
 * CSRView (linalg/packages/utilities/inc/CSRView.hpp:11-86) over DEVICE arrays,
 * plus the SpMV schedule chosen by the autotuner.  The arrays are not copied and
 * must outlive the handle (the view is non-owning, like CSRView).
 * Constructor checks of CSROperator.cpp:21-29. */
int ciecu_csr_create(ciecu_space space, int32_t rowCount, int32_t columnCount, int64_t nnz,
                     const int32_t* d_rowExtents, const int32_t* d_columnIndices,
                     const void* d_entries, int valueType, ciecu_csr* out);
int ciecu_csr_destroy(ciecu_csr csr);
/* SpMV kernel choice: 0 = autotune (default), 1 = row-block stream kernel
 * (bit-compatible row sums), 2/4/8/16/32 = that many lanes per row. */
int ciecu_csr_set_kernel(ciecu_csr csr, int kernel);
int ciecu_csr_get_kernel(ciecu_csr csr, int* kernel);
/* Number of diagonals of the matrix's diagonal-storage copy, used by the FP64
 * PCG (schedule 64) and the mixed solver's inner matrix (innerKernel -2): the
 * distinct offsets c - r when there are at most 32 of them, the columns of every
 * row strictly ascend and at least 60 % of the stored entries are nonzeros; 0
 * otherwise.  The analysis runs once per handle (one pass over the pattern). */
int ciecu_csr_diagonals(ciecu_csr csr, int* ndiag);
/* Runs the autotuner now (otherwise it runs on the first product). */
int ciecu_csr_autotune(ciecu_csr csr);

/* CSROperator<int,double>::product (CSROperator.cpp:33-111),
 * SYCLCSROperator::product (SYCLCSROperator.cpp:32-89). */
int ciecu_csr_spmv_f64(ciecu_csr csr, double inScale, const double* d_in, double outScale, double* d_out);
/* CSROperator<int,float>::product for a CIECU_F32 matrix. */
int ciecu_csr_spmv_f32(ciecu_csr csr, float inScale, const float* d_in, float outScale, float* d_out);
/* MaskedCSROperator<int,double,double,uint16_t>::product (MaskedCSROperator.cpp:37-118):
 * rows/columns with mask >= threshold are excluded; masked rows receive
 * combine(inScale, out, outScale, 0) (CPU semantics, :51-66). */
int ciecu_csr_masked_spmv_f64(ciecu_csr csr, const uint16_t* d_mask, uint16_t threshold,
                              double inScale, const double* d_in, double outScale, double* d_out);

/* ---- diagonal / smoothers ----------------------------------------------------- */

/* makeDiagonalOperator (DiagonalOperator.cpp:56-88): d_inverse[i] = 1 / a_ii.
 * Fails with CIECU_ERR_DIAGONAL naming the first row whose diagonal is missing
 * or zero (the CPU semantics; the SYCL variant stores max() instead). */
int ciecu_diagonal_inverse_f64(ciecu_csr csr, double* d_inverse);
/* DiagonalOperator::product (DiagonalOperator.cpp:37-53): out = inScale*out + outScale*(in (.) D^-1). */
int ciecu_diagonal_apply_f64(ciecu_space space, int64_t n, const double* d_inverse, double inScale,
                             const double* d_in, double outScale, double* d_out);
/* JacobiOperator<..>::product (JacobiOperator.cpp:36-62) with the diagonal
 * preconditioner as inverse diagonal: from x0 = 0, `iterations` sweeps of
 * x <- x + relaxation * D^-1 (in - A x); out = inScale*out + outScale*x.
 * d_mask may be NULL; otherwise A is the masked operator of
 * ciecu_csr_masked_spmv_f64 (the p-multigrid smoother of solver.cpp:178-206).
 * d_work: 2n doubles of scratch. */
int ciecu_jacobi_f64(ciecu_csr csr, const double* d_inverse, const uint16_t* d_mask, uint16_t threshold,
                     int64_t iterations, double relaxation, double inScale, const double* d_in,
                     double outScale, double* d_out, double* d_work);
/* Allocation-free ciecu_jacobi_f64: the same sweeps and result, without d_work.
 * No counterpart in the reference.
 * It is for callers that cannot allocate device memory at the call: hosts whose
 * own pool owns every byte of device memory and that forbid a library from
 * calling cudaMalloc behind their back, and code on a path where cudaMalloc or
 * cudaFree would fail or stall -- both are refused while a stream is being
 * captured in global mode, and cudaFree waits for the whole device.
 * The two iterates live in a static device array inside this library, 4 MiB:
 * matrices of more than CIECU_JACOBI_STATIC_MAX_ROWS rows are rejected with
 * CIECU_ERR_ARGUMENT.  The call makes no cudaMalloc, cudaFree or other
 * allocating call (an untuned matrix is not tuned, since tuning allocates; its
 * row schedule then follows from the mean row length).
 * The first call on a device looks up the array's device address once, with
 * that device current (it must be the matrix's device): make the first call
 * before any stream capture.  The address is remembered with the identity of the
 * device's context; after a reset of the device (cudaDeviceReset) the next call
 * looks it up again, so that call too belongs before any capture.  All calls on a device share the one array, which
 * keeps the last call's contents; every iterate is written in full before it is
 * read, so nothing has to start at zero.  Calls that overlap on the GPU (other
 * streams, other host threads, other matrices on the same device) race on the
 * array and corrupt each other's results: serialise them. */
#define CIECU_JACOBI_STATIC_MAX_ROWS 262144
int ciecu_jacobi_f64_static(ciecu_csr csr, const double* d_inverse, const uint16_t* d_mask, uint16_t threshold,
                            int64_t iterations, double relaxation, double inScale, const double* d_in,
                            double outScale, double* d_out);
/* MaskedIdentityOperator<..>::product (MaskedIdentityOperator.cpp:14-74):
 * out = combine(inScale, out, outScale, mask < threshold ? in : 0). */
int ciecu_masked_identity_f64(ciecu_space space, int64_t n, const uint16_t* d_mask, uint16_t threshold,
                              double inScale, const double* d_in, double outScale, double* d_out);
/* Chebyshev polynomial smoother of the given degree for D^-1 A on
 * [lambdaMin, lambdaMax] (no reference counterpart; replaces damped Jacobi in the
 * multigrid).  out = inScale*out + outScale*S(in).  d_work: 3n doubles. */
int ciecu_chebyshev_f64(ciecu_csr csr, const double* d_inverse, int degree, double lambdaMin,
                        double lambdaMax, double inScale, const double* d_in, double outScale,
                        double* d_out, double* d_work);
/* Largest eigenvalue estimate of D^-1 A by `iterations` power steps (Chebyshev
 * bounds).  d_work: 2n doubles. */
int ciecu_power_lambda_max_f64(ciecu_csr csr, const double* d_inverse, int iterations, uint64_t seed,
                               double* d_work, double* h_lambda);

/* ---- conjugate gradients ------------------------------------------------------
 * ConjugateGradients<TSpace> (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201)
 * with an optional inverse-diagonal (Jacobi) preconditioner.  The solver object
 * owns its work vectors and device scalars, like the reference's buffers.
 * Initial guess = d_out on entry; on return out = inScale*out + outScale*x.
 * Stopping rule, breakdown errors and reported statistics follow the reference:
 * stop on the recursive residual with Comparison::less against the absolute or
 * relative limit; iterationCount = loop index at the break. */
int ciecu_pcg_create(ciecu_csr lhs, const double* d_inverseDiagonal, ciecu_statistics settings,
                     int verbosity, ciecu_pcg* out);
int ciecu_pcg_destroy(ciecu_pcg solver);
int ciecu_pcg_product(ciecu_pcg solver, double inScale, const double* d_in, double outScale,
                      double* d_out, ciecu_statistics* h_stats);
/* Iterations captured per CUDA graph launch between host convergence checks
 * (used when the device-side loop of conditional graph nodes is unavailable). */
int ciecu_pcg_set_graph_chunk(ciecu_pcg solver, int iterations);
/* Pins the schedule of the solver's fused q = A p kernel (1 = row-block stream
 * kernel, 2..32 = lanes per row, 64 = a diagonal-storage copy of the matrix, for
 * square matrices with strictly ascending columns whose nonzeros lie on at most
 * 32 diagonals, at least 60 % filled; the copy is refilled from the CSR values at
 * every solve) instead of autotuning it at the first solve; 0 returns to
 * autotuning.  For runs whose timings would mislead the autotuner (under a
 * profiler).  A pinned 64 on a matrix without a diagonal copy fails at the solve
 * with CIECU_ERR_ARGUMENT.  The schedules are kernels of the graph loop: with the
 * loop mode 0 a pinned schedule (non-zero) selects the graph loop, and with mode 2
 * (single launch) the pin has no effect. */
int ciecu_pcg_set_schedule(ciecu_pcg solver, int schedule);
/* SpMV schedule the solver's autotuner chose for its fused q = A p kernel (0 before
 * the first solve or when the solve ran as a single launch; 1 = row-block stream
 * kernel, else lanes per row) and how the last solve ran: host-polled graph chunks
 * (0), a device-side graph loop (1) or a single cooperative launch (2). */
int ciecu_pcg_info(ciecu_pcg solver, int* spmvSchedule, int* deviceLoop);
/* The diagonal-storage copy at the last solve: the diagonals K1 reads (0: no
 * copy) and whether they are the upper half (main diagonal included) of a bitwise
 * symmetric matrix, checked at every solve, whose lower entries K1 reads back from
 * it (about half the matrix bytes; CIECU_DIA_SYMMETRIC=0 keeps the full copy). */
int ciecu_pcg_dia_info(ciecu_pcg solver, int* storedDiagonals, int* symmetric);
/* How the iterations run.  mode 0 (default): a single cooperative launch of at
 * most one block per SM (the fewest of SMs/4, SMs/2, SMs that fit), each block
 * holding its rows of the matrix in shared memory, when the rows fit there at one
 * block per SM, else the graph of three kernels per iteration; 1: always the
 * graph; 2: always the single launch (CIECU_ERR_ARGUMENT at the next solve when
 * the matrix does not fit).  The single launch gives results within rounding of
 * the graph's (its dot products are summed over another grid); a grid-wide wait
 * that gives up fails with CIECU_ERR_TIMEOUT. */
int ciecu_pcg_set_loop(ciecu_pcg solver, int mode);
/* Controls the bounded waits of the single-launch solve, for tests of its timeout
 * path (no counterpart in the reference).  waitNanoseconds bounds each grid-wide
 * exchange wait in global-timer nanoseconds (default 2 s; [1 us, 60 s]);
 * withholdExchange > 0 makes the last block skip publishing its partial sums at
 * that exchange of the next launches (counted from 1), so every wait on it runs
 * out, the launch ends and the solve fails with CIECU_ERR_TIMEOUT; 0 (default)
 * publishes normally.  The solver stays usable after a timeout. */
int ciecu_pcg_debug_exchange(ciecu_pcg solver, int64_t waitNanoseconds, int64_t withholdExchange);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_H */
