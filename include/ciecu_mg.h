/*
 * ciecu two-level multigrid-preconditioned conjugate gradients on the device.
 *
 * No reference counterpart as a class: the reference composes multigrid from its
 * operator algebra (executables/fem_examples/src/poisson2D/solver.cpp:111-232) and
 * runs ConjugateGradients (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201).
 * Here the outer CG and the whole cycle run on the device in one CUDA graph with
 * a device-side loop: no host synchronisation per iteration.
 */
#ifndef CIECU_MG_H
#define CIECU_MG_H

#include <stdint.h>

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ciecu_mgcg_s* ciecu_mgcg;

typedef struct {
    int degree;           /* Chebyshev degree of the pre- and of the post-smoothing (>= 1) */
    double lambdaMax;     /* upper spectral bound of D^-1 A; <= 0: 1.1 x a 20-step power estimate */
    double ratio;         /* the smoother damps [lambdaMax / ratio, lambdaMax] (> 1) */
    int coarseIterations; /* Jacobi-PCG iterations of the coarse solve in every cycle (>= 1) */
    int flexible;         /* 1: flexible CG (beta = r+^T (z+ - z) / r^T z), for a cycle that is not a fixed
                             linear operator (truncated coarse solve, single-precision smoothing) */
} ciecu_mg_options;

/* Conjugate gradients on `fine` (FP64; Jacobi diagonal d_fineInverseDiagonal)
 * preconditioned by the symmetric two-level cycle
 *     z  = S r;   z += P C (R (r - A z));   z += S (r - A z)
 * S: Chebyshev polynomial in D^-1 A of options.degree; P (fine x coarse) and
 * R (coarse x fine): transfer operators; C: options.coarseIterations Jacobi-PCG
 * iterations on `coarse` from zero.  smoother32 (may be NULL): an FP32 copy of
 * the fine matrix in the same pattern (e.g. from ciecu_assemble_embedded_f32);
 * then the smoothing and the cycle's residuals run in FP32 on it, the transfers
 * and the coarse solve in FP64, and the outer iteration in FP64 on `fine`.
 * Statistics and stopping rule follow ConjugateGradients (recursive residual,
 * relative to ||b - A x0||).  The matrices' arrays must outlive the solver. */
int ciecu_mgcg_create(ciecu_csr fine, const double* d_fineInverseDiagonal, ciecu_csr smoother32,
                      ciecu_csr prolongation, ciecu_csr restriction, ciecu_csr coarse,
                      const double* d_coarseInverseDiagonal, ciecu_mg_options options, ciecu_statistics settings,
                      ciecu_mgcg* out);
int ciecu_mgcg_destroy(ciecu_mgcg solver);
/* out = inScale * out + outScale * x, x = the solution from the initial guess out. */
int ciecu_mgcg_product(ciecu_mgcg solver, double inScale, const double* d_in, double outScale, double* d_out,
                       ciecu_statistics* h_stats);
/* The smoother's spectral bound and the cycles applied by the last solve. */
int ciecu_mgcg_info(ciecu_mgcg solver, double* h_lambdaMax, int64_t* h_cycles);
/* The FP32 smoother's column storage: offsets16 = 1 when it reads 16-bit column
 * offsets from the row (every |col - row| < 2^15; 6 instead of 8 bytes per entry,
 * built at creation), with the lanes per row chosen by timing; 0 / 0 otherwise
 * (int32 columns through the CSR handle's own tuned kernel, or no FP32 smoother). */
int ciecu_mgcg_smoother_info(ciecu_mgcg solver, int* offsets16, int* lanesPerRow);
/* The coarse solve's form.  clusterCtas > 0: the coarse matrix has a structured
 * Q1 stencil (27 diagonals in 3D, 9 in 2D, lexicographic order) small enough for
 * one thread-block cluster of that many CTAs to hold its FP32 upper half in shared
 * memory, and every coarse solve of a cycle then runs in one launch (checked at
 * creation); 0: the pipelined kernels, one launch per coarse iteration.  active =
 * 1 when the last solve used the cluster (its values were bitwise symmetric in
 * FP32; checked at every solve). */
int ciecu_mgcg_coarse_info(ciecu_mgcg solver, int* clusterCtas, int* active);
/* enable = 0: the pipelined coarse kernels even where the cluster form applies
 * (for comparison); 1 (the default): the cluster form where it applies.  Takes
 * effect at the next solve. */
int ciecu_mgcg_set_coarse_cluster(ciecu_mgcg solver, int enable);
/* d_out = C d_in: the cycle's coarse solve alone (coarse rows; the form of
 * ciecu_mgcg_coarse_info, the coarse values read as at a solve). */
int ciecu_mgcg_coarse_apply(ciecu_mgcg solver, const double* d_in, double* d_out);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_MG_H */
