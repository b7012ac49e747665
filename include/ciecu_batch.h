/*
 * ciecu batched solvers: many independent SPD systems in one device-resident
 * Jacobi-preconditioned CG.  No reference counterpart as one object: the reference
 * runs one ConjugateGradients per system
 * (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201); here every
 * system follows that algorithm -- its own alpha, beta, stopping test
 * (Comparison::less on the recursive residual, relative to its own ||r0||) and
 * iteration count -- while all systems share each kernel launch.
 */
#ifndef CIECU_BATCH_H
#define CIECU_BATCH_H

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ciecu_batch_s* ciecu_batch;

/* lhs: the systems' matrices as one block-diagonal FP64 CSR; system s owns rows
 * and columns h_rowOffsets[s] .. h_rowOffsets[s+1]-1 (systems + 1 offsets, the
 * first 0, the last the row count; every system at least one row).  An entry
 * outside its system's column block is rejected (CIECU_ERR_ARGUMENT).
 * d_inverseDiagonal: the Jacobi preconditioner of all rows (ciecu_diagonal_inverse_f64).
 * settings apply to every system.  Creation autotunes the lanes per row of the
 * SpMV on lhs. */
int ciecu_batch_create(ciecu_csr lhs, int64_t systems, const int64_t* h_rowOffsets,
                       const double* d_inverseDiagonal, ciecu_statistics settings, ciecu_batch* out);
int ciecu_batch_destroy(ciecu_batch solver);
/* Lanes per row chosen by the autotuner, whether the solve loop runs on the device
 * (conditional graph nodes), and the number of row tiles -- of the form the solver
 * is set to (FP64, restarted FP32 refinement or FP32 with reliable updates; the
 * loop flag is known once that form has solved). */
int ciecu_batch_info(ciecu_batch solver, int* lanesPerRow, int* deviceLoop, int64_t* tiles);
/* All systems at once: initial guess = d_out; on return out = inScale*out +
 * outScale*x per row.  h_stats (may be NULL): one ciecu_statistics per system.
 * A breakdown in any system returns CIECU_ERR_BREAKDOWN naming the first such
 * system; the other systems are solved and their statistics filled. */
int ciecu_batch_product(ciecu_batch solver, double inScale, const double* d_in, double outScale,
                        double* d_out, ciecu_statistics* h_stats);
/* innerTolerance > 0: later products run FP32 inner solves with FP64 refinement
 * -- each round solves the FP32 copy of the matrix to innerTolerance relative
 * to the current residual for the systems not yet converged, adds the
 * correction to the FP64 solution and recomputes r = b - A x in FP64; a system
 * stops on its true FP64 residual.  statistics: inner (FP32) iterations and the
 * true residuals.  0 (the default): the FP64 solve.  The first call with a
 * positive tolerance allocates the FP32 copies and autotunes their SpMV. */
int ciecu_batch_set_refinement(ciecu_batch solver, double innerTolerance);
/* delta in (0, 1): every system iterates in FP32 (FP32 copies of the values and
 * of D^-1, FP32 vectors, FP64 dot products) with FP64 reliable updates: when a
 * system's FP32 residual norm fell below delta times its largest value since the
 * last replacement (or below the stopping tolerance, or at the iteration limit),
 * its FP32 solution is added to the FP64 one and its residual recomputed as
 * b - A x in FP64; the Krylov space is kept across replacements.  The stopping
 * test and the statistics use that FP64 residual (iterationCount = FP32
 * iterations).  Takes precedence over ciecu_batch_set_refinement; 0 (default):
 * off. */
int ciecu_batch_set_reliable_updates(ciecu_batch solver, double delta);
/* FP64 residual replacements of each system in the last reliable-update solve. */
int ciecu_batch_refinements(ciecu_batch solver, int64_t* h_perSystem);

#ifdef __cplusplus
}
#endif

#endif /* CIECU_BATCH_H */
