/*
 * ciecu multi-right-hand-side solver (SpMM-CG): k <= 32 independent
 * Jacobi-preconditioned CG solves against one FP64 CSR matrix, sharing every
 * matrix read.  Each right-hand side follows ConjugateGradients::product
 * (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201) with its own
 * scalars, stopping test and statistics; no reference counterpart as one object
 * (the reference would run one solver per right-hand side).
 * Blocks of vectors are row-major n x k: entry (i, c) at i*k + c.
 */
#ifndef CIECU_MULTI_H
#define CIECU_MULTI_H

#include <stdint.h>

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ciecu_multi_s* ciecu_multi;

int ciecu_multi_create(ciecu_csr lhs, int rhsCount, const double* d_inverseDiagonal, ciecu_statistics settings,
                       ciecu_multi* out);
int ciecu_multi_destroy(ciecu_multi solver);
/* Lanes per row group (the power of two >= rhsCount; 8 when rhsCount = 32 and
 * the right-hand sides are 16-byte aligned: four columns per lane) and whether
 * the solve loop runs on the device (conditional graph nodes). */
int ciecu_multi_info(ciecu_multi solver, int* lanesPerRow, int* deviceLoop);
/* SpMM format chosen at the first solve: the number of diagonals of the
 * diagonal-storage copy (a matrix of at most 32 diagonals, see
 * ciecu_csr_diagonals, whose copy timed faster than the CSR SpMM; the copy is
 * refilled from the CSR values at every solve), or 0 for the CSR SpMM. */
int ciecu_multi_format(ciecu_multi solver, int* diagonals);
/* Pins the SpMM format instead of timing it at the first solve: 1 the DIA copy
 * (when the matrix has one; CSR otherwise), 0 CSR, -1 timed (default).  For
 * tests and profiling.  With 32 right-hand sides and a stencil whose offsets come
 * in consecutive triples (the Q1 stencils), the DIA SpMM keeps four rows per lane
 * and loads each operand row of a triple once; ciecu_multi_format reports the
 * diagonal count either way. */
int ciecu_multi_set_format(ciecu_multi solver, int format);
/* delta in (0, 1): FP32-refined form -- every column iterates in FP32 (FP32
 * copies of the matrix in the format of the FP64 solve and of D^-1, FP32 blocks,
 * FP64 dot products) with FP64 reliable updates: every running column's FP32
 * solution is added to its FP64 one and its residual recomputed as B - A X in
 * FP64 (one FP64 SpMM serves all columns, so they replace together) when some
 * column's FP32 residual norm fell below the stopping tolerance, or it hit the
 * iteration limit or an FP32 breakdown, or when at least half of the running
 * columns saw their FP32 residual norm fall below delta times its largest value
 * since the last replacement; each column keeps its search direction.  The
 * stopping test and the statistics use that FP64 residual (iterationCount = FP32
 * iterations).  delta = 0 (default): FP64 iterations as
 * ConjugateGradients::product. */
int ciecu_multi_set_refinement(ciecu_multi solver, double delta);
/* FP64 residual recomputations of each column in the last refined solve. */
int ciecu_multi_refinements(ciecu_multi solver, int64_t* h_perColumn);
/* Initial guesses = d_out (n x k); on return out = inScale*out + outScale*X.
 * h_stats (may be NULL): one ciecu_statistics per right-hand side.  A breakdown
 * returns CIECU_ERR_BREAKDOWN naming the first such right-hand side; the others
 * are solved and reported. */
int ciecu_multi_product(ciecu_multi solver, double inScale, const double* d_in, double outScale, double* d_out,
                        ciecu_statistics* h_stats);

#ifdef __cplusplus
}
#endif

#endif /* CIECU_MULTI_H */
