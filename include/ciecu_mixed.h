/*
 * ciecu mixed precision: FP32-inner Jacobi-PCG with FP64 refinement.
 * No counterpart in the reference, which solves in one precision
 * (ConjugateGradients<DefaultSpace<float|double>>, ConjugateGradients.cpp:10-17);
 * the settings, stopping rule and output combination follow
 * ConjugateGradients_impl.hpp:49-201, with the stop decided on the TRUE FP64
 * residual ||b - A x|| of the FP64 matrix.
 */
#ifndef CIECU_MIXED_H
#define CIECU_MIXED_H

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ciecu_mixed_s* ciecu_mixed;

typedef struct ciecu_mixed_options {
    /* 0: reliable updates (residual replacement keeping the search direction);
     * 1: classic iterative refinement (inner CG restarted after each correction). */
    int mode;
    /* mode 0: replace the residual when the FP32 residual norm fell below
     *         delta * its maximum since the last replacement (e.g. 0.1);
     * mode 1: inner relative tolerance of each correction solve (e.g. 1e-4). */
    double delta;
    /* 1: store column indices as 16-bit offsets from the row when the matrix
     * bandwidth is below 2^15 (checked; int32 otherwise). */
    int compressColumns;
    /* Inner SpMV kernel: 0 lets the autotuner choose; 1, 2 or 4 fixes the groups
     * of four entries each thread keeps in flight; -1 fixes the TMA-pipelined
     * kernel (matrix streamed through shared memory by bulk copies); -2 fixes a
     * diagonal-storage FP32 copy (square matrices with strictly ascending
     * columns whose nonzeros lie on at most 32 diagonals, at least 60 % filled;
     * CIECU_ERR_ARGUMENT otherwise).  The autotuner considers the diagonal copy
     * whenever the matrix qualifies. */
    int innerKernel;
    /* 1: the FP32 inner system is the symmetrically Jacobi-scaled matrix
     * D^-1/2 A D^-1/2 (unit diagonal), for matrices whose entries span many orders
     * of magnitude (embedded domains with a small material factor), where an
     * unscaled FP32 copy loses the small couplings and definiteness; the FP64
     * residuals, solution and stopping test are unchanged.  0: the unscaled copy. */
    int scaleInner;
    /* 1: keep z = D^-1 r as a vector and form the search direction and its
     * product inside the inner SpMV (w = A32 z, p = z + beta p, q = w + beta q):
     * two kernels per inner iteration instead of three, same vector traffic, and
     * q carried by recurrence (FP32 rounding drifts between residual
     * replacements).  0: q = A32 p after a separate direction kernel.  Measured
     * at 128^3 over the FP32 DIA copy: 28.0 ms fused against 29.4 ms.
     * 2: one kernel per inner iteration over the diagonal-storage copy: the
     * pending step x += alpha p, r -= alpha q, the direction p = D^-1 r + beta p
     * and q = A32 p in one row pass (neighbour rows' p formed from their gathered
     * r, q, p, D^-1), rho and ||r|| of the next residual expanded from FP64 sums
     * of r and q; r, p, q double-buffered.  With any other inner kernel it runs
     * as form 1 (ciecu_mixed_form reports which).  Measured at 128^3: 38.0 ms
     * against 27.7 ms for form 1 -- forming each operand entry from four gathered
     * vectors costs registers and instructions, and the latency-bound pass loses
     * more than the kernel it saves. */
    int fuseDirection;
} ciecu_mixed_options;

typedef struct ciecu_mixed_statistics {
    int64_t iterationCount;       /* FP32 inner iterations (FP32 SpMVs) */
    double absoluteResidual;      /* ||b - A64 x64|| at the last refinement */
    double relativeResidual;      /* ... / ||b - A64 x0|| */
    int64_t innerIterations;      /* = iterationCount */
    int64_t refinements;          /* FP64 residual recomputations */
    double trueRelativeResidual;  /* = relativeResidual */
} ciecu_mixed_statistics;

/* Builds the FP32 inner matrix -- SELL-32 layout (slices of 32 rows, one thread
 * per row, coalesced loads), FP32 values, 16-bit row-relative or int32 columns --
 * and the FP32 inverse diagonal from the FP64 matrix and its inverse diagonal
 * (both device).
 * settings: iteration limit (FP32 inner iterations) and tolerances. */
int ciecu_mixed_create(ciecu_csr lhs, const double* d_inverseDiagonal, ciecu_statistics settings,
                       ciecu_mixed_options options, ciecu_mixed* out);
int ciecu_mixed_destroy(ciecu_mixed solver);
/* compressedColumns: 1 when the inner matrix stores 16-bit offsets; groupUnroll:
 * groups of four entries each thread keeps in flight (chosen by the autotuner),
 * 0 when the autotuner chose the TMA-pipelined inner SpMV (the matrix streamed
 * through shared memory by bulk copies).  Synchronises the solver's stream and
 * returns CIECU_ERR_TIMEOUT if a pipelined ciecu_mixed_apply_f32 gave up a wait. */
int ciecu_mixed_info(ciecu_mixed solver, int* compressedColumns, int* groupUnroll);
int ciecu_mixed_set_graph_chunk(ciecu_mixed solver, int iterations);
/* d_out = A32 d_in: the solver's FP32 inner operator (FP32 values, 16-bit or
 * int32 columns) on its own, e.g. to time it. */
int ciecu_mixed_apply_f32(ciecu_mixed solver, const float* d_in, float* d_out);
/* Stored entries of the SELL-32 inner matrix, padding included (>= nnz). */
int ciecu_mixed_padded_entries(ciecu_mixed solver, int64_t* h_entries);
/* The FP32 diagonal-storage copy: its diagonals (0: none) and whether its row pass
 * loads each operand entry of a consecutive offset triple (o - 1, o, o + 1) once
 * (the Q1 stencils; CIECU_DIA_TRIPLES=0 in the environment turns it off). */
int ciecu_mixed_dia_info(ciecu_mixed solver, int* diagonals, int* triples);
/* Kernels per inner iteration of the solver's loop: 3, 2 (fuseDirection 1, or 2
 * without the diagonal copy) or 1 (fuseDirection 2 over the diagonal copy). */
int ciecu_mixed_form(ciecu_mixed solver, int* kernelsPerIteration);
/* out = inScale*out + outScale*x, x the refined solution (initial guess = out). */
int ciecu_mixed_product(ciecu_mixed solver, double inScale, const double* d_in, double outScale, double* d_out,
                        ciecu_mixed_statistics* h_stats);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_MIXED_H */
