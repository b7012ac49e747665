/*
 * ciecu host utilities: set-up of the assembly path that the reference also runs
 * on the host (DoF numbering, sparsity pattern, colouring) and the seeded
 * synthetic inputs.  These functions need no GPU.
 */
#ifndef CIECU_HOST_H
#define CIECU_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* DoF map of a structured grid of Q_order Lagrange cells (cells[0..dim-1]
 * elements per axis on the unit box): nodes numbered lexicographically, x
 * fastest; local basis index first-1-D-index-fastest (AnsatzSpace_impl.hpp:599-657).
 * Replaces Assembler::addGraph's BFS numbering (fem/packages/graph/impl/Assembler_impl.hpp:22-153)
 * for structured grids.  h_dofmap: ncells * (order+1)^dim. */
int ciecu_structured_dofmap(int dim, int order, const int32_t* cells, int32_t* h_dofmap, int32_t* h_ndofs);
/* 1 for nodes on the boundary of the box, else 0. */
int ciecu_structured_boundary(int dim, int order, const int32_t* cells, uint8_t* h_isBoundary);
/* Assembler::makeCSRMatrix (fem/packages/graph/src/Assembler.cpp:55-175): row
 * extents (ndofs+1) and, when h_columnIndices is non-NULL, the sorted unique
 * column indices.  Call once with h_columnIndices = NULL to size it. */
int ciecu_csr_pattern(int64_t ncells, int nb, const int32_t* h_dofmap, int32_t ndofs, int32_t* h_rowExtents,
                      int32_t* h_columnIndices, int64_t* h_nnz);
/* 2^dim colours of a structured grid (parity of the cell coordinates): cells of
 * one colour share no DoF, so their scatter needs no atomics. */
int ciecu_structured_colors(int dim, const int32_t* cells, int32_t* h_color);
/* Greedy colouring of an arbitrary DoF map (at most 64 colours). */
int ciecu_greedy_colors(int64_t ncells, int nb, const int32_t* h_dofmap, int32_t ndofs, int32_t* h_color,
                        int32_t* h_colorCount);
/* std::mt19937_64(seed) mapped to [-1, 1] as ((x >> 11) * 2^-53) * 2 - 1. */
int ciecu_random_uniform(uint64_t seed, int64_t n, double* h_out);
/* Box-Muller normals from the same stream (u1, u2 consecutive). */
int ciecu_random_normal(uint64_t seed, int64_t n, double* h_out);
/* kappa_e = exp(g_e): i.i.d. N(0,1) per cell convolved with a separable Gaussian
 * kernel (standard deviation sigma cells, truncated at +-truncation cells,
 * clamped at the boundary), standardised to zero mean and unit variance. */
int ciecu_kappa_field(uint64_t seed, int dim, const int32_t* cells, double sigma, int truncation, double* h_kappa);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_HOST_H */
