/*
 * ciecu graph set-up on the device: the bandwidth-reducing reordering of a CSR
 * matrix (Cuthill-McKee and reverse Cuthill-McKee) with the matching permutation
 * of matrices and vectors, and the sparsity pattern of a DoF map.
 */
#ifndef CIECU_GRAPH_H
#define CIECU_GRAPH_H

#include <stdint.h>

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Most rows per row of the graph the device set-up handles: a row (reordering,
 * permutation) or the DoFs of the cells around a DoF (pattern) may hold at most
 * this many entries; longer ones fail with CIECU_ERR_ARGUMENT. */
#define CIECU_GRAPH_MAX_ROW 1024

/* makeReordering (linalg/packages/utilities/src/reorder.cpp:23-173) on the device.
 * map[k] = the old row placed at position k.  strategy 1: Cuthill-McKee, 2:
 * reverse Cuthill-McKee (the CM map reversed).  The traversal starts at the row
 * of least degree (row length; the lowest index among equals), visits rows in
 * the order they were queued, and queues each visited row's unqueued neighbours
 * (its column indices) by ascending degree, equal degrees in ascending index;
 * when the queue runs dry the unqueued row of least degree starts the next
 * component.  It runs breadth-first level by level: the rows of a level are
 * claimed by the first (lowest-placed) row of the previous level adjacent to
 * them, which is the row that queues them in the sequential order.  The
 * reference sorts each queued batch with std::sort, whose order among equal
 * degrees is unspecified; for batches of at most 16 rows the library's sort is
 * an insertion sort, which keeps the ascending index order used here.
 * d_rowExtents / d_columnIndices: a square pattern whose rows hold distinct
 * columns. */
int ciecu_make_reordering(ciecu_space space, int32_t n, const int32_t* d_rowExtents, const int32_t* d_columnIndices,
                          int strategy, int32_t* d_map);
/* reorder<int,double,false> (reorder.cpp:215-365) out of place: new row i is old
 * row map[i], every column c becomes inverse(map)[c], and each new row is sorted
 * by its new columns (values follow their columns).  The output arrays hold
 * n + 1, nnz and nnz entries. */
int ciecu_reorder_csr(ciecu_space space, int32_t n, const int32_t* d_map, const int32_t* d_rowExtents,
                      const int32_t* d_columnIndices, const double* d_entries, int32_t* d_newRowExtents,
                      int32_t* d_newColumnIndices, double* d_newEntries);
/* reorder (reverse = 0: out[i] = in[map[i]]) and reverseReorder (reverse = 1:
 * out[map[i]] = in[i]) of a vector (reorder.cpp:368-425). */
int ciecu_reorder_vector(ciecu_space space, int64_t n, const int32_t* d_map, int reverse, const double* d_in,
                         double* d_out);

/* Assembler::makeCSRMatrix (fem/packages/graph/src/Assembler.cpp:55-175) on the
 * device: row i holds the sorted, distinct DoFs of every cell whose DoF list
 * contains i.  Call once with d_columnIndices = NULL to get the row extents
 * (ndofs + 1 on the device) and the entry count in *h_nnz, then again with the
 * column array (the row extents of the first call in d_rowExtents) to fill it.
 * d_dofmap: ncells * nb DoF indices in [0, ndofs). */
int ciecu_csr_pattern_device(ciecu_space space, int64_t ncells, int nb, const int32_t* d_dofmap, int32_t ndofs,
                             int32_t* d_rowExtents, int32_t* d_columnIndices, int64_t* h_nnz);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_GRAPH_H */
