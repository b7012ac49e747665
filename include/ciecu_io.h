/*
 * ciecu I/O: the linear system in MatrixMarket text, as the reference writes it
 * before solving (executables/fem_examples/src/poisson2D/solver.cpp:521-539).
 */
#ifndef CIECU_IO_H
#define CIECU_IO_H

#include <stdint.h>

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* cie::io::MatrixMarket::Output::operator() for a CSR matrix
 * (cieutils/packages/io/inc/MatrixMarket.hpp:17-61, src/MatrixMarket.cpp): the
 * header "%%MatrixMarket matrix coordinate real general", the line
 * "rows columns nonzeros", then one line "row column value" per stored entry
 * (1-based indices, rows in order, entries in storage order, values as a C++
 * stream prints a double by default, i.e. printf "%g").  Host arrays; the text
 * is formatted on all host threads and written in order.  The file is replaced. */
int ciecu_write_matrix_market_host(const char* path, int64_t rows, int64_t columns, const int32_t* h_rowExtents,
                                   const int32_t* h_columnIndices, const double* h_entries);
/* The same for a device CSR handle (FP64 values): copies the arrays to the host
 * on the handle's stream, then writes them as above. */
int ciecu_write_matrix_market(ciecu_csr csr, const char* path);
/* The vector overload (MatrixMarket.cpp, "array" format): header
 * "%%MatrixMarket matrix array real general", the line "n 1", then one value per
 * line.  d_values: n doubles on the device of `space`, copied on its stream. */
int ciecu_write_matrix_market_vector(ciecu_space space, int64_t n, const double* d_values, const char* path);
int ciecu_write_matrix_market_vector_host(const char* path, int64_t n, const double* h_values);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_IO_H */
