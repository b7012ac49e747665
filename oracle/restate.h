/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the kelofm/cie algorithms on the linear-solve hot path.
 * It is the checker for the CUDA product (parity tests, smoke(), the CPU-baseline
 * leg of bench.py) and is never linked into or called by the product.
 *
 * Pinned by: the reference's own known-answer tests (tests/golden/, generated by
 * tests/golden/make_golden.py from the reference test sources) and, for the solver
 * half, by the reference's compiled CPU code (oracle/_ref/libcieref.so).
 */
#ifndef CIE_ORACLE_RESTATE_H
#define CIE_ORACLE_RESTATE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- linalg ---------------------------------------------------------- */
void ora_spmv(int nrows, const int* rowptr, const int* col, const double* val,
              double inScale, const double* in, double outScale, double* out);
void ora_masked_spmv(int nrows, const int* rowptr, const int* col, const double* val,
                     const uint16_t* mask, uint16_t threshold, double inScale,
                     const double* in, double outScale, double* out);
int ora_diag_inverse(int n, const int* rowptr, const int* col, const double* val, double* dinv);
double ora_dot(long n, const double* a, const double* b);
int ora_pcg(int n, const int* rowptr, const int* col, const double* val, const double* b,
            double* x, long maxIterations, double absoluteTolerance, double relativeTolerance,
            int precondition, double* stats);
void ora_jacobi(int n, const int* rowptr, const int* col, const double* val, const double* dinv,
                long iterations, double relaxation, double inScale, const double* in,
                double outScale, double* out);
void ora_chebyshev(int n, const int* rowptr, const int* col, const double* val,
                   const double* dinv, int degree, double lambdaMin, double lambdaMax,
                   const double* in, double* out);
double ora_power_lambda_max(int n, const int* rowptr, const int* col, const double* val,
                            const double* dinv, int iterations, uint64_t seed);

/* ---- fem ------------------------------------------------------------- */
int ora_gauss_legendre(int order, double* nodes, double* weights);
void ora_lagrange_1d(int count, const double* nodes, double x, double* values, double* derivatives);
void ora_stiffness_point(int dim, int setSize, const double* coefficients, int degree,
                         const double* point, double modulus, double* out);
void ora_element_stiffness(int dim, int order, int nq, const double* points,
                           const double* weights, double kappa, const double* h, int convention,
                           double* K);
void ora_structured_dofmap(int dim, int order, const int* cells, int* dofmap);
long ora_csr_pattern(long ncells, int nb, const int* dofmap, int ndofs, int* rowptr, int* col);
int ora_assemble(long ncells, int nb, const int* dofmap, const double* Ke, const int* rowptr,
                 const int* col, double* val);
void ora_element_gradient(long ncells, int nb, const int* dofmap, const double* Kunit,
                          const double* lambda, const double* u, double* grad);
void ora_dirichlet_eliminate(int n, const int* rowptr, const int* col, double* val,
                             const uint8_t* isBoundary, double* rhs);
int ora_cut_cell_points(int dim, int depth, int order, const double* center, double radius,
                        const double* cellOrigin, const double* cellSize, int maxPoints,
                        double* points, double* weights, double* scales, double alpha);
/* The same tree for the half-space normal . x < offset (physical coordinates). */
int ora_cut_cell_points_halfspace(int dim, int depth, int order, const double* normal, double offset,
                                  const double* cellOrigin, const double* cellSize, int maxPoints,
                                  double* points, double* weights, double* scales, double alpha);

int ora_dirichlet_penalty(int dim, int order, int quadratureOrder, const int* cells, const double* h,
                          double penalty, int faceMask, const double* g, const int* dofmap, const int* rowptr,
                          const int* col, double* val, double* rhs);

/* ---- graph ----------------------------------------------------------- */
int ora_cuthill_mckee(int n, const int* rowptr, const int* col, int strategy, int* map);

/* ---- seeded workload inputs (no CUDA library needed) ------------------ */
void ora_random_uniform(uint64_t seed, long n, double* out);
void ora_random_normal(uint64_t seed, long n, double* out);
void ora_kappa_field(uint64_t seed, int dim, const int* cells, double sigma, int truncation, double* kappa);
void ora_structured_boundary(int dim, int order, const int* cells, uint8_t* isBoundary);
int ora_assemble_structured(int dim, int order, int quadratureOrder, const int* cells, const int* dofmap,
                            const double* kappa, const int* rowptr, const int* col, double* val);

#ifdef __cplusplus
}
#endif
#endif
