/*
 * ciecu assembly: per-element stiffness integration and CSR scatter on the GPU,
 * the device counterpart of IntegrandProcessor (SYCLIntegrandProcessor,
 * fem/packages/utilities/inc/IntegrandProcessor.hpp:138-158) evaluating
 * TransformedIntegrand<LinearIsotropicStiffnessIntegrand> and of
 * Assembler::addContribution (fem/packages/graph/impl/Assembler_impl.hpp:156-194).
 */
#ifndef CIECU_ASSEMBLY_H
#define CIECU_ASSEMBLY_H

#include "ciecu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ciecu_assembly_s* ciecu_assembly;

/* Plan for repeated assembly into the pattern of `csr` (FP64 values): tensor
 * Lagrange Q_order cells on equispaced nodes, quadratureOrder^dim Gauss-Legendre
 * points (the reference uses order + 1, definitions.hpp:36), device DoF map
 * (ncells x (order+1)^dim, local index first-1-D-index fastest), host colours
 * (cells of one colour must share no DoF; NULL = one colour).  Builds the
 * element -> CSR-entry map once and fails with CIECU_ERR_PATTERN if an element
 * entry is missing from the pattern (CIE_OUT_OF_RANGE_CHECK of
 * Assembler_impl.hpp:178-180). */
int ciecu_assembly_create(ciecu_csr csr, int dim, int order, int quadratureOrder, int64_t ncells,
                          const int32_t* d_dofmap, const int32_t* h_color, ciecu_assembly* out);
int ciecu_assembly_destroy(ciecu_assembly plan);
int ciecu_assembly_color_count(ciecu_assembly plan, int* h_count);

/* d_entries (+)= sum_e K_e scattered into the CSR values, one launch per colour,
 * no atomics.  K_e = kappa_e * |det J^-1| * sum_q w_q G_q^T G_q with parametric
 * gradients (convention 0, the reference's TransformedIntegrand.hpp:73-83 with
 * the inverse Jacobian passed by integration.cpp:92-97) or the physical
 * kappa_e * det J * sum_q w_q (J^-T G_q)^T (J^-T G_q) (convention 1).
 * h_cellSize: dim edge lengths of the (uniform) cells.  accumulate = 0 zeroes
 * d_entries first. */
int ciecu_assemble_stiffness(ciecu_assembly plan, const double* d_kappa, const double* h_cellSize, int convention,
                             int accumulate, double* d_entries);

/* Embedded-domain (finite-cell) stiffness on a structured grid of h_cells cells of
 * size h_cellSize starting at h_origin (cell e at index (e % cells[0], ...), first
 * axis fastest): the physical domain is the sphere |x - h_center| < radius, the
 * rest is fictitious with material factor alpha
 * (ScaledMultiMaterialIntegrand_impl.hpp:33-60).  A cell whose base quadrature
 * points (the plan's quadratureOrder^dim Gauss rule) all lie on one side is
 * integrated with that rule; a cut cell with the tree of
 * KDTreeQuadraturePointFactory.hpp:67-173 over depths [0, maxDepth]: the base
 * rule on every tree node, weights times the node's Jacobian, nodes kept when
 * homogeneous and inside, at the maximum depth, or homogeneous at depth 0, and
 * refined while not homogeneous.  K_e in FP64, convention as
 * ciecu_assemble_stiffness; d_kappa may be NULL (kappa = 1).  The plan's basis has
 * at most 64 functions.  The cut cells' Gram contractions run on the tensor cores
 * in FP64 (eight CTAs per cut cell, one per depth-1 tree node); cells of one
 * colour are scattered together, so the result does not depend on the schedule.
 * d_work: nb*nb doubles (kept for the interface; the call allocates its own
 * work arrays).  h_cutCells (may be NULL): the number of cut cells.  The call
 * synchronises the stream. */
int ciecu_assemble_embedded(ciecu_assembly plan, const double* d_kappa, const double* h_cellSize,
                            const int32_t* h_cells, const double* h_origin, const double* h_center, double radius,
                            double alpha, int maxDepth, int convention, int accumulate, double* d_entries,
                            double* d_work, int64_t* h_cutCells);

/* The same finite-cell matrix in single precision, for inner or preconditioner
 * operators: d_entries32 (FP32 values in the plan's CSR pattern) (+)= the element
 * matrices with the Gram contraction B^T W B on the tensor cores in BF16 with
 * FP32 accumulation, each operand split into a high and a low BF16 part and the
 * three significant products summed (about 16 significant bits per product); the
 * regular cells add the FP64 standard-rule matrix rounded to FP32. */
int ciecu_assemble_embedded_f32(ciecu_assembly plan, const double* d_kappa, const double* h_cellSize,
                                const int32_t* h_cells, const double* h_origin, const double* h_center, double radius,
                                double alpha, int maxDepth, int convention, int accumulate, float* d_entries32,
                                int64_t* h_cutCells);

/* Adjoint gradient of J(u) with respect to the cell conductivities:
 * d_grad[e] = -lambda_e^T (dK_e/dkappa_e) u_e = -lambda_e^T K_e(kappa = 1) u_e.
 * d_work: nb*nb doubles. */
int ciecu_element_gradient(ciecu_assembly plan, const double* h_cellSize, int convention, const double* d_lambda,
                           const double* d_u, double* d_grad, double* d_work);

/* Adjoint sensitivities of an objective J(u) of u = A(kappa)^-1 P b, where
 * A(kappa) = sum_e kappa_e K_e with the DoFs flagged in d_isBoundary eliminated
 * symmetrically and P zeroes those DoFs (homogeneous Dirichlet).  The method of
 * the reference's 1-D adjoint model (fem/python/modules/fem/optcontrol/
 * adjointmodel.py:16-126, adjointelement.py:70-84), for the Q_p stiffness here:
 *     lambda        = A^-1 P dJ/du     (the transposed solve: A is symmetric, so
 *                                       the same PCG `solver`, started from 0)
 *     dJ/db         = lambda           (written to d_lambda)
 *     dJ/dkappa_e   = -(P lambda)_e^T K_e(kappa = 1) (P u)_e   (d_gradKappa)
 * d_isBoundary may be NULL (nothing eliminated).  solver and plan must use the
 * same space.  d_work: 2n + nb*nb doubles.  h_stats (may be NULL): statistics of
 * the adjoint solve. */
int ciecu_adjoint_gradient(ciecu_pcg solver, ciecu_assembly plan, const double* h_cellSize, int convention,
                           const uint8_t* d_isBoundary, const double* d_u, const double* d_dJdu, double* d_lambda,
                           double* d_gradKappa, double* d_work, ciecu_statistics* h_stats);

/* Weak Dirichlet condition by penalty on the faces of the box of a structured
 * grid: DirichletPenaltyIntegrand (fem/packages/integrands/impl/DirichletPenaltyIntegrand_impl.hpp:38-88)
 * integrated over boundary faces and scattered as in constraints.cpp:306-380.
 * On every boundary face selected by faceMask (bit 2d: the face x_d = 0 of the
 * box, bit 2d + 1: the face x_d = max; 0 selects all), at the tensor
 * Gauss-Legendre points of the face (quadratureOrder per tangential axis; 0 =
 * the plan's order):
 *     K_e += penalty |J| w_q N(xi_q) N(xi_q)^T
 *     f_e += penalty |J| w_q u_d(x_q) N(xi_q)
 * where N are the cell's Q_p basis functions at the face point's parametric
 * coordinates, |J| = prod over the face's tangential axes of h_t / 2 (the
 * embedding's Jacobian, TransformedIntegrand.hpp:73-83), and the prescribed value
 * u_d = sum_b N_b(xi) g_b interpolates nodal values g (d_boundaryValues, one per
 * DoF; NULL: u_d = 0, and d_rhs is untouched).  Faces of one side are scattered
 * by colour (parity of the tangential cell coordinates), sides one after another:
 * no atomics.  h_cells: the grid's cells per axis (cell e at (e % cells[0], ...)),
 * matching the plan's cell count. */
int ciecu_assemble_dirichlet_penalty(ciecu_assembly plan, const int32_t* h_cells, const double* h_cellSize,
                                     double penalty, int faceMask, int quadratureOrder,
                                     const double* d_boundaryValues, double* d_entries, double* d_rhs);

/* Symmetric elimination of homogeneous Dirichlet DoFs (fem/test/test_1d.cpp:291-313):
 * rows and columns of boundary DoFs zeroed (structural zeros kept), diagonal 1,
 * d_rhs[boundary] = 0 (d_rhs may be NULL). */
int ciecu_dirichlet_eliminate(ciecu_csr csr, const uint8_t* d_isBoundary, double* d_entries, double* d_rhs);
/* The same elimination on an FP32 copy of the values (d_entries32 in the pattern of csr). */
int ciecu_dirichlet_eliminate_f32(ciecu_csr csr, const uint8_t* d_isBoundary, float* d_entries32);

#ifdef __cplusplus
}
#endif
#endif /* CIECU_ASSEMBLY_H */
