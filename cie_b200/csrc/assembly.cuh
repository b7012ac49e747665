// Shared by the assembly kernels: the assembly plan, the 1-D rules and bases,
// the integrand conventions and the finite-cell geometry.
#pragma once

#include "ciecu_assembly.h"
#include "spmv.cuh"

#include <vector>

struct ciecu_assembly_s {
    ciecu_csr_s* csr = nullptr;
    int dim = 0, order = 0, nb = 0, nq = 0;
    long ncells = 0;
    const int* d_dofmap = nullptr;
    int* d_cellOrder = nullptr;       // cells sorted by colour
    std::vector<long> colorOffsets;   // host
    int* d_slots = nullptr;           // ncells * nb * nb CSR entry indices
    double* d_gtab = nullptr;         // nq * dim * nb parametric gradients
    double* d_wq = nullptr;           // nq weights
    int q1 = 0;                       // 1-D quadrature points (nq = q1^dim)
    std::vector<double> gn, gw;       // 1-D Gauss-Legendre rule on [-1, 1]
};

namespace ciecu {

// Gauss-Legendre nodes and weights by Newton iteration on P_n from the
// Tricomi initial guess (the method of GaussLegendreQuadrature.cpp:82-175).
int gauss_legendre(int order, std::vector<double>& nodes, std::vector<double>& weights);

// Lagrange basis on equispaced nodes -1 + 2i/p and its derivative at x.
__host__ __device__ inline void lagrange(int p, double x, double* v, double* dv) {
    const int n = p + 1;
    double nodes[16];
    for (int i = 0; i < n; ++i) nodes[i] = -1.0 + 2.0 * i / p;
    for (int i = 0; i < n; ++i) {
        double value = 1.0, deriv = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double f = (x - nodes[j]) / (nodes[i] - nodes[j]);
            deriv = deriv * f + value / (nodes[i] - nodes[j]);
            value *= f;
        }
        v[i] = value;
        dv[i] = deriv;
    }
}

// Scale and per-axis factors of the two stiffness conventions:
//   reference (0): scale = prod_d 2/h_d, f_d = 1
//   physical  (1): scale = prod_d h_d/2, f_d = (2/h_d)^2
inline void convention_factors(int dim, const double* h, int convention, double& scale, double f[3]) {
    scale = 1.0;
    for (int d = 0; d < 3; ++d) f[d] = 1.0;
    for (int d = 0; d < dim; ++d) {
        if (convention == 1) {
            scale *= 0.5 * h[d];
            f[d] = (2.0 / h[d]) * (2.0 / h[d]);
        } else {
            scale *= 2.0 / h[d];
        }
    }
}

// The standard-rule element matrix with kappa = 1, scale * sum_q w_q sum_d f_d
// G_q[d][a] G_q[d][b], into d_out (nb * nb doubles) on stream st.
int unit_element(const ciecu_assembly_s* P, double scale, const double f[3], double* d_out, cudaStream_t st);

// ---- finite-cell geometry -------------------------------------------------------

struct EmbeddedArgs {
    int dim, order, nb, q1, nq, maxDepth;
    int cells[3];
    double gn[16], gw[16];
    double origin[3], h[3], center[3];
    double radius2, alpha, scale;
    double f[3];
};

// Inside test of the sphere domain at the parametric point xi of a cell.
__device__ __forceinline__ bool embedded_inside(const EmbeddedArgs& P, const double* corg, const double* xi) {
    double r2 = 0.0;
    for (int d = 0; d < P.dim; ++d) {
        const double x = corg[d] + 0.5 * (xi[d] + 1.0) * P.h[d];
        r2 += (x - P.center[d]) * (x - P.center[d]);
    }
    return r2 < P.radius2;
}

// Parametric position and base weight of point q of a tree node (first index fastest).
__device__ __forceinline__ double embedded_point(const EmbeddedArgs& P, const double* base, double length, int q,
                                                 double* xi) {
    int rest = q;
    double w = 1.0;
    for (int d = 0; d < P.dim; ++d) {
        const int i = rest % P.q1;
        rest /= P.q1;
        xi[d] = base[d] + 0.5 * length * (P.gn[i] + 1.0);
        w *= P.gw[i];
    }
    return w;
}

}  // namespace ciecu
