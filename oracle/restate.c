/* ORACLE / TEST INFRASTRUCTURE ONLY -- see restate.h.
 *
 * Each function cites the kelofm/cie source it restates (paths relative to the
 * reference project root).  Compiled with -ffp-contract=off so that the
 * restatement evaluates every expression exactly as written.
 */
#include "restate.h"

#define ORA_PI 3.14159265358979323846

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

/* out = inScale*out + outScale*sum, with the reference's special cases for
 * scales in {-1, 0, 1}, including the (-1, -1) quirk that yields sum - out.
 * linalg/packages/solvers/src/CSROperator.cpp:78-110 */
static double combine(double inScale, double old, double outScale, double sum) {
    if (inScale == 1.0) {
        if (outScale == 1.0) return old + sum;
        if (outScale == -1.0) return old - sum;
        return old + outScale * sum;
    }
    if (inScale == 0.0) {
        if (outScale == 1.0) return sum;
        if (outScale == -1.0) return -sum;
        return outScale * sum;
    }
    if (inScale == -1.0) {
        if (outScale == 1.0 || outScale == -1.0) return sum - old;
        return outScale * sum - old;
    }
    if (outScale == 1.0) return inScale * old + sum;
    if (outScale == -1.0) return inScale * old - sum;
    return inScale * old + outScale * sum;
}

/* linalg/packages/solvers/src/CSROperator.cpp:46-58 (row loop), :78-110 (combine) */
void ora_spmv(int nrows, const int* rowptr, const int* col, const double* val,
              double inScale, const double* in, double outScale, double* out) {
    for (int i = 0; i < nrows; ++i) {
        double s = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s += val[k] * in[col[k]];
        out[i] = combine(inScale, out[i], outScale, s);
    }
}

/* linalg/packages/solvers/src/MaskedCSROperator.cpp:51-66: masked rows contribute 0
 * (CPU semantics), masked columns are skipped. */
void ora_masked_spmv(int nrows, const int* rowptr, const int* col, const double* val,
                     const uint16_t* mask, uint16_t threshold, double inScale,
                     const double* in, double outScale, double* out) {
    for (int i = 0; i < nrows; ++i) {
        double s = 0.0;
        if (mask[i] < threshold)
            for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
                if (mask[col[k]] < threshold) s += val[k] * in[col[k]];
        out[i] = combine(inScale, out[i], outScale, s);
    }
}

/* linalg/packages/solvers/src/DiagonalOperator.cpp:56-88.  Returns -1 on success,
 * else the first row with a missing or zero diagonal. */
int ora_diag_inverse(int n, const int* rowptr, const int* col, const double* val, double* dinv) {
    for (int i = 0; i < n; ++i) {
        int found = 0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (col[k] == i) {
                if (val[k] == 0.0) return i;
                dinv[i] = 1.0 / val[k];
                found = 1;
                break;
            }
        if (!found) return i;
    }
    return -1;
}

/* linalg/packages/solvers/src/DefaultSpace.cpp:71-76 (serial inner_product) */
double ora_dot(long n, const double* a, const double* b) {
    double s = 0.0;
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* cieutils/packages/maths/impl/Comparison_impl.hpp:32-63 with the default
 * tolerances (DBL_MIN, DBL_EPSILON). */
static int float_less(double a, double b) {
    double norm = fabs(a) + fabs(b);
    if (norm > DBL_MAX) norm = DBL_MAX;
    double tol = DBL_EPSILON * norm;
    if (tol < DBL_MIN) tol = DBL_MIN;
    const int equal = fabs(a - b) < tol;
    return a < b && !equal;
}

/* linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201, Jacobi
 * preconditioner from DiagonalOperator.cpp:37-53.  out (x) is the initial guess
 * and receives the solution (inScale 0, outScale 1).  stats = {iterations,
 * absolute residual, relative residual}.  Returns 0, or 1 (r^T z <= 0 at start),
 * 2 (p^T A p <= 0), 3 (missing/zero diagonal). */
int ora_pcg(int n, const int* rowptr, const int* col, const double* val, const double* b,
            double* x, long maxIterations, double absoluteTolerance, double relativeTolerance,
            int precondition, double* stats) {
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* q = (double*)calloc((size_t)n, sizeof(double));
    double* z = (double*)malloc(sizeof(double) * (size_t)n);
    double* dinv = (double*)malloc(sizeof(double) * (size_t)n);
    int status = 0;
    long it = 0;
    double absres = DBL_MAX, relres = DBL_MAX;
    if (precondition && ora_diag_inverse(n, rowptr, col, val, dinv) >= 0) {
        status = 3;
        goto done;
    }
    if (maxIterations > 0) {
        memcpy(r, b, sizeof(double) * (size_t)n);
        ora_spmv(n, rowptr, col, val, 1.0, x, -1.0, r); /* r = b - A x  (:86-88) */
        double rr = ora_dot(n, r, r);
        const double r0 = sqrt(rr);
        absres = r0;
        relres = 1.0;
        if (float_less(absres, absoluteTolerance) || float_less(relres, relativeTolerance)) goto done;
        double rz;
        if (precondition) {
            for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
            rz = ora_dot(n, r, z);
            memcpy(p, z, sizeof(double) * (size_t)n);
        } else {
            rz = rr;
            memcpy(p, r, sizeof(double) * (size_t)n);
        }
        if (!(0.0 < rz)) { status = 1; goto done; }
        for (; it < maxIterations; ++it) {
            ora_spmv(n, rowptr, col, val, 0.0, p, 1.0, q); /* :136 */
            const double pq = ora_dot(n, p, q);
            if (!(0.0 < pq)) { status = 2; goto done; }
            const double alpha = rz / pq;
            for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
            const double malpha = -alpha;
            for (int i = 0; i < n; ++i) r[i] = r[i] + malpha * q[i];
            rr = ora_dot(n, r, r);
            const double rzOld = rz;
            if (precondition) {
                for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
                rz = ora_dot(n, r, z);
            } else {
                rz = rr;
            }
            const double beta = rz / rzOld;
            const double* zz = precondition ? z : r;
            for (int i = 0; i < n; ++i) p[i] = p[i] * beta;
            for (int i = 0; i < n; ++i) p[i] = p[i] + zz[i];
            absres = sqrt(rr);
            relres = absres / r0;
            if (float_less(absres, absoluteTolerance) || float_less(relres, relativeTolerance)) break;
        }
    }
done:
    if (stats) {
        stats[0] = (double)it;
        stats[1] = absres;
        stats[2] = relres;
    }
    free(r); free(p); free(q); free(z); free(dinv);
    return status;
}

/* linalg/packages/solvers/src/JacobiOperator.cpp:36-62 with a DiagonalOperator
 * as inverse diagonal: starting from 0, x <- x + w * D^-1 (in - A x), then
 * out = inScale*out_old + outScale*x (scale(out,outScale); add(out,memory,inScale)). */
void ora_jacobi(int n, const int* rowptr, const int* col, const double* val, const double* dinv,
                long iterations, double relaxation, double inScale, const double* in,
                double outScale, double* out) {
    double* memory = (double*)malloc(sizeof(double) * (size_t)n);
    double* x = (double*)calloc((size_t)n, sizeof(double));
    double* res = (double*)malloc(sizeof(double) * (size_t)n);
    memcpy(memory, out, sizeof(double) * (size_t)n);
    for (long s = 0; s < iterations; ++s) {
        memcpy(res, in, sizeof(double) * (size_t)n);
        ora_spmv(n, rowptr, col, val, 1.0, x, -1.0, res); /* res = in - A x */
        for (int i = 0; i < n; ++i) {
            /* DiagonalOperator::product(1, res, w, x): buffer = res*dinv*w; x += buffer */
            const double t = relaxation == 1.0 ? res[i] * dinv[i]
                             : (relaxation == -1.0 ? -res[i] * dinv[i] : relaxation * res[i] * dinv[i]);
            x[i] = x[i] + t;
        }
    }
    for (int i = 0; i < n; ++i) {
        const double sx = x[i] * outScale;
        out[i] = inScale == 1.0 ? sx + memory[i]
               : (inScale == -1.0 ? sx - memory[i] : sx + inScale * memory[i]);
    }
    free(memory); free(x); free(res);
}

/* Chebyshev polynomial smoother for D^-1 A on [lambdaMin, lambdaMax], applied to
 * in from a zero initial guess (no reference counterpart).  Three-term recurrence
 * of Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., Alg. 12.1:
 *   theta = (lmax+lmin)/2, delta = (lmax-lmin)/2, sigma = theta/delta, rho_0 = 1/sigma
 *   d_0 = D^-1 r_0 / theta;  x_1 = d_0
 *   rho_k = 1/(2 sigma - rho_{k-1});  d_k = rho_k rho_{k-1} d_{k-1} + 2 rho_k/delta D^-1 r_k
 *   x_{k+1} = x_k + d_k,  r_{k+1} = r_k - A d_k. */
void ora_chebyshev(int n, const int* rowptr, const int* col, const double* val,
                   const double* dinv, int degree, double lambdaMin, double lambdaMax,
                   const double* in, double* out) {
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* d = (double*)malloc(sizeof(double) * (size_t)n);
    double* ad = (double*)malloc(sizeof(double) * (size_t)n);
    const double theta = 0.5 * (lambdaMax + lambdaMin);
    const double delta = 0.5 * (lambdaMax - lambdaMin);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    memcpy(r, in, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        d[i] = dinv[i] * r[i] / theta;
        out[i] = 0.0;
    }
    for (int k = 0; k < degree; ++k) {
        for (int i = 0; i < n; ++i) out[i] += d[i];
        if (k + 1 == degree) break;
        ora_spmv(n, rowptr, col, val, 0.0, d, 1.0, ad);
        for (int i = 0; i < n; ++i) r[i] -= ad[i];
        const double rhoNew = 1.0 / (2.0 * sigma - rho);
        for (int i = 0; i < n; ++i) d[i] = rhoNew * rho * d[i] + 2.0 * rhoNew / delta * dinv[i] * r[i];
        rho = rhoNew;
    }
    free(r); free(d); free(ad);
}

static uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Largest eigenvalue of D^-1 A by power iteration (Chebyshev bounds). */
double ora_power_lambda_max(int n, const int* rowptr, const int* col, const double* val,
                            const double* dinv, int iterations, uint64_t seed) {
    double* v = (double*)malloc(sizeof(double) * (size_t)n);
    double* w = (double*)malloc(sizeof(double) * (size_t)n);
    uint64_t s = seed;
    for (int i = 0; i < n; ++i) v[i] = (double)(splitmix(&s) >> 11) * 0x1.0p-53 + 0.5;
    double lambda = 0.0;
    for (int it = 0; it < iterations; ++it) {
        double nv = sqrt(ora_dot(n, v, v));
        for (int i = 0; i < n; ++i) v[i] /= nv;
        ora_spmv(n, rowptr, col, val, 0.0, v, 1.0, w);
        for (int i = 0; i < n; ++i) w[i] *= dinv[i];
        lambda = ora_dot(n, v, w);
        memcpy(v, w, sizeof(double) * (size_t)n);
    }
    free(v); free(w);
    return lambda;
}

/* ---- fem ------------------------------------------------------------- */

/* Legendre P_n(x) by the three-term recurrence (std::legendre in the reference). */
static double legendre(int n, double x) {
    if (n == 0) return 1.0;
    double p0 = 1.0, p1 = x;
    for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

/* fem/packages/numeric/src/GaussLegendreQuadrature.cpp:82-175: Newton iteration on
 * P_n from the initial guess (1 - (1/8 - 1/(8n))/n^2) cos(pi (4i-1)/(4n+2)), i = n-index,
 * convergence when |P_n| is "equal" to 0 under Comparison(256 eps, 256 eps);
 * weight = 2 / P_n'^2 / (1 - x^2); nodes ascending, mirrored. */
int ora_gauss_legendre(int order, double* nodes, double* weights) {
    if (order < 1) return 1;
    const double tol = 256.0 * DBL_EPSILON;
    int pivot;
    if (order % 2 == 1 && order > 1) {
        pivot = order / 2 + 1;
        nodes[pivot] = 0.0;
        double w = order * legendre(order - 1, 0.0);
        weights[pivot] = 2.0 / w / w;
        --pivot;
    } else {
        pivot = order / 2;
    }
    for (int index = 0; index <= pivot && index < order; ++index) {
        const int i = order - index;
        double node = (1.0 - (0.125 - 0.125 / order) / ((double)order * order)) *
                      cos(ORA_PI * (4.0 * i - 1.0) / (4.0 * order + 2.0));
        double omx2 = 1.0 - node * node;
        double value = 0.0, deriv = 0.0;
        int converged = 0;
        for (int k = 0; k < 50; ++k) {
            value = legendre(order, node);
            deriv = order * (-node * value + legendre(order - 1, node)) / omx2;
            /* Comparison::equal(|value|, 0) */
            double t = tol * fabs(value);
            if (t < tol) t = tol;
            if (fabs(value) < t) { converged = 1; break; }
            node -= value / deriv;
            omx2 = 1.0 - node * node;
        }
        if (!converged) return 2;
        const double w = 2.0 / deriv / deriv / omx2;
        nodes[index] = node;
        weights[index] = w;
        nodes[order - index - 1] = -node;
        weights[order - index - 1] = w;
    }
    return 0;
}

/* Lagrange basis on the given nodes in product form and its derivative
 * (fem/packages/maths/src/LagrangePolynomial.cpp:18-72 builds the same
 * polynomials as coefficient vectors). */
void ora_lagrange_1d(int count, const double* nodes, double x, double* values, double* derivatives) {
    for (int i = 0; i < count; ++i) {
        double v = 1.0;
        for (int j = 0; j < count; ++j)
            if (j != i) v *= (x - nodes[j]) / (nodes[i] - nodes[j]);
        double d = 0.0;
        for (int k = 0; k < count; ++k) {
            if (k == i) continue;
            double t = 1.0 / (nodes[i] - nodes[k]);
            for (int j = 0; j < count; ++j)
                if (j != i && j != k) t *= (x - nodes[j]) / (nodes[i] - nodes[j]);
            d += t;
        }
        values[i] = v;
        derivatives[i] = d;
    }
}

/* Horner evaluation of a polynomial with ascending coefficients and of its
 * derivative (fem/packages/maths/impl/Polynomial_impl.hpp:83-105). */
static void horner(const double* c, int degree, double x, double* value, double* deriv) {
    double v = c[degree], d = 0.0;
    for (int k = degree - 1; k >= 0; --k) {
        d = d * x + v;
        v = v * x + c[k];
    }
    *value = v;
    *deriv = d;
}

/* Parametric gradient matrix G (dim x setSize^dim, row-major) of the tensor-product
 * basis, first 1-D index fastest (fem/packages/maths/impl/AnsatzSpace_impl.hpp:231-328). */
static void tensor_gradients(int dim, int setSize, const double* values /*dim x setSize*/,
                             const double* derivs /*dim x setSize*/, double* G) {
    int nb = 1;
    for (int d = 0; d < dim; ++d) nb *= setSize;
    for (int dd = 0; dd < dim; ++dd)
        for (int a = 0; a < nb; ++a) {
            int rest = a;
            double g = 1.0;
            for (int d = 0; d < dim; ++d) {
                const int i = rest % setSize;
                rest /= setSize;
                g *= (d == dd) ? derivs[d * setSize + i] : values[d * setSize + i];
            }
            G[dd * nb + a] = g;
        }
}

/* LinearIsotropicStiffnessIntegrand::evaluate at one point:
 * out = modulus * G^T G (fem/packages/integrands/impl/LinearIsotropicStiffnessIntegrand_impl.hpp:62-75)
 * with a 1-D basis given as ascending monomial coefficients. */
void ora_stiffness_point(int dim, int setSize, const double* coefficients, int degree,
                         const double* point, double modulus, double* out) {
    double values[3 * 16], derivs[3 * 16];
    int nb = 1;
    for (int d = 0; d < dim; ++d) nb *= setSize;
    for (int d = 0; d < dim; ++d)
        for (int i = 0; i < setSize; ++i)
            horner(coefficients + i * (degree + 1), degree, point[d], &values[d * setSize + i],
                   &derivs[d * setSize + i]);
    double* G = (double*)malloc(sizeof(double) * (size_t)(dim * nb));
    tensor_gradients(dim, setSize, values, derivs, G);
    for (int a = 0; a < nb; ++a)
        for (int b = 0; b < nb; ++b) {
            double s = 0.0;
            for (int d = 0; d < dim; ++d) s += G[d * nb + a] * G[d * nb + b];
            out[a * nb + b] = modulus * s;
        }
    free(G);
}

/* Element stiffness for a Lagrange basis of the given order on equispaced nodes
 * -1 + 2i/order, integrated over the supplied parametric points (nq x dim) and
 * weights:
 *  convention 0 (reference): K = kappa * prod_d(2/h_d) * sum_q w_q G_q^T G_q
 *     (TransformedIntegrand.hpp:73-83 scales by |det| of the passed inverse
 *      Jacobian; QuadraturePoint.hpp:84-90 multiplies by the weight)
 *  convention 1 (physical): K = kappa * prod_d(h_d/2) * sum_q w_q (J^-T G)^T (J^-T G). */
void ora_element_stiffness(int dim, int order, int nq, const double* points,
                           const double* weights, double kappa, const double* h, int convention,
                           double* K) {
    const int setSize = order + 1;
    int nb = 1;
    for (int d = 0; d < dim; ++d) nb *= setSize;
    double nodes[16];
    for (int i = 0; i < setSize; ++i) nodes[i] = -1.0 + 2.0 * i / order;
    double values[3 * 16], derivs[3 * 16];
    double* G = (double*)malloc(sizeof(double) * (size_t)(dim * nb));
    memset(K, 0, sizeof(double) * (size_t)(nb * nb));
    for (int q = 0; q < nq; ++q) {
        for (int d = 0; d < dim; ++d)
            ora_lagrange_1d(setSize, nodes, points[q * dim + d], &values[d * setSize], &derivs[d * setSize]);
        tensor_gradients(dim, setSize, values, derivs, G);
        if (convention == 1)
            for (int d = 0; d < dim; ++d)
                for (int a = 0; a < nb; ++a) G[d * nb + a] *= 2.0 / h[d];
        for (int a = 0; a < nb; ++a)
            for (int b = 0; b < nb; ++b) {
                double s = 0.0;
                for (int d = 0; d < dim; ++d) s += G[d * nb + a] * G[d * nb + b];
                K[a * nb + b] += weights[q] * s;
            }
    }
    double scale = kappa;
    for (int d = 0; d < dim; ++d) scale *= convention == 1 ? 0.5 * h[d] : 2.0 / h[d];
    for (int k = 0; k < nb * nb; ++k) K[k] *= scale;
    free(G);
}

/* DoF map of a structured grid of cells[0] x cells[1] (x cells[2]) elements of the
 * given order: nodes numbered lexicographically (x fastest), local basis index
 * a = i0 + (p+1) i1 + (p+1)^2 i2 (first index fastest). */
void ora_structured_dofmap(int dim, int order, const int* cells, int* dofmap) {
    const int setSize = order + 1;
    int nb = 1, ncells = 1;
    int nodesPerAxis[3] = {1, 1, 1}, c[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) {
        nb *= setSize;
        ncells *= cells[d];
        nodesPerAxis[d] = order * cells[d] + 1;
        c[d] = cells[d];
    }
    for (int e = 0; e < ncells; ++e) {
        const int ex = e % c[0], ey = (e / c[0]) % c[1], ez = e / (c[0] * c[1]);
        for (int a = 0; a < nb; ++a) {
            const int i0 = a % setSize, i1 = (a / setSize) % setSize, i2 = a / (setSize * setSize);
            int g = order * ex + i0;
            if (dim >= 2) g += nodesPerAxis[0] * (order * ey + i1);
            if (dim >= 3) g += nodesPerAxis[0] * nodesPerAxis[1] * (order * ez + i2);
            dofmap[(long)e * nb + a] = g;
        }
    }
}

static int cmp_int(const void* a, const void* b) {
    const int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* Sparsity pattern = per row, the sorted unique union of the DoFs of every cell
 * that contains the row's DoF (fem/packages/graph/src/Assembler.cpp:55-175).
 * Returns nnz; fills rowptr/col when col is non-NULL (rowptr must then hold the
 * counts from a first call with col == NULL ... simplest: always recomputes). */
long ora_csr_pattern(long ncells, int nb, const int* dofmap, int ndofs, int* rowptr, int* col) {
    /* bucket (row, col) pairs per row */
    long* count = (long*)calloc((size_t)ndofs + 1, sizeof(long));
    for (long e = 0; e < ncells; ++e)
        for (int a = 0; a < nb; ++a) count[dofmap[e * nb + a] + 1] += nb;
    for (int i = 0; i < ndofs; ++i) count[i + 1] += count[i];
    int* buf = (int*)malloc(sizeof(int) * (size_t)count[ndofs]);
    long* fill = (long*)malloc(sizeof(long) * (size_t)ndofs);
    for (int i = 0; i < ndofs; ++i) fill[i] = count[i];
    for (long e = 0; e < ncells; ++e)
        for (int a = 0; a < nb; ++a) {
            const int row = dofmap[e * nb + a];
            for (int b = 0; b < nb; ++b) buf[fill[row]++] = dofmap[e * nb + b];
        }
    long nnz = 0;
    if (rowptr) rowptr[0] = 0;
    for (int i = 0; i < ndofs; ++i) {
        int* seg = buf + count[i];
        const long len = count[i + 1] - count[i];
        qsort(seg, (size_t)len, sizeof(int), cmp_int);
        long u = 0;
        for (long k = 0; k < len; ++k)
            if (k == 0 || seg[k] != seg[k - 1]) {
                if (col) col[nnz + u] = seg[k];
                ++u;
            }
        nnz += u;
        if (rowptr) rowptr[i + 1] = (int)nnz;
    }
    free(count); free(buf); free(fill);
    return nnz;
}

/* Assembler::addContribution (fem/packages/graph/impl/Assembler_impl.hpp:156-194):
 * for every local (i, j), lower_bound the global column inside the global row and
 * add K_e[i*nb + j].  Returns 0, or 1 when an entry is missing from the pattern. */
int ora_assemble(long ncells, int nb, const int* dofmap, const double* Ke, const int* rowptr,
                 const int* col, double* val) {
    for (long e = 0; e < ncells; ++e) {
        const int* dofs = dofmap + e * nb;
        const double* K = Ke + e * (long)nb * nb;
        for (int i = 0; i < nb; ++i) {
            const int row = dofs[i];
            for (int j = 0; j < nb; ++j) {
                int lo = rowptr[row], hi = rowptr[row + 1];
                const int target = dofs[j];
                while (lo < hi) {
                    const int mid = lo + (hi - lo) / 2;
                    if (col[mid] < target) lo = mid + 1; else hi = mid;
                }
                if (lo == rowptr[row + 1] || col[lo] != target) return 1;
                val[lo] += K[i * nb + j];
            }
        }
    }
    return 0;
}

/* Per-element adjoint gradient dJ/dkappa_e = -lambda_e^T (dK_e/dkappa_e) u_e with
 * K_e linear in kappa_e, i.e. -lambda_e^T K_e(kappa=1) u_e. */
void ora_element_gradient(long ncells, int nb, const int* dofmap, const double* Kunit,
                          const double* lambda, const double* u, double* grad) {
    for (long e = 0; e < ncells; ++e) {
        const int* dofs = dofmap + e * nb;
        double s = 0.0;
        for (int i = 0; i < nb; ++i) {
            double t = 0.0;
            for (int j = 0; j < nb; ++j) t += Kunit[i * nb + j] * u[dofs[j]];
            s += lambda[dofs[i]] * t;
        }
        grad[e] = -s;
    }
}

/* Symmetric elimination of homogeneous Dirichlet DoFs (fem/test/test_1d.cpp:291-313):
 * boundary rows and columns zeroed (structural zeros kept), diagonal 1, rhs 0. */
void ora_dirichlet_eliminate(int n, const int* rowptr, const int* col, double* val,
                             const uint8_t* isBoundary, double* rhs) {
    for (int i = 0; i < n; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k)
            if (isBoundary[i] || isBoundary[col[k]]) val[k] = (i == col[k]) ? 1.0 : 0.0;
    if (rhs)
        for (int i = 0; i < n; ++i)
            if (isBoundary[i]) rhs[i] = 0.0;
}

/* Cut-cell quadrature of fem/packages/numeric/inc/KDTreeQuadraturePointFactory.hpp:67-173
 * for a domain given by an inside test of physical points, depth range [0, depth],
 * a (order)^dim Gauss-Legendre base rule per tree node.  Keep rule (:156-160):
 * keep = (homogeneous && inside) || depth == max || (depth == min && homogeneous);
 * descend while not homogeneous.  points: parametric coordinates in [-1,1]^dim,
 * weights scaled by the node's Jacobian determinant (length/2)^dim, scales:
 * 1 inside, alpha outside (ScaledMultiMaterialIntegrand_impl.hpp:33-60 with the
 * material map {(0, alpha), (1, 1)}).  Returns the number of points, or -1 when
 * maxPoints is exceeded. */
typedef struct {
    int kind;               /* 0: sphere |x - c|^2 < r^2;  1: half-space n . x < offset */
    double center[3], radius;
    double normal[3], offset;
} cut_domain;

static int cut_inside(const cut_domain* D, int dim, const double* x) {
    double acc = 0.0;
    if (D->kind == 0) {
        for (int d = 0; d < dim; ++d) acc += (x[d] - D->center[d]) * (x[d] - D->center[d]);
        return acc < D->radius * D->radius;
    }
    for (int d = 0; d < dim; ++d) acc += D->normal[d] * x[d];
    return acc < D->offset;
}

static int cut_visit(int dim, int depth, int maxDepth, const double* base, double length,
                     int order, const double* gn, const double* gw, const cut_domain* D,
                     const double* cellOrigin, const double* cellSize,
                     int maxPoints, int count, double* points, double* weights, double* scales,
                     double alpha) {
    int nbase = 1;
    for (int d = 0; d < dim; ++d) nbase *= order;
    if (count + nbase > maxPoints) return -1;
    int inside0 = -1, homogeneous = 1;
    const double jac = pow(0.5 * length, dim);
    for (int q = 0; q < nbase; ++q) {
        int rest = q;
        double w = 1.0, x[3];
        for (int d = 0; d < dim; ++d) {
            const int i = rest % order;
            rest /= order;
            const double xi = base[d] + 0.5 * length * (gn[i] + 1.0);
            points[(long)(count + q) * dim + d] = xi;
            w *= gw[i];
            x[d] = cellOrigin[d] + 0.5 * (xi + 1.0) * cellSize[d];
        }
        weights[count + q] = w * jac;
        const int inside = cut_inside(D, dim, x);
        scales[count + q] = inside ? 1.0 : alpha;
        if (inside0 < 0) inside0 = inside;
        else if (inside != inside0) homogeneous = 0;
    }
    int keep = homogeneous && inside0;
    keep |= depth == maxDepth;
    keep |= depth == 0 && homogeneous;
    if (keep) count += nbase;
    if (homogeneous || depth == maxDepth) return count;
    const double half = 0.5 * length;
    const int children = 1 << dim;
    for (int c = 0; c < children; ++c) {
        double childBase[3];
        for (int d = 0; d < dim; ++d) childBase[d] = base[d] + ((c >> d) & 1) * half;
        count = cut_visit(dim, depth + 1, maxDepth, childBase, half, order, gn, gw, D,
                          cellOrigin, cellSize, maxPoints, count, points, weights, scales, alpha);
        if (count < 0) return -1;
    }
    return count;
}

static int cut_points(int dim, int depth, int order, const cut_domain* D, const double* cellOrigin,
                      const double* cellSize, int maxPoints, double* points, double* weights,
                      double* scales, double alpha) {
    double gn[16], gw[16];
    if (order < 1 || order > 16 || ora_gauss_legendre(order, gn, gw)) return -1;
    const double base[3] = {-1.0, -1.0, -1.0};
    return cut_visit(dim, 0, depth, base, 2.0, order, gn, gw, D, cellOrigin, cellSize,
                     maxPoints, 0, points, weights, scales, alpha);
}

int ora_cut_cell_points(int dim, int depth, int order, const double* center, double radius,
                        const double* cellOrigin, const double* cellSize, int maxPoints,
                        double* points, double* weights, double* scales, double alpha) {
    cut_domain D;
    memset(&D, 0, sizeof(D));
    for (int d = 0; d < dim; ++d) D.center[d] = center[d];
    D.radius = radius;
    return cut_points(dim, depth, order, &D, cellOrigin, cellSize, maxPoints, points, weights, scales, alpha);
}

int ora_cut_cell_points_halfspace(int dim, int depth, int order, const double* normal, double offset,
                                  const double* cellOrigin, const double* cellSize, int maxPoints,
                                  double* points, double* weights, double* scales, double alpha) {
    cut_domain D;
    memset(&D, 0, sizeof(D));
    D.kind = 1;
    for (int d = 0; d < dim; ++d) D.normal[d] = normal[d];
    D.offset = offset;
    return cut_points(dim, depth, order, &D, cellOrigin, cellSize, maxPoints, points, weights, scales, alpha);
}

/* ---- seeded workload inputs ------------------------------------------------
 * The benchmark and parity systems are built from seeded host arrays.  These
 * functions regenerate them without the CUDA library, so that the reference's CPU
 * solver can run on exactly the system the GPU solves.  They restate published
 * algorithms (64-bit Mersenne Twister, Box-Muller) and the workload definition
 * (uniform ((x >> 11) 2^-53) 2 - 1; kappa = exp of a smoothed, standardised
 * Gaussian field), not reference code. */

/* MT19937-64 (Matsumoto and Nishimura, ACM TOMACS 1998; Nishimura 2000), the
 * engine of std::mt19937_64: state of 312 words, default seeding
 * x_i = 6364136223846793005 (x_{i-1} ^ (x_{i-1} >> 62)) + i. */
typedef struct {
    uint64_t mt[312];
    int index;
} ora_mt64;

static void mt64_seed(ora_mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->index = 312;
}

static uint64_t mt64_next(ora_mt64* g) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    const uint64_t matrixA = 0xB5026F5AA96619E9ULL;
    if (g->index >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t y = (g->mt[i] & upper) | (g->mt[(i + 1) % 312] & lower);
            g->mt[i] = g->mt[(i + 156) % 312] ^ (y >> 1) ^ ((y & 1ULL) ? matrixA : 0ULL);
        }
        g->index = 0;
    }
    uint64_t x = g->mt[g->index++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

void ora_random_uniform(uint64_t seed, long n, double* out) {
    ora_mt64 g;
    mt64_seed(&g, seed);
    for (long i = 0; i < n; ++i) out[i] = (double)(mt64_next(&g) >> 11) * 0x1.0p-53 * 2.0 - 1.0;
}

void ora_random_normal(uint64_t seed, long n, double* out) {
    ora_mt64 g;
    mt64_seed(&g, seed);
    const double twoPi = 6.283185307179586476925286766559;
    for (long i = 0; i < n; i += 2) {
        const double u1 = (double)(mt64_next(&g) >> 11) * 0x1.0p-53;
        const double u2 = (double)(mt64_next(&g) >> 11) * 0x1.0p-53;
        const double rad = sqrt(-2.0 * log(1.0 - u1));
        out[i] = rad * cos(twoPi * u2);
        if (i + 1 < n) out[i + 1] = rad * sin(twoPi * u2);
    }
}

/* kappa_e = exp(g_e): N(0,1) per cell, convolved axis by axis (x first) with the
 * normalised kernel exp(-j^2 / (2 sigma^2)), |j| <= truncation, indices clamped at
 * the grid boundary, then standardised by the sample mean and variance. */
void ora_kappa_field(uint64_t seed, int dim, const int* cells, double sigma, int truncation, double* kappa) {
    long c[3] = {1, 1, 1}, n = 1;
    for (int d = 0; d < dim; ++d) {
        c[d] = cells[d];
        n *= cells[d];
    }
    double* g = (double*)malloc(sizeof(double) * (size_t)n);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
    double* w = (double*)malloc(sizeof(double) * (size_t)(2 * truncation + 1));
    ora_random_normal(seed, n, g);
    double wsum = 0.0;
    for (int j = -truncation; j <= truncation; ++j) {
        w[j + truncation] = exp(-0.5 * j * j / (sigma * sigma));
        wsum += w[j + truncation];
    }
    for (int j = 0; j < 2 * truncation + 1; ++j) w[j] /= wsum;
    const long stride[3] = {1, c[0], c[0] * c[1]};
    for (int d = 0; d < dim; ++d) {
        for (long e = 0; e < n; ++e) {
            const long coord = (e / stride[d]) % c[d];
            double s = 0.0;
            for (int j = -truncation; j <= truncation; ++j) {
                long k = coord + j;
                k = k < 0 ? 0 : (k >= c[d] ? c[d] - 1 : k);
                s += w[j + truncation] * g[e + (k - coord) * stride[d]];
            }
            tmp[e] = s;
        }
        double* t = g;
        g = tmp;
        tmp = t;
    }
    double mean = 0.0;
    for (long e = 0; e < n; ++e) mean += g[e];
    mean /= (double)n;
    double var = 0.0;
    for (long e = 0; e < n; ++e) var += (g[e] - mean) * (g[e] - mean);
    var /= (double)n;
    const double inv = var > 0.0 ? 1.0 / sqrt(var) : 1.0;
    for (long e = 0; e < n; ++e) kappa[e] = exp((g[e] - mean) * inv);
    free(g); free(tmp); free(w);
}

/* 1 for the nodes of a structured Q_order grid that lie on the box boundary. */
void ora_structured_boundary(int dim, int order, const int* cells, uint8_t* isBoundary) {
    long nodes[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) nodes[d] = (long)order * cells[d] + 1;
    const long n = nodes[0] * nodes[1] * nodes[2];
    for (long i = 0; i < n; ++i) {
        const long ix = i % nodes[0], iy = (i / nodes[0]) % nodes[1], iz = i / (nodes[0] * nodes[1]);
        int b = ix == 0 || ix == nodes[0] - 1;
        if (dim >= 2) b = b || iy == 0 || iy == nodes[1] - 1;
        if (dim >= 3) b = b || iz == 0 || iz == nodes[2] - 1;
        isBoundary[i] = (uint8_t)b;
    }
}

/* Element stiffness of a uniform grid scattered colour by colour (colour of a
 * cell = parity of its coordinates, so no two cells of a colour share a node),
 * with the summation order the GPU kernel uses, so that the two matrices can be
 * compared bit for bit:
 *   S[a][b] = sum_q w_q (sum_d G_q[d][a] G_q[d][b])   (fused multiply-adds, q and d ascending)
 *   val[slot] = fma(kappa_e * prod_d(2/h_d), S[a][b], val[slot])   (reference convention)
 * with the Gauss-Legendre rule of ora_gauss_legendre and Lagrange values and
 * derivatives on equispaced nodes by the running product
 *   f = (x - x_j)/(x_i - x_j);  dv = dv f + v/(x_i - x_j);  v = v f.
 * Returns 0, or 1 when an entry is missing from the pattern. */
int ora_assemble_structured(int dim, int order, int quadratureOrder, const int* cells, const int* dofmap,
                            const double* kappa, const int* rowptr, const int* col, double* val) {
    const int n1 = order + 1;
    int nb = 1, nq = 1;
    long ncells = 1, c[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) {
        nb *= n1;
        nq *= quadratureOrder;
        ncells *= cells[d];
        c[d] = cells[d];
    }
    double gn[16], gw[16], nodes[16], v1[16 * 16], d1[16 * 16];
    if (quadratureOrder < 1 || quadratureOrder > 16 || n1 > 16 || ora_gauss_legendre(quadratureOrder, gn, gw)) return 1;
    for (int i = 0; i < n1; ++i) nodes[i] = -1.0 + 2.0 * i / order;
    for (int q = 0; q < quadratureOrder; ++q)
        for (int i = 0; i < n1; ++i) {
            double value = 1.0, deriv = 0.0;
            for (int j = 0; j < n1; ++j) {
                if (j == i) continue;
                const double f = (gn[q] - nodes[j]) / (nodes[i] - nodes[j]);
                deriv = deriv * f + value / (nodes[i] - nodes[j]);
                value *= f;
            }
            v1[q * n1 + i] = value;
            d1[q * n1 + i] = deriv;
        }
    double* gtab = (double*)malloc(sizeof(double) * (size_t)nq * dim * nb);
    double* wq = (double*)malloc(sizeof(double) * (size_t)nq);
    double* S = (double*)malloc(sizeof(double) * (size_t)nb * nb);
    for (int q = 0; q < nq; ++q) {
        int qi[3] = {0, 0, 0}, rest = q;
        double w = 1.0;
        for (int d = 0; d < dim; ++d) {
            qi[d] = rest % quadratureOrder;
            rest /= quadratureOrder;
            w *= gw[qi[d]];
        }
        wq[q] = w;
        for (int dd = 0; dd < dim; ++dd)
            for (int a = 0; a < nb; ++a) {
                int ra = a;
                double g = 1.0;
                for (int d = 0; d < dim; ++d) {
                    const int i = ra % n1;
                    ra /= n1;
                    g *= (d == dd) ? d1[qi[d] * n1 + i] : v1[qi[d] * n1 + i];
                }
                gtab[((long)q * dim + dd) * nb + a] = g;
            }
    }
    for (int a = 0; a < nb; ++a)
        for (int b = 0; b < nb; ++b) {
            double s = 0.0;
            for (int q = 0; q < nq; ++q) {
                const double* g = gtab + (long)q * dim * nb;
                double gg = 0.0;
                for (int d = 0; d < dim; ++d) gg = fma(g[d * nb + a], g[d * nb + b], gg);
                s = fma(wq[q], gg, s);
            }
            S[a * nb + b] = s;
        }
    double scale = 1.0;
    for (int d = 0; d < dim; ++d) scale *= 2.0 / (1.0 / (double)cells[d]);
    int missing = 0;
    const int colors = 1 << dim;
    for (int color = 0; color < colors && !missing; ++color)
        for (long e = 0; e < ncells && !missing; ++e) {
            const long ex = e % c[0], ey = (e / c[0]) % c[1], ez = e / (c[0] * c[1]);
            if ((int)((ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2)) != color) continue;
            const int* dofs = dofmap + e * nb;
            const double ks = kappa[e] * scale;
            for (int a = 0; a < nb && !missing; ++a) {
                const int row = dofs[a];
                for (int b = 0; b < nb; ++b) {
                    int lo = rowptr[row], hi = rowptr[row + 1];
                    const int target = dofs[b];
                    while (lo < hi) {
                        const int mid = lo + (hi - lo) / 2;
                        if (col[mid] < target) lo = mid + 1; else hi = mid;
                    }
                    if (lo == rowptr[row + 1] || col[lo] != target) { missing = 1; break; }
                    val[lo] = fma(ks, S[a * nb + b], val[lo]);
                }
            }
        }
    free(gtab); free(wq); free(S);
    return missing;
}

/* ---- graph ------------------------------------------------------------------ */

/* Cuthill-McKee ordering of linalg/packages/utilities/src/reorder.cpp:23-173,
 * sequentially: start at the least-degree row (lowest index among equals), visit
 * rows in FIFO order, queue each visited row's unqueued neighbours in column
 * order and then order that batch by degree with a stable sort (insertion), and
 * restart at the least-degree unqueued row when the queue is empty; reverse for
 * RCM (strategy 2).  map[k] = the row placed at k.  Returns the largest batch
 * queued at once (the reference's std::sort keeps the column order of equal
 * degrees only for batches of at most 16 rows), or -1 on a bad column. */
int ora_cuthill_mckee(int n, const int* rowptr, const int* col, int strategy, int* map) {
    if (n <= 0) return 0;
    int* degree = (int*)malloc(sizeof(int) * (size_t)n);
    char* queued = (char*)calloc((size_t)n, 1);
    int* queue = (int*)malloc(sizeof(int) * (size_t)n);
    int head = 0, tail = 0, placed = 0, largest = 0;
    for (int i = 0; i < n; ++i) degree[i] = rowptr[i + 1] - rowptr[i];
    while (placed < n) {
        if (head == tail) {
            int best = -1;
            for (int i = 0; i < n; ++i)
                if (!queued[i] && (best < 0 || degree[i] < degree[best])) best = i;
            queue[tail++] = best;
            queued[best] = 1;
        }
        const int u = queue[head++];
        const int batch = tail;
        for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) {
            const int v = col[e];
            if (v < 0 || v >= n) { free(degree); free(queued); free(queue); return -1; }
            if (!queued[v]) {
                queued[v] = 1;
                /* stable insertion by degree into the batch */
                int pos = tail;
                while (pos > batch && degree[queue[pos - 1]] > degree[v]) {
                    queue[pos] = queue[pos - 1];
                    --pos;
                }
                queue[pos] = v;
                ++tail;
            }
        }
        if (tail - batch > largest) largest = tail - batch;
        map[placed++] = u;
    }
    if (strategy == 2)
        for (int i = 0; i < n / 2; ++i) {
            const int t = map[i];
            map[i] = map[n - 1 - i];
            map[n - 1 - i] = t;
        }
    free(degree); free(queued); free(queue);
    return largest;
}

/* Weak Dirichlet condition by penalty on the faces of the box of a structured
 * Q_order grid: DirichletPenaltyIntegrand::evaluate
 * (fem/packages/integrands/impl/DirichletPenaltyIntegrand_impl.hpp:38-88) -- at a
 * boundary point, LHS = N penalty N^T and RHS = penalty u_d N -- times the
 * weight and the embedding Jacobian |J| = prod over the tangential axes of h/2
 * (TransformedIntegrand.hpp:73-83), summed over the tensor Gauss points of every
 * selected face (faceMask bit 2d: x_d = 0, bit 2d+1: x_d = max; 0 = all) and
 * scattered like Assembler::addContribution (constraints.cpp:306-380).
 * u_d = sum_b N_b g_b from nodal values g (NULL: no RHS).  Returns 0, or 1 when
 * an entry is missing from the pattern. */
int ora_dirichlet_penalty(int dim, int order, int quadratureOrder, const int* cells, const double* h,
                          double penalty, int faceMask, const double* g, const int* dofmap, const int* rowptr,
                          const int* col, double* val, double* rhs) {
    const int n1 = order + 1;
    int nb = 1;
    long c[3] = {1, 1, 1}, ncells = 1;
    for (int d = 0; d < dim; ++d) {
        nb *= n1;
        c[d] = cells[d];
        ncells *= cells[d];
    }
    double gn[16], gw[16], nodes[16];
    if (ora_gauss_legendre(quadratureOrder, gn, gw)) return 1;
    for (int i = 0; i < n1; ++i) nodes[i] = -1.0 + 2.0 * i / order;
    if (faceMask == 0) faceMask = (1 << (2 * dim)) - 1;
    int nqf = 1;
    for (int d = 1; d < dim; ++d) nqf *= quadratureOrder;
    double* N = (double*)malloc(sizeof(double) * (size_t)nb);
    for (int side = 0; side < 2 * dim; ++side) {
        if (!((faceMask >> side) & 1)) continue;
        const int dn = side / 2, hi = side % 2;
        double jac = 1.0;
        for (int d = 0; d < dim; ++d)
            if (d != dn) jac *= 0.5 * h[d];
        for (long e = 0; e < ncells; ++e) {
            const long co[3] = {e % c[0], (e / c[0]) % c[1], e / (c[0] * c[1])};
            if (co[dn] != (hi ? c[dn] - 1 : 0)) continue;
            const int* dofs = dofmap + e * nb;
            for (int q = 0; q < nqf; ++q) {
                double xi[3] = {0.0, 0.0, 0.0}, w = 1.0;
                int rest = q;
                for (int d = 0; d < dim; ++d) {
                    if (d == dn) continue;
                    const int i = rest % quadratureOrder;
                    rest /= quadratureOrder;
                    xi[d] = gn[i];
                    w *= gw[i];
                }
                xi[dn] = hi ? 1.0 : -1.0;
                double vals[3][16], ders[3][16];
                for (int d = 0; d < dim; ++d) ora_lagrange_1d(n1, nodes, xi[d], vals[d], ders[d]);
                for (int a = 0; a < nb; ++a) {
                    int ra = a;
                    double prod = 1.0;
                    for (int d = 0; d < dim; ++d) {
                        prod *= vals[d][ra % n1];
                        ra /= n1;
                    }
                    N[a] = prod;
                }
                const double s = w * jac * penalty;
                for (int a = 0; a < nb; ++a) {
                    const int row = dofs[a];
                    for (int b = 0; b < nb; ++b) {
                        int lo = rowptr[row], hiE = rowptr[row + 1];
                        while (lo < hiE) {
                            const int mid = lo + (hiE - lo) / 2;
                            if (col[mid] < dofs[b]) lo = mid + 1; else hiE = mid;
                        }
                        if (lo == rowptr[row + 1] || col[lo] != dofs[b]) { free(N); return 1; }
                        val[lo] += s * N[a] * N[b];
                    }
                }
                if (g && rhs) {
                    double ud = 0.0;
                    for (int b = 0; b < nb; ++b) ud += N[b] * g[dofs[b]];
                    for (int a = 0; a < nb; ++a) rhs[dofs[a]] += s * ud * N[a];
                }
            }
        }
    }
    free(N);
    return 0;
}
