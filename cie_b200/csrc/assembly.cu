// Per-element stiffness integration and CSR scatter:
//   IntegrandProcessor::process (fem/packages/utilities/impl/IntegrandProcessor_impl.hpp:171-494)
//   evaluating TransformedIntegrand<LinearIsotropicStiffnessIntegrand>
//   (integrands/impl/LinearIsotropicStiffnessIntegrand_impl.hpp:40-92,
//    integrands/inc/TransformedIntegrand.hpp:51-85) at tensor-product Gauss points
//   (numeric/src/GaussLegendreQuadrature.cpp:82-175), then
//   Assembler::addContribution (graph/impl/Assembler_impl.hpp:156-194).
//
// B200 design: the element -> CSR slot map (the reference's per-entry lower_bound)
// is computed once per pattern on the device; cells are sorted by colour so that
// one launch per colour scatters without atomics; the parametric gradient table
// G[q][d][a] is shared by every cell and sits in shared memory.
//
//   K_e[a][b] = scale_e * sum_q w_q sum_d f_d G[q][d][a] G[q][d][b]
//   reference convention (0): scale_e = kappa_e prod_d 2/h_d, f_d = 1
//   physical convention  (1): scale_e = kappa_e prod_d h_d/2, f_d = (2/h_d)^2
#include "assembly.cuh"
#include "space.cuh"

#include <cmath>
#include <string>
#include <vector>


namespace ciecu {

// Gauss-Legendre nodes and weights by Newton iteration on P_n from the
// Tricomi initial guess (the method of GaussLegendreQuadrature.cpp:82-175).
int gauss_legendre(int order, std::vector<double>& nodes, std::vector<double>& weights) {
    nodes.assign(order, 0.0);
    weights.assign(order, 0.0);
    const double pi = 3.14159265358979323846;
    auto legendre = [](int n, double x, double& pn, double& pn1) {
        double p0 = 1.0, p1 = x;
        if (n == 0) {
            pn = 1.0;
            pn1 = 0.0;
            return;
        }
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        pn = p1;
        pn1 = p0;
    };
    for (int i = 0; i < (order + 1) / 2; ++i) {
        double x = (1.0 - (0.125 - 0.125 / order) / (double(order) * order)) *
                   std::cos(pi * (4.0 * (order - i) - 1.0) / (4.0 * order + 2.0));
        double pn = 0, pn1 = 0, dp = 0;
        for (int it = 0; it < 100; ++it) {
            legendre(order, x, pn, pn1);
            dp = order * (pn1 - x * pn) / (1.0 - x * x);
            const double dx = pn / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        legendre(order, x, pn, pn1);
        dp = order * (pn1 - x * pn) / (1.0 - x * x);
        const double w = 2.0 / ((1.0 - x * x) * dp * dp);
        nodes[i] = x;
        weights[i] = w;
        nodes[order - 1 - i] = -x;
        weights[order - 1 - i] = w;
    }
    if (order % 2 == 1) nodes[order / 2] = 0.0;
    return CIECU_OK;
}

namespace {

constexpr int kT = 256;

// slot[e][a][b] = index of column dof[b] in row dof[a]; -1 if absent.
__global__ void slot_kernel(long ncells, int nb, const int* __restrict__ dofmap, int nrows,
                            const int* __restrict__ rowptr, const int* __restrict__ col, int* __restrict__ slots,
                            int* missing) {
    const long total = ncells * nb * nb;
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
        const long e = t / (nb * nb);
        const int ab = static_cast<int>(t - e * nb * nb);
        const int row = dofmap[e * nb + ab / nb];
        const int target = dofmap[e * nb + ab % nb];
        if (row < 0 || row >= nrows) {
            slots[t] = -1;
            atomicExch(missing, 1);
            continue;
        }
        int lo = rowptr[row], hi = rowptr[row + 1];
        const int end = hi;
        while (lo < hi) {
            const int mid = lo + ((hi - lo) >> 1);
            if (col[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        if (lo == end || col[lo] != target) {
            slots[t] = -1;
            atomicExch(missing, 1);
        } else {
            slots[t] = lo;
        }
    }
}

// One thread per (cell, a, b) of one colour: integrate and add into the CSR entry.
__global__ void stiffness_scatter_kernel(long count, int nb, int dim, int nq, const int* __restrict__ cellOrder,
                                         const double* __restrict__ gtab, const double* __restrict__ wq,
                                         const double* __restrict__ kappa, double scale, double f0, double f1,
                                         double f2, const int* __restrict__ slots, double* __restrict__ val) {
    extern __shared__ double s_tab[];
    const int tabSize = nq * dim * nb;
    for (int k = threadIdx.x; k < tabSize; k += blockDim.x) s_tab[k] = gtab[k];
    double* s_w = s_tab + tabSize;
    for (int k = threadIdx.x; k < nq; k += blockDim.x) s_w[k] = wq[k];
    __syncthreads();
    const int nb2 = nb * nb;
    const long total = count * nb2;
    const double f[3] = {f0, f1, f2};
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
        const long le = t / nb2;
        const int ab = static_cast<int>(t - le * nb2);
        const int a = ab / nb, b = ab - (ab / nb) * nb;
        const int e = cellOrder[le];
        double s = 0.0;
        for (int q = 0; q < nq; ++q) {
            const double* g = s_tab + q * dim * nb;
            double gg = 0.0;
            for (int d = 0; d < dim; ++d) gg = fma(f[d] * g[d * nb + a], g[d * nb + b], gg);
            s = fma(s_w[q], gg, s);
        }
        const int slot = slots[static_cast<long>(e) * nb2 + ab];
        // one rounding per contribution, written out so that the host restatement
        // of this summation order reproduces the matrix bit for bit
        val[slot] = fma(kappa[e] * scale, s, val[slot]);
    }
}

// Reference element matrix (kappa = 1) K1[a][b], computed once per call.
__global__ void unit_element_kernel(int nb, int dim, int nq, const double* __restrict__ gtab,
                                    const double* __restrict__ wq, double scale, double f0, double f1, double f2,
                                    double* __restrict__ K1) {
    const double f[3] = {f0, f1, f2};
    for (int ab = blockIdx.x * blockDim.x + threadIdx.x; ab < nb * nb; ab += gridDim.x * blockDim.x) {
        const int a = ab / nb, b = ab % nb;
        double s = 0.0;
        for (int q = 0; q < nq; ++q) {
            const double* g = gtab + q * dim * nb;
            double gg = 0.0;
            for (int d = 0; d < dim; ++d) gg = fma(f[d] * g[d * nb + a], g[d * nb + b], gg);
            s = fma(wq[q], gg, s);
        }
        K1[ab] = scale * s;
    }
}

// dJ/dkappa_e = -lambda_e^T K1 u_e: one warp per cell, K1 in shared memory.
__global__ void element_gradient_kernel(long ncells, int nb, const int* __restrict__ dofmap,
                                        const double* __restrict__ K1, const double* __restrict__ lambda,
                                        const double* __restrict__ u, double* __restrict__ grad) {
    extern __shared__ double s_K[];
    for (int k = threadIdx.x; k < nb * nb; k += blockDim.x) s_K[k] = K1[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long warp = (static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const long warps = (static_cast<long>(gridDim.x) * blockDim.x) >> 5;
    for (long e = warp; e < ncells; e += warps) {
        const int* dofs = dofmap + e * nb;
        double acc = 0.0;
        // lane handles rows a = lane, lane + 32, ...
        for (int a = lane; a < nb; a += 32) {
            double t = 0.0;
            for (int b = 0; b < nb; ++b) t = fma(s_K[a * nb + b], u[dofs[b]], t);
            acc = fma(lambda[dofs[a]], t, acc);
        }
        acc = warp_sum(acc);
        if (lane == 0) grad[e] = -acc;
    }
}

template <typename V>
__global__ void dirichlet_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                 V* __restrict__ val, const uint8_t* __restrict__ bnd, double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool bi = bnd[i] != 0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            const int j = col[k];
            if (bi || bnd[j]) val[k] = (i == j) ? V(1) : V(0);
        }
        if (rhs && bi) rhs[i] = 0.0;
    }
}

// out = v with the entries of eliminated (boundary) DoFs set to zero.
__global__ void interior_kernel(int n, const double* __restrict__ v, const uint8_t* __restrict__ bnd,
                                double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = bnd[i] ? 0.0 : v[i];
}

// ---- Dirichlet penalty on boundary faces -------------------------------------

// One thread per (face, a, b) with a and b on the face: the face mass term
// penalty |J| sum_q w_q N_q[a] N_q[b] added into the CSR entry.  `onFace` lists
// the local indices of the face's basis functions (the others vanish there).
__global__ void penalty_matrix_kernel(long faces, int nb, int nf, int nqf, const int* __restrict__ faceCells,
                                      const int* __restrict__ onFace, const double* __restrict__ table,
                                      const double* __restrict__ wq, double scale, const int* __restrict__ slots,
                                      double* __restrict__ val) {
    const long total = faces * nf * nf;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const long f = t / (nf * nf);
        const int ij = static_cast<int>(t - f * nf * nf);
        const int a = onFace[ij / nf], b = onFace[ij % nf];
        double s = 0.0;
        for (int q = 0; q < nqf; ++q) s = fma(wq[q] * table[q * nb + a], table[q * nb + b], s);
        const long e = faceCells[f];
        const int slot = slots[e * nb * nb + a * nb + b];
        val[slot] = fma(scale, s, val[slot]);
    }
}

// One thread per (face, a) with a on the face: penalty |J| sum_q w_q N_q[a] u_d(x_q),
// u_d(x_q) = sum_b N_q[b] g[dof_b], added into rhs[dof_a].
__global__ void penalty_rhs_kernel(long faces, int nb, int nf, int nqf, const int* __restrict__ faceCells,
                                   const int* __restrict__ onFace, const double* __restrict__ table,
                                   const double* __restrict__ wq, double scale, const int* __restrict__ dofmap,
                                   const double* __restrict__ g, double* __restrict__ rhs) {
    const long total = faces * nf;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const long f = t / nf;
        const int a = onFace[t - f * nf];
        const int* dofs = dofmap + static_cast<long>(faceCells[f]) * nb;
        double s = 0.0;
        for (int q = 0; q < nqf; ++q) {
            double ud = 0.0;
            for (int j = 0; j < nf; ++j) ud = fma(table[q * nb + onFace[j]], g[dofs[onFace[j]]], ud);
            s = fma(wq[q] * table[q * nb + a], ud, s);
        }
        rhs[dofs[a]] = fma(scale, s, rhs[dofs[a]]);
    }
}

}  // namespace

int unit_element(const ciecu_assembly_s* P, double scale, const double f[3], double* d_out, cudaStream_t st) {
    const int nb2 = P->nb * P->nb;
    unit_element_kernel<<<(nb2 + kT - 1) / kT, kT, 0, st>>>(P->nb, P->dim, P->nq, P->d_gtab, P->d_wq, scale, f[0],
                                                           f[1], f[2], d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("unit_element_kernel");
    return CIECU_OK;
}

}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_assembly_create(ciecu_csr csr, int dim, int order, int quadratureOrder, int64_t ncells,
                          const int32_t* d_dofmap, const int32_t* h_color, ciecu_assembly* out) {
    CIECU_REQUIRE(csr && out && d_dofmap, "assembly_create: null argument");
    CIECU_REQUIRE(dim >= 1 && dim <= 3 && order >= 1 && order <= 8, "assembly_create: dim in [1,3], order in [1,8]");
    CIECU_REQUIRE(quadratureOrder >= 1 && quadratureOrder <= 16, "assembly_create: quadrature order in [1,16]");
    CIECU_REQUIRE(ncells >= 0, "assembly_create: negative cell count");
    auto* P = new ciecu_assembly_s();
    P->csr = csr;
    P->dim = dim;
    P->order = order;
    P->ncells = ncells;
    P->d_dofmap = d_dofmap;
    int nb = 1, nq = 1;
    for (int d = 0; d < dim; ++d) {
        nb *= order + 1;
        nq *= quadratureOrder;
    }
    P->nb = nb;
    P->nq = nq;
    cudaStream_t st = csr->space->stream;
    // Gradient table G[q][d][a]: points first-index-fastest (OuterProduct_impl.hpp:27-45).
    std::vector<double> gn, gw;
    gauss_legendre(quadratureOrder, gn, gw);
    P->q1 = quadratureOrder;
    P->gn = gn;
    P->gw = gw;
    const int n1 = order + 1;
    std::vector<double> v1(static_cast<size_t>(quadratureOrder) * n1), d1(v1.size());
    for (int q = 0; q < quadratureOrder; ++q) lagrange(order, gn[q], &v1[q * n1], &d1[q * n1]);
    std::vector<double> gtab(static_cast<size_t>(nq) * dim * nb), wq(nq);
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
                gtab[(static_cast<size_t>(q) * dim + dd) * nb + a] = g;
            }
    }
    // Colour order (counting sort of cells by colour).
    std::vector<int> order_(static_cast<size_t>(ncells));
    {
        int colors = 0;
        for (long e = 0; e < ncells; ++e) colors = std::max(colors, h_color ? h_color[e] + 1 : 1);
        std::vector<long> count(static_cast<size_t>(colors) + 1, 0);
        for (long e = 0; e < ncells; ++e) ++count[(h_color ? h_color[e] : 0) + 1];
        for (int c = 0; c < colors; ++c) count[c + 1] += count[c];
        P->colorOffsets = count;
        std::vector<long> fill(count.begin(), count.end() - 1);
        for (long e = 0; e < ncells; ++e) order_[fill[h_color ? h_color[e] : 0]++] = static_cast<int>(e);
        if (!h_color) P->colorOffsets = {0, ncells};  // single colour: caller promises no sharing
    }
    cudaError_t e = cudaSuccess;
    const size_t slotCount = static_cast<size_t>(ncells) * nb * nb;
    e = cudaMalloc(&P->d_cellOrder, sizeof(int) * std::max<size_t>(1, order_.size()));
    if (e == cudaSuccess) e = cudaMalloc(&P->d_slots, sizeof(int) * std::max<size_t>(1, slotCount));
    if (e == cudaSuccess) e = cudaMalloc(&P->d_gtab, sizeof(double) * gtab.size());
    if (e == cudaSuccess) e = cudaMalloc(&P->d_wq, sizeof(double) * wq.size());
    if (e == cudaSuccess && ncells)
        e = cudaMemcpyAsync(P->d_cellOrder, order_.data(), sizeof(int) * order_.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->d_gtab, gtab.data(), sizeof(double) * gtab.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->d_wq, wq.data(), sizeof(double) * wq.size(), cudaMemcpyHostToDevice, st);
    int* d_missing = reinterpret_cast<int*>(csr->space->d_result);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_missing, 0, sizeof(int), st);
    if (e != cudaSuccess) {
        ciecu_assembly_destroy(P);
        return cuda_fail(e, "assembly_create");
    }
    if (slotCount) {
        slot_kernel<<<grid_for(static_cast<long>(slotCount), kT, 8), kT, 0, st>>>(ncells, nb, d_dofmap, csr->rows,
                                                                                  csr->rowptr, csr->col, P->d_slots,
                                                                                  d_missing);
        count_launch();
    }
    int missing = 0;
    e = cudaMemcpyAsync(&missing, d_missing, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ciecu_assembly_destroy(P);
        return cuda_fail(e, "assembly_create: slot map");
    }
    if (missing) {
        ciecu_assembly_destroy(P);
        return fail(CIECU_ERR_PATTERN, "assembly_create: an element entry is not part of the CSR pattern");
    }
    *out = P;
    return CIECU_OK;
}

int ciecu_assembly_destroy(ciecu_assembly P) {
    if (!P) return CIECU_OK;
    // No access to P->csr (it may already be gone); cudaFree synchronises the device.
    cudaFree(P->d_cellOrder);
    cudaFree(P->d_slots);
    cudaFree(P->d_gtab);
    cudaFree(P->d_wq);
    delete P;
    return CIECU_OK;
}

int ciecu_assembly_color_count(ciecu_assembly P, int* h_count) {
    CIECU_REQUIRE(P && h_count, "assembly_color_count: null argument");
    *h_count = static_cast<int>(P->colorOffsets.size()) - 1;
    return CIECU_OK;
}

int ciecu_assemble_stiffness(ciecu_assembly P, const double* d_kappa, const double* h_cellSize, int convention,
                             int accumulate, double* d_entries) {
    CIECU_REQUIRE(P && d_kappa && h_cellSize && d_entries, "assemble_stiffness: null argument");
    CIECU_REQUIRE(convention == 0 || convention == 1, "assemble_stiffness: convention must be 0 or 1");
    cudaStream_t st = P->csr->space->stream;
    if (!accumulate) CIECU_CUDA(cudaMemsetAsync(d_entries, 0, sizeof(double) * P->csr->nnz, st));
    double scale, f[3];
    convention_factors(P->dim, h_cellSize, convention, scale, f);
    const size_t smem = sizeof(double) * (static_cast<size_t>(P->nq) * P->dim * P->nb + P->nq);
    if (smem > 48 * 1024) {
        static bool attr = false;
        if (!attr) {
            CIECU_CUDA(cudaFuncSetAttribute(stiffness_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            200 * 1024));
            attr = true;
        }
    }
    const int nb2 = P->nb * P->nb;
    for (size_t c = 0; c + 1 < P->colorOffsets.size(); ++c) {
        const long begin = P->colorOffsets[c], count = P->colorOffsets[c + 1] - begin;
        if (count == 0) continue;
        stiffness_scatter_kernel<<<grid_for(count * nb2, kT, 8), kT, smem, st>>>(
            count, P->nb, P->dim, P->nq, P->d_cellOrder + begin, P->d_gtab, P->d_wq, d_kappa, scale, f[0], f[1], f[2],
            P->d_slots, d_entries);
        count_launch();
        CIECU_CHECK_LAUNCH("stiffness_scatter_kernel");
    }
    return CIECU_OK;
}

int ciecu_element_gradient(ciecu_assembly P, const double* h_cellSize, int convention, const double* d_lambda,
                           const double* d_u, double* d_grad, double* d_work) {
    CIECU_REQUIRE(P && h_cellSize && d_lambda && d_u && d_grad && d_work, "element_gradient: null argument");
    cudaStream_t st = P->csr->space->stream;
    double scale, f[3];
    convention_factors(P->dim, h_cellSize, convention, scale, f);
    const int nb2 = P->nb * P->nb;
    unit_element_kernel<<<(nb2 + kT - 1) / kT, kT, 0, st>>>(P->nb, P->dim, P->nq, P->d_gtab, P->d_wq, scale, f[0],
                                                           f[1], f[2], d_work);
    count_launch();
    if (P->ncells > 0) {
        const long warps = P->ncells;
        const long blocks = std::min<long>((warps * 32 + kT - 1) / kT, static_cast<long>(sm_count()) * 16);
        element_gradient_kernel<<<static_cast<int>(blocks), kT, sizeof(double) * nb2, st>>>(
            P->ncells, P->nb, P->d_dofmap, d_work, d_lambda, d_u, d_grad);
        count_launch();
    }
    CIECU_CHECK_LAUNCH("element_gradient_kernel");
    return CIECU_OK;
}

int ciecu_adjoint_gradient(ciecu_pcg solver, ciecu_assembly P, const double* h_cellSize, int convention,
                           const uint8_t* d_isBoundary, const double* d_u, const double* d_dJdu, double* d_lambda,
                           double* d_gradKappa, double* d_work, ciecu_statistics* h_stats) {
    CIECU_REQUIRE(solver && P && h_cellSize && d_u && d_dJdu && d_lambda && d_gradKappa && d_work,
                  "adjoint_gradient: null argument");
    const int n = P->csr->rows;
    cudaStream_t st = P->csr->space->stream;
    double* lamMasked = d_work;
    double* uMasked = d_work + n;
    double* unit = d_work + 2L * n;
    const double* rhs = d_dJdu;
    if (d_isBoundary && n > 0) {
        interior_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, d_dJdu, d_isBoundary, lamMasked);
        count_launch();
        CIECU_CHECK_LAUNCH("interior_kernel");
        rhs = lamMasked;
    }
    // adjoint solve from lambda = 0; A is symmetric, so A^T lambda = P dJ/du is the same PCG
    if (n > 0) CIECU_CUDA(cudaMemsetAsync(d_lambda, 0, sizeof(double) * n, st));
    CIECU_TRY(ciecu_pcg_product(solver, 0.0, rhs, 1.0, d_lambda, h_stats));
    const double* lam = d_lambda;
    const double* u = d_u;
    if (d_isBoundary && n > 0) {
        interior_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, d_lambda, d_isBoundary, lamMasked);
        interior_kernel<<<grid_for(n, kT, 8), kT, 0, st>>>(n, d_u, d_isBoundary, uMasked);
        count_launch(2);
        CIECU_CHECK_LAUNCH("interior_kernel");
        lam = lamMasked;
        u = uMasked;
    }
    return ciecu_element_gradient(P, h_cellSize, convention, lam, u, d_gradKappa, unit);
}

int ciecu_assemble_dirichlet_penalty(ciecu_assembly P, const int32_t* h_cells, const double* h_cellSize,
                                     double penalty, int faceMask, int quadratureOrder,
                                     const double* d_boundaryValues, double* d_entries, double* d_rhs) {
    CIECU_REQUIRE(P && h_cells && h_cellSize && d_entries, "assemble_dirichlet_penalty: null argument");
    CIECU_REQUIRE(quadratureOrder >= 0 && quadratureOrder <= 16, "assemble_dirichlet_penalty: quadrature order in [0, 16]");
    CIECU_REQUIRE(faceMask >= 0 && faceMask < (1 << (2 * P->dim)), "assemble_dirichlet_penalty: invalid face mask");
    CIECU_REQUIRE(!d_boundaryValues || d_rhs, "assemble_dirichlet_penalty: boundary values need a right-hand side");
    const int dim = P->dim, p = P->order, n1 = p + 1, nb = P->nb;
    long c[3] = {1, 1, 1}, total = 1;
    for (int d = 0; d < dim; ++d) {
        CIECU_REQUIRE(h_cells[d] >= 1, "assemble_dirichlet_penalty: empty grid");
        c[d] = h_cells[d];
        total *= h_cells[d];
    }
    CIECU_REQUIRE(total == P->ncells, "assemble_dirichlet_penalty: grid size differs from the plan's cell count");
    if (faceMask == 0) faceMask = (1 << (2 * dim)) - 1;
    const int q1 = quadratureOrder ? quadratureOrder : P->q1;
    std::vector<double> gn, gw;
    gauss_legendre(q1, gn, gw);
    int nqf = 1;
    for (int d = 1; d < dim; ++d) nqf *= q1;
    cudaStream_t st = P->csr->space->stream;
    // per side: face point basis table (nqf x nb), weights, on-face indices, and
    // the side's cells by colour
    struct Side {
        std::vector<double> table, wq;
        std::vector<int> onFace;
        std::vector<std::vector<int>> colors;
        double jac;
    };
    std::vector<Side> sides;
    size_t doubles = 0, ints = 0;
    for (int side = 0; side < 2 * dim; ++side) {
        if (!((faceMask >> side) & 1)) continue;
        const int dn = side / 2, hi = side % 2;
        Side S;
        S.jac = 1.0;
        int tang[2] = {0, 0}, nt = 0;
        for (int d = 0; d < dim; ++d)
            if (d != dn) {
                tang[nt++] = d;
                S.jac *= 0.5 * h_cellSize[d];
            }
        S.table.assign(static_cast<size_t>(nqf) * nb, 0.0);
        S.wq.assign(static_cast<size_t>(nqf), 1.0);
        std::vector<double> v(n1), dv(n1);
        for (int q = 0; q < nqf; ++q) {
            double xi[3] = {0.0, 0.0, 0.0};
            int rest = q;
            for (int t = 0; t < nt; ++t) {
                const int i = rest % q1;
                rest /= q1;
                xi[tang[t]] = gn[i];
                S.wq[q] *= gw[i];
            }
            xi[dn] = hi ? 1.0 : -1.0;
            double vals[3][16];
            for (int d = 0; d < dim; ++d) {
                lagrange(p, xi[d], v.data(), dv.data());
                for (int i = 0; i < n1; ++i) vals[d][i] = v[i];
            }
            for (int a = 0; a < nb; ++a) {
                int ra = a;
                double prod = 1.0;
                for (int d = 0; d < dim; ++d) {
                    prod *= vals[d][ra % n1];
                    ra /= n1;
                }
                S.table[static_cast<size_t>(q) * nb + a] = prod;
            }
        }
        for (int a = 0; a < nb; ++a) {
            int ra = a, id = 0;
            for (int d = 0; d <= dn; ++d) {
                id = ra % n1;
                ra /= n1;
            }
            if (id == (hi ? p : 0)) S.onFace.push_back(a);
        }
        const int ncol = 1 << (dim - 1);
        S.colors.assign(static_cast<size_t>(ncol), {});
        for (long e = 0; e < total; ++e) {
            const long co[3] = {e % c[0], (e / c[0]) % c[1], e / (c[0] * c[1])};
            if (co[dn] != (hi ? c[dn] - 1 : 0)) continue;
            int color = 0;
            for (int t = 0; t < nt; ++t) color |= static_cast<int>(co[tang[t]] & 1) << t;
            S.colors[static_cast<size_t>(color)].push_back(static_cast<int>(e));
        }
        doubles += S.table.size() + S.wq.size();
        ints += S.onFace.size();
        for (auto& l : S.colors) ints += l.size();
        sides.push_back(std::move(S));
    }
    if (sides.empty()) return CIECU_OK;
    // one device buffer for every side's tables and lists
    std::vector<double> hostDoubles;
    std::vector<int> hostInts;
    hostDoubles.reserve(doubles);
    hostInts.reserve(ints);
    for (auto& S : sides) {
        hostDoubles.insert(hostDoubles.end(), S.table.begin(), S.table.end());
        hostDoubles.insert(hostDoubles.end(), S.wq.begin(), S.wq.end());
        hostInts.insert(hostInts.end(), S.onFace.begin(), S.onFace.end());
        for (auto& l : S.colors) hostInts.insert(hostInts.end(), l.begin(), l.end());
    }
    void* buf = nullptr;
    const size_t bytes = sizeof(double) * hostDoubles.size() + sizeof(int) * std::max<size_t>(hostInts.size(), 1);
    CIECU_CUDA(cudaMalloc(&buf, bytes));
    double* dd = static_cast<double*>(buf);
    int* di = reinterpret_cast<int*>(dd + hostDoubles.size());
    cudaError_t e = cudaMemcpyAsync(dd, hostDoubles.data(), sizeof(double) * hostDoubles.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !hostInts.empty())
        e = cudaMemcpyAsync(di, hostInts.data(), sizeof(int) * hostInts.size(), cudaMemcpyHostToDevice, st);
    size_t od = 0, oi = 0;
    for (auto& S : sides) {
        if (e != cudaSuccess) break;
        const double* table = dd + od;
        const double* wq = table + S.table.size();
        const int* onFace = di + oi;
        od += S.table.size() + S.wq.size();
        oi += S.onFace.size();
        const int nf = static_cast<int>(S.onFace.size());
        const double scale = penalty * S.jac;
        for (auto& l : S.colors) {
            const int* faceCells = di + oi;
            oi += l.size();
            const long faces = static_cast<long>(l.size());
            if (faces == 0) continue;
            penalty_matrix_kernel<<<grid_for(faces * nf * nf, kT, 8), kT, 0, st>>>(
                faces, nb, nf, nqf, faceCells, onFace, table, wq, scale, P->d_slots, d_entries);
            count_launch();
            if (d_boundaryValues) {
                penalty_rhs_kernel<<<grid_for(faces * nf, kT, 8), kT, 0, st>>>(
                    faces, nb, nf, nqf, faceCells, onFace, table, wq, scale, P->d_dofmap, d_boundaryValues, d_rhs);
                count_launch();
            }
            e = cudaGetLastError();
            if (e != cudaSuccess) break;
        }
    }
    // the buffer is in use by the launches above: free after they finish
    const cudaError_t s2 = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(e, "assemble_dirichlet_penalty");
    if (s2 != cudaSuccess) return cuda_fail(s2, "assemble_dirichlet_penalty");
    return CIECU_OK;
}

int ciecu_dirichlet_eliminate(ciecu_csr csr, const uint8_t* d_isBoundary, double* d_entries, double* d_rhs) {
    CIECU_REQUIRE(csr && d_isBoundary && d_entries, "dirichlet_eliminate: null argument");
    CIECU_REQUIRE(csr->rows == csr->cols, "dirichlet_eliminate: square matrix expected");
    if (csr->rows == 0) return CIECU_OK;
    dirichlet_kernel<double><<<grid_for(csr->rows, kT, 8), kT, 0, csr->space->stream>>>(
        csr->rows, csr->rowptr, csr->col, d_entries, d_isBoundary, d_rhs);
    count_launch();
    CIECU_CHECK_LAUNCH("dirichlet_kernel");
    return CIECU_OK;
}

int ciecu_dirichlet_eliminate_f32(ciecu_csr csr, const uint8_t* d_isBoundary, float* d_entries32) {
    CIECU_REQUIRE(csr && d_isBoundary && d_entries32, "dirichlet_eliminate_f32: null argument");
    CIECU_REQUIRE(csr->rows == csr->cols, "dirichlet_eliminate_f32: square matrix expected");
    if (csr->rows == 0) return CIECU_OK;
    dirichlet_kernel<float><<<grid_for(csr->rows, kT, 8), kT, 0, csr->space->stream>>>(
        csr->rows, csr->rowptr, csr->col, d_entries32, d_isBoundary, nullptr);
    count_launch();
    CIECU_CHECK_LAUNCH("dirichlet_kernel");
    return CIECU_OK;
}

}  // extern "C"
