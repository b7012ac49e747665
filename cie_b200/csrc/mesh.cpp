// Host-side set-up of the assembly path (no GPU needed):
//  * DoF maps of structured Q_p grids (lexicographic nodes, x fastest; local basis
//    index with the first 1-D index fastest, like AnsatzSpace_impl.hpp:599-657),
//  * the CSR sparsity pattern of a DoF map = Assembler::makeCSRMatrix
//    (fem/packages/graph/src/Assembler.cpp:55-175): per row the sorted, unique
//    union of the DoFs of every cell that contains the row's DoF,
//  * element colouring for the atomic-free scatter,
//  * the seeded synthetic inputs: std::mt19937_64 uniforms mapped to [-1, 1] by
//    ((x >> 11) * 2^-53) * 2 - 1, Box-Muller normals, and kappa = exp(g) with g a
//    unit-variance Gaussian field smoothed by a separable Gaussian kernel.
#include "ciecu.h"
#include "ciecu_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace ciecu {
void set_error(const std::string& message);
int fail(int status, const std::string& message);
}  // namespace ciecu

namespace {

template <typename F>
void parallel_rows(long n, F&& f) {
    unsigned threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 4096) threads = 1;
    std::vector<std::thread> pool;
    const long chunk = (n + threads - 1) / threads;
    for (unsigned t = 0; t < threads; ++t) {
        const long a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        pool.emplace_back([a, b, &f] { f(a, b); });
    }
    for (auto& th : pool) th.join();
}

double uniform_pm1(std::mt19937_64& g) { return static_cast<double>(g() >> 11) * 0x1.0p-53 * 2.0 - 1.0; }
double uniform_01(std::mt19937_64& g) { return static_cast<double>(g() >> 11) * 0x1.0p-53; }

}  // namespace

extern "C" {

int ciecu_structured_dofmap(int dim, int order, const int32_t* cells, int32_t* h_dofmap, int32_t* h_ndofs) {
    if (dim < 1 || dim > 3 || order < 1 || order > 8 || !cells || !h_dofmap)
        return ciecu::fail(CIECU_ERR_ARGUMENT, "structured_dofmap: invalid arguments");
    const int setSize = order + 1;
    long nb = 1, ncells = 1;
    long nodes[3] = {1, 1, 1}, c[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) {
        if (cells[d] < 1) return ciecu::fail(CIECU_ERR_ARGUMENT, "structured_dofmap: empty grid");
        nb *= setSize;
        ncells *= cells[d];
        nodes[d] = static_cast<long>(order) * cells[d] + 1;
        c[d] = cells[d];
    }
    const long ndofs = nodes[0] * nodes[1] * nodes[2];
    if (ndofs >= (1L << 31)) return ciecu::fail(CIECU_ERR_ARGUMENT, "structured_dofmap: more than 2^31 DoFs");
    parallel_rows(ncells, [&](long e0, long e1) {
        for (long e = e0; e < e1; ++e) {
            const long ex = e % c[0], ey = (e / c[0]) % c[1], ez = e / (c[0] * c[1]);
            for (long a = 0; a < nb; ++a) {
                const long i0 = a % setSize, i1 = (a / setSize) % setSize, i2 = a / (setSize * setSize);
                long g = order * ex + i0;
                if (dim >= 2) g += nodes[0] * (order * ey + i1);
                if (dim >= 3) g += nodes[0] * nodes[1] * (order * ez + i2);
                h_dofmap[e * nb + a] = static_cast<int32_t>(g);
            }
        }
    });
    if (h_ndofs) *h_ndofs = static_cast<int32_t>(ndofs);
    return CIECU_OK;
}

int ciecu_structured_boundary(int dim, int order, const int32_t* cells, uint8_t* h_isBoundary) {
    if (dim < 1 || dim > 3 || order < 1 || !cells || !h_isBoundary)
        return ciecu::fail(CIECU_ERR_ARGUMENT, "structured_boundary: invalid arguments");
    long nodes[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) nodes[d] = static_cast<long>(order) * cells[d] + 1;
    const long n = nodes[0] * nodes[1] * nodes[2];
    parallel_rows(n, [&](long a, long b) {
        for (long i = a; i < b; ++i) {
            const long ix = i % nodes[0], iy = (i / nodes[0]) % nodes[1], iz = i / (nodes[0] * nodes[1]);
            bool bnd = ix == 0 || ix == nodes[0] - 1;
            if (dim >= 2) bnd = bnd || iy == 0 || iy == nodes[1] - 1;
            if (dim >= 3) bnd = bnd || iz == 0 || iz == nodes[2] - 1;
            h_isBoundary[i] = bnd ? 1 : 0;
        }
    });
    return CIECU_OK;
}

int ciecu_csr_pattern(int64_t ncells, int nb, const int32_t* h_dofmap, int32_t ndofs, int32_t* h_rowExtents,
                      int32_t* h_columnIndices, int64_t* h_nnz) {
    if (ncells < 0 || nb < 1 || ndofs < 0 || (ncells > 0 && !h_dofmap) || !h_rowExtents)
        return ciecu::fail(CIECU_ERR_ARGUMENT, "csr_pattern: invalid arguments");
    // node -> cells (counting sort)
    std::vector<int64_t> start(static_cast<size_t>(ndofs) + 1, 0);
    for (int64_t k = 0; k < ncells * nb; ++k) {
        const int32_t d = h_dofmap[k];
        if (d < 0 || d >= ndofs) return ciecu::fail(CIECU_ERR_ARGUMENT, "csr_pattern: DoF index out of range");
        ++start[static_cast<size_t>(d) + 1];
    }
    for (int32_t i = 0; i < ndofs; ++i) start[i + 1] += start[i];
    std::vector<int64_t> cellsOf(static_cast<size_t>(start[ndofs]));
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int64_t e = 0; e < ncells; ++e)
            for (int a = 0; a < nb; ++a) cellsOf[fill[h_dofmap[e * nb + a]]++] = e;
    }
    std::vector<int32_t> counts(static_cast<size_t>(ndofs));
    auto rowUnion = [&](int32_t i, std::vector<int32_t>& buf) {
        buf.clear();
        for (int64_t k = start[i]; k < start[i + 1]; ++k) {
            const int64_t e = cellsOf[k];
            buf.insert(buf.end(), h_dofmap + e * nb, h_dofmap + (e + 1) * nb);
        }
        std::sort(buf.begin(), buf.end());
        buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    };
    parallel_rows(ndofs, [&](long a, long b) {
        std::vector<int32_t> buf;
        for (long i = a; i < b; ++i) {
            rowUnion(static_cast<int32_t>(i), buf);
            counts[i] = static_cast<int32_t>(buf.size());
        }
    });
    int64_t nnz = 0;
    h_rowExtents[0] = 0;
    for (int32_t i = 0; i < ndofs; ++i) {
        nnz += counts[i];
        if (nnz >= (1LL << 31)) return ciecu::fail(CIECU_ERR_ARGUMENT, "csr_pattern: more than 2^31-1 entries");
        h_rowExtents[i + 1] = static_cast<int32_t>(nnz);
    }
    if (h_nnz) *h_nnz = nnz;
    if (h_columnIndices) {
        parallel_rows(ndofs, [&](long a, long b) {
            std::vector<int32_t> buf;
            for (long i = a; i < b; ++i) {
                rowUnion(static_cast<int32_t>(i), buf);
                std::memcpy(h_columnIndices + h_rowExtents[i], buf.data(), sizeof(int32_t) * buf.size());
            }
        });
    }
    return CIECU_OK;
}

int ciecu_structured_colors(int dim, const int32_t* cells, int32_t* h_color) {
    if (dim < 1 || dim > 3 || !cells || !h_color) return ciecu::fail(CIECU_ERR_ARGUMENT, "structured_colors: invalid arguments");
    long c[3] = {1, 1, 1}, ncells = 1;
    for (int d = 0; d < dim; ++d) {
        c[d] = cells[d];
        ncells *= cells[d];
    }
    for (long e = 0; e < ncells; ++e) {
        const long ex = e % c[0], ey = (e / c[0]) % c[1], ez = e / (c[0] * c[1]);
        h_color[e] = static_cast<int32_t>((ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2));
    }
    return CIECU_OK;
}

int ciecu_greedy_colors(int64_t ncells, int nb, const int32_t* h_dofmap, int32_t ndofs, int32_t* h_color,
                        int32_t* h_colorCount) {
    if (ncells < 0 || nb < 1 || !h_color) return ciecu::fail(CIECU_ERR_ARGUMENT, "greedy_colors: invalid arguments");
    // Smallest colour not used by any earlier cell sharing a DoF with this one.
    std::vector<uint64_t> used(static_cast<size_t>(ndofs), 0);
    int32_t colors = 0;
    for (int64_t e = 0; e < ncells; ++e) {
        uint64_t taken = 0;
        for (int a = 0; a < nb; ++a) taken |= used[h_dofmap[e * nb + a]];
        int c = 0;
        while (c < 64 && (taken >> c) & 1u) ++c;
        if (c == 64) return ciecu::fail(CIECU_ERR_ARGUMENT, "greedy_colors: more than 64 colours needed");
        h_color[e] = c;
        colors = std::max(colors, c + 1);
        for (int a = 0; a < nb; ++a) used[h_dofmap[e * nb + a]] |= (1ull << c);
    }
    if (h_colorCount) *h_colorCount = colors;
    return CIECU_OK;
}

int ciecu_random_uniform(uint64_t seed, int64_t n, double* h_out) {
    if (n < 0 || (n > 0 && !h_out)) return ciecu::fail(CIECU_ERR_ARGUMENT, "random_uniform: invalid arguments");
    std::mt19937_64 g(seed);
    for (int64_t i = 0; i < n; ++i) h_out[i] = uniform_pm1(g);
    return CIECU_OK;
}

int ciecu_random_normal(uint64_t seed, int64_t n, double* h_out) {
    if (n < 0 || (n > 0 && !h_out)) return ciecu::fail(CIECU_ERR_ARGUMENT, "random_normal: invalid arguments");
    std::mt19937_64 g(seed);
    const double twoPi = 6.283185307179586476925286766559;
    for (int64_t i = 0; i < n; i += 2) {
        const double u1 = uniform_01(g), u2 = uniform_01(g);
        const double rad = std::sqrt(-2.0 * std::log(1.0 - u1));
        h_out[i] = rad * std::cos(twoPi * u2);
        if (i + 1 < n) h_out[i + 1] = rad * std::sin(twoPi * u2);
    }
    return CIECU_OK;
}

int ciecu_kappa_field(uint64_t seed, int dim, const int32_t* cells, double sigma, int truncation, double* h_kappa) {
    if (dim < 1 || dim > 3 || !cells || !h_kappa || sigma <= 0.0 || truncation < 0)
        return ciecu::fail(CIECU_ERR_ARGUMENT, "kappa_field: invalid arguments");
    long c[3] = {1, 1, 1};
    long n = 1;
    for (int d = 0; d < dim; ++d) {
        c[d] = cells[d];
        n *= cells[d];
    }
    std::vector<double> g(static_cast<size_t>(n)), tmp(static_cast<size_t>(n));
    ciecu_random_normal(seed, n, g.data());
    std::vector<double> w(static_cast<size_t>(2 * truncation + 1));
    double wsum = 0.0;
    for (int j = -truncation; j <= truncation; ++j) {
        w[j + truncation] = std::exp(-0.5 * j * j / (sigma * sigma));
        wsum += w[j + truncation];
    }
    for (double& v : w) v /= wsum;
    const long stride[3] = {1, c[0], c[0] * c[1]};
    for (int d = 0; d < dim; ++d) {
        parallel_rows(n, [&](long a, long b) {
            for (long e = a; e < b; ++e) {
                const long coord = (e / stride[d]) % c[d];
                double s = 0.0;
                for (int j = -truncation; j <= truncation; ++j) {
                    long k = coord + j;
                    k = k < 0 ? 0 : (k >= c[d] ? c[d] - 1 : k);  // clamp at the boundary
                    s += w[j + truncation] * g[e + (k - coord) * stride[d]];
                }
                tmp[e] = s;
            }
        });
        g.swap(tmp);
    }
    double mean = 0.0;
    for (double v : g) mean += v;
    mean /= static_cast<double>(n);
    double var = 0.0;
    for (double v : g) var += (v - mean) * (v - mean);
    var /= static_cast<double>(n);
    const double inv = var > 0.0 ? 1.0 / std::sqrt(var) : 1.0;
    for (long e = 0; e < n; ++e) h_kappa[e] = std::exp((g[e] - mean) * inv);
    return CIECU_OK;
}

}  // extern "C"
