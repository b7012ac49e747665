// Finite-cell stiffness: the cut-cell quadrature of KDTreeQuadraturePointFactory
// (fem/packages/numeric/inc/KDTreeQuadraturePointFactory.hpp:67-173) with the
// material scaling of ScaledMultiMaterialIntegrand (integrands/impl/
// ScaledMultiMaterialIntegrand_impl.hpp:33-60) and the stiffness integrand
// (LinearIsotropicStiffnessIntegrand_impl.hpp:62-75), load-balanced and with the
// element contraction on tensor cores.
//
// The element matrix of a cut cell is a Gram matrix over its kept quadrature
// points: K = sum_{p,d} w_p s_p f_d G_p[d] G_p[d]^T = B^T W B, B of (points x dim)
// rows and nb <= 64 columns.  It is computed in three passes:
//   1. classify every cell by its base points (one warp per cell); a prefix sum
//      numbers the cut cells in cell order;
//   2. one CTA per (cut cell, depth-1 tree node) walks that node's subtree with
//      the keep / refine rules, stages the basis gradients of 16 kept points at a
//      time in shared memory and accumulates B^T W B with warp-level tensor-core
//      MMAs into a partial element matrix -- eight CTAs per cut cell instead of
//      one, so no SM waits for a few cut cells of a colour;
//   3. per colour (cells of a colour share no DoF), every cell adds its matrix
//      into the CSR values: regular cells s K1 (s = 1 inside, alpha outside, K1
//      the standard-rule matrix), cut cells the sum of their partials in node
//      order.  The result does not depend on the schedule.
//
// Two contractions:
//   FP64 (the solver's matrix): mma.sync m8n8k4 f64 (DMMA) -- FP64 products and
//     sums, the same accuracy as the scalar FP64 loop (parity 1e-12 with the
//     restatement);
//   FP32 (a single-precision copy for inner / preconditioner operators):
//     mma.sync m16n8k16 bf16 with FP32 accumulation, each operand split into a
//     high and a low bf16 part and the three significant products summed
//     (hi*hi + hi*lo + lo*hi): about 16 significant bits per product, FP32 sums.
#include "assembly.cuh"
#include "sortscan.cuh"
#include "space.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <string>
#include <type_traits>

namespace ciecu {
namespace {

constexpr int kFcWarps = 8;
constexpr int kFcThreads = 32 * kFcWarps;
constexpr int kFcPoints = 16;               // kept points staged per chunk
constexpr int kFcRows = 3 * kFcPoints;      // rows (point, axis) of B per chunk
constexpr int kFcStride = 72;               // doubles per staged row: 64 columns + 8 (spreads the banks)
constexpr int kFcStack = 64;

// One warp per cell: number of the cell's base points inside the domain.
// cut[e] = 1 for a cell with points on both sides; side[e] = 1 for a cell fully
// inside.
__global__ void fc_classify_kernel(EmbeddedArgs P, long ncells, int* __restrict__ cut, signed char* __restrict__ side) {
    const int lane = threadIdx.x & 31;
    const long warps = static_cast<long>(gridDim.x) * (blockDim.x >> 5);
    for (long e = static_cast<long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); e < ncells; e += warps) {
        double corg[3] = {0.0, 0.0, 0.0};
        long rest = e;
        for (int d = 0; d < P.dim; ++d) {
            corg[d] = P.origin[d] + static_cast<double>(rest % P.cells[d]) * P.h[d];
            rest /= P.cells[d];
        }
        const double root[3] = {-1.0, -1.0, -1.0};
        int inside = 0;
        for (int q = lane; q < P.nq; q += 32) {
            double xi[3];
            embedded_point(P, root, 2.0, q, xi);
            inside += embedded_inside(P, corg, xi) ? 1 : 0;
        }
        inside = __reduce_add_sync(0xffffffffu, inside);
        if (lane == 0) {
            cut[e] = (inside > 0 && inside < P.nq) ? 1 : 0;
            side[e] = inside == P.nq ? 1 : 0;
        }
    }
}

__global__ void fc_compact_kernel(long ncells, const int* __restrict__ cut, const int* __restrict__ index,
                                  int* __restrict__ cutCells) {
    for (long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; e < ncells;
         e += static_cast<long>(gridDim.x) * blockDim.x)
        if (cut[e]) cutCells[index[e]] = static_cast<int>(e);
}

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void bmma_16x8x16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// (x0, x1) -> packed bf16 pairs of their high and low parts (x0 in the low half).
__device__ __forceinline__ void split_bf16x2(float x0, float x1, unsigned& hi, unsigned& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - __low2float(h), x1 - __high2float(h));
    hi = *reinterpret_cast<const unsigned*>(&h);
    lo = *reinterpret_cast<const unsigned*>(&l);
}

// Tensor-core accumulator of one CTA's partial element matrix.
//   FP64: warp w owns rows 8w..8w+7, all 8 column tiles of 8 (DMMA 8x8x4).
//   FP32: warp w owns rows 16(w/2)..+15, column tiles 4(w%2)..+3 (BF16 16x8x16).
template <bool F64>
struct Accumulator;

template <>
struct Accumulator<true> {
    double c[8][2];
    __device__ void zero() {
#pragma unroll
        for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = 0.0;
    }
    // rows: staged rows (a multiple of 4, zero-filled); w: their weights.
    __device__ void add(const double* G, const double* w, int rows, int nt) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (warp >= nt) return;
        const int col = lane >> 2, kk = lane & 3;
        for (int k0 = 0; k0 < rows; k0 += 4) {
            const double* g = G + (k0 + kk) * kFcStride + col;
            const double a = g[warp * 8] * w[k0 + kk];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < nt) dmma_8x8x4(c[j][0], c[j][1], a, g[j * 8]);
        }
    }
    __device__ void store(double* out, int nb) const {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int row = warp * 8 + (lane >> 2);
        if (row >= nb) return;
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = j * 8 + (lane & 3) * 2 + h;
                if (col < nb) out[row * nb + col] = c[j][h];
            }
    }
};

template <>
struct Accumulator<false> {
    float c[4][4];
    __device__ void zero() {
#pragma unroll
        for (int j = 0; j < 4; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
    }
    // rows: staged rows (a multiple of 16, zero-filled).  nt16: row tiles of 16,
    // nt8: column tiles of 8 in use.
    __device__ void add(const double* G, const double* w, int rows, int nt16, int nt8) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int tr = warp >> 1, tc0 = (warp & 1) * 4;
        if (tr >= nt16 || tc0 >= nt8) return;
        const int g = lane >> 2, t = lane & 3;
        for (int k0 = 0; k0 < rows; k0 += 16) {
            // A[i][k] = w_k G[k][16 tr + i]: (g, 2t..2t+1), (g+8, ..), (g, 2t+8..), (g+8, 2t+8..)
            unsigned ahi[4], alo[4];
            const int ks[2] = {k0 + 2 * t, k0 + 2 * t + 8};
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int k = ks[half];
                const double w0 = w[k], w1 = w[k + 1];
#pragma unroll
                for (int rr = 0; rr < 2; ++rr) {
                    const int i = tr * 16 + g + rr * 8;
                    split_bf16x2(static_cast<float>(w0 * G[k * kFcStride + i]),
                                 static_cast<float>(w1 * G[(k + 1) * kFcStride + i]), ahi[half * 2 + rr],
                                 alo[half * 2 + rr]);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (tc0 + j >= nt8) break;
                const int n = (tc0 + j) * 8 + g;
                unsigned bhi[2], blo[2];
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const int k = ks[half];
                    split_bf16x2(static_cast<float>(G[k * kFcStride + n]), static_cast<float>(G[(k + 1) * kFcStride + n]),
                                 bhi[half], blo[half]);
                }
                bmma_16x8x16(c[j], ahi, bhi);
                bmma_16x8x16(c[j], ahi, blo);
                bmma_16x8x16(c[j], alo, bhi);
            }
        }
    }
    __device__ void store(float* out, int nb) const {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int tr = warp >> 1, tc0 = (warp & 1) * 4;
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int row = tr * 16 + g + (h >> 1) * 8;
                const int col = (tc0 + j) * 8 + t * 2 + (h & 1);
                if (row < nb && col < nb) out[row * nb + col] = c[j][h];
            }
    }
};

// One CTA per (cut cell of the batch, start node).  Start nodes: the 2^dim
// children of the root (depth 1) when maxDepth >= 1, else the root.  The CTA
// walks the start node's subtree depth-first with the rules of
// KDTreeQuadraturePointFactory.hpp:156-170 and adds the kept points' terms.
template <bool F64>
__global__ void __launch_bounds__(kFcThreads)
    fc_partial_kernel(EmbeddedArgs P, const int* __restrict__ cutCells, int first, int nstart,
                      typename std::conditional<F64, double, float>::type* __restrict__ partial) {
    __shared__ double s_G[kFcRows * kFcStride];
    __shared__ double s_w[kFcRows];
    __shared__ double s_v[kFcPoints][3][16], s_dv[kFcPoints][3][16];
    __shared__ double s_stack[kFcStack][4];  // base[3], length
    __shared__ int s_stackDepth[kFcStack];
    __shared__ int s_top;
    __shared__ double s_node[4];
    __shared__ int s_nodeDepth;
    __shared__ int s_inside;
    const int t = threadIdx.x;
    const int dim = P.dim, nb = P.nb, nq = P.nq, n1 = P.order + 1;
    const int item = blockIdx.x;
    const int e = cutCells[first + item / nstart];
    const int startChild = item % nstart;
    double corg[3] = {0.0, 0.0, 0.0};
    {
        long rest = e;
        for (int d = 0; d < dim; ++d) {
            corg[d] = P.origin[d] + static_cast<double>(rest % P.cells[d]) * P.h[d];
            rest /= P.cells[d];
        }
    }
    Accumulator<F64> acc;
    acc.zero();
    const int nt8 = (nb + 7) / 8, nt16 = (nb + 15) / 16;
    if (t == 0) {
        s_top = 1;
        if (nstart == 1) {
            s_stack[0][0] = s_stack[0][1] = s_stack[0][2] = -1.0;
            s_stack[0][3] = 2.0;
            s_stackDepth[0] = 0;
        } else {
            for (int d = 0; d < 3; ++d) s_stack[0][d] = d < dim ? -1.0 + ((startChild >> d) & 1) : -1.0;
            s_stack[0][3] = 1.0;
            s_stackDepth[0] = 1;
        }
    }
    __syncthreads();
    for (;;) {
        const int top = s_top;  // every thread reads it before thread 0 pops
        __syncthreads();
        if (top == 0) break;
        if (t == 0) {
            const int k = --s_top;
            for (int j = 0; j < 4; ++j) s_node[j] = s_stack[k][j];
            s_nodeDepth = s_stackDepth[k];
        }
        __syncthreads();
        const double base[3] = {s_node[0], s_node[1], s_node[2]};
        const double length = s_node[3];
        const int depth = s_nodeDepth;
        int mine = 0;
        for (int q = t; q < nq; q += kFcThreads) {
            double xi[3];
            embedded_point(P, base, length, q, xi);
            mine += embedded_inside(P, corg, xi) ? 1 : 0;
        }
        // number of inside points of the node
        if (t == 0) s_inside = 0;
        __syncthreads();
        if (mine) atomicAdd(&s_inside, mine);
        __syncthreads();
        const int nin = s_inside;
        const bool homogeneous = nin == 0 || nin == nq;
        const bool keep = (homogeneous && nin == nq) || depth == P.maxDepth || (depth == 0 && homogeneous);
        if (keep) {
            double jac = 1.0;
            for (int d = 0; d < dim; ++d) jac *= 0.5 * length;
            for (int q0 = 0; q0 < nq; q0 += kFcPoints) {
                const int np = min(kFcPoints, nq - q0);
                const int rows = np * dim;
                const int padded = F64 ? (rows + 3) & ~3 : (rows + 15) & ~15;
                if (t < np * dim) {
                    const int p = t / dim, d = t - (t / dim) * dim;
                    double xi[3];
                    embedded_point(P, base, length, q0 + p, xi);
                    lagrange(P.order, xi[d], s_v[p][d], s_dv[p][d]);
                }
                if (t < np) {
                    double xi[3];
                    const double w = embedded_point(P, base, length, q0 + t, xi) * jac *
                                     (embedded_inside(P, corg, xi) ? 1.0 : P.alpha);
                    for (int d = 0; d < dim; ++d) s_w[t * dim + d] = w * P.f[d];
                }
                for (int r = rows + t; r < padded; r += kFcThreads) s_w[r] = 0.0;
                __syncthreads();
                // B rows (point p, axis dd): G[a] = prod_d (d == dd ? dN : N)_{i_d(a)}; columns >= nb are 0
                for (int idx = t; idx < padded * 64; idx += kFcThreads) {
                    const int r = idx >> 6, a = idx & 63;
                    double g = 0.0;
                    if (r < rows && a < nb) {
                        const int p = r / dim, dd = r - (r / dim) * dim;
                        int ra = a;
                        g = 1.0;
                        for (int d = 0; d < dim; ++d) {
                            const int i = ra % n1;
                            ra /= n1;
                            g *= (d == dd) ? s_dv[p][d][i] : s_v[p][d][i];
                        }
                    }
                    s_G[r * kFcStride + a] = g;
                }
                __syncthreads();
                if constexpr (F64)
                    acc.add(s_G, s_w, padded, nt8);
                else
                    acc.add(s_G, s_w, padded, nt16, nt8);
                __syncthreads();
            }
        }
        if (t == 0 && !homogeneous && depth < P.maxDepth) {
            const double half = 0.5 * length;
            const int children = 1 << dim;
            for (int c = children - 1; c >= 0; --c) {  // pushed in reverse: child 0 is visited first
                const int k = s_top++;
                for (int d = 0; d < 3; ++d) s_stack[k][d] = d < dim ? base[d] + ((c >> d) & 1) * half : -1.0;
                s_stack[k][3] = half;
                s_stackDepth[k] = depth + 1;
            }
        }
        __syncthreads();
    }
    acc.store(partial + static_cast<long>(item) * nb * nb, nb);
}

// Cells of one colour: regular cells add kappa s K1 (first batch only), the cut
// cells of the batch the sum of their partials in start-node order.
template <typename V>
__global__ void fc_scatter_kernel(long count, int nb, const int* __restrict__ cellOrder, const int* __restrict__ cut,
                                  const int* __restrict__ index, const signed char* __restrict__ side,
                                  const V* __restrict__ K1, const V* __restrict__ partial, int nstart, int batchFirst,
                                  int batchEnd, int withRegular, const double* __restrict__ kappa, double alpha,
                                  double scale, const int* __restrict__ slots, V* __restrict__ val) {
    const int nb2 = nb * nb;
    const long total = count * nb2;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const long le = t / nb2;
        const int ab = static_cast<int>(t - le * nb2);
        const int e = cellOrder[le];
        const double kap = kappa ? kappa[e] : 1.0;
        const int slot = slots[static_cast<long>(e) * nb2 + ab];
        if (!cut[e]) {
            if (!withRegular) continue;
            const double s = side[e] ? 1.0 : alpha;
            val[slot] += static_cast<V>(kap * s) * K1[ab];
        } else {
            const int idx = index[e];
            if (idx < batchFirst || idx >= batchEnd) continue;
            const V* part = partial + static_cast<long>(idx - batchFirst) * nstart * nb2 + ab;
            V sum = V(0);
            for (int j = 0; j < nstart; ++j) sum += part[static_cast<long>(j) * nb2];
            val[slot] += static_cast<V>(kap * scale) * sum;
        }
    }
}

__global__ void to_float_kernel(int n, const double* __restrict__ a, float* __restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = static_cast<float>(a[i]);
}

template <bool F64>
int assemble_finite_cell(ciecu_assembly_s* P, const double* d_kappa, const double* h_cellSize, const int32_t* h_cells,
                         const double* h_origin, const double* h_center, double radius, double alpha, int maxDepth,
                         int convention, int accumulate, void* d_entries, int64_t* h_cutCells) {
    using V = typename std::conditional<F64, double, float>::type;
    CIECU_REQUIRE(P && h_cellSize && h_cells && h_origin && h_center && d_entries, "assemble_embedded: null argument");
    CIECU_REQUIRE(convention == 0 || convention == 1, "assemble_embedded: convention must be 0 or 1");
    CIECU_REQUIRE(P->nb <= 64 && P->order + 1 <= 16, "assemble_embedded: at most 64 basis functions per cell");
    CIECU_REQUIRE(P->q1 <= 16, "assemble_embedded: at most 16 quadrature points per axis");
    CIECU_REQUIRE(maxDepth >= 0 && maxDepth <= 4, "assemble_embedded: tree depth must be in [0, 4]");
    CIECU_REQUIRE(radius > 0.0, "assemble_embedded: radius must be positive");
    long cellsTotal = 1;
    for (int d = 0; d < P->dim; ++d) {
        CIECU_REQUIRE(h_cells[d] >= 1, "assemble_embedded: empty grid");
        cellsTotal *= h_cells[d];
    }
    CIECU_REQUIRE(cellsTotal == P->ncells, "assemble_embedded: grid size differs from the plan's cell count");
    cudaStream_t st = P->csr->space->stream;
    const long ncells = P->ncells;
    const int nb = P->nb, nb2 = nb * nb;
    if (!accumulate) CIECU_CUDA(cudaMemsetAsync(d_entries, 0, sizeof(V) * P->csr->nnz, st));
    if (ncells == 0) {
        if (h_cutCells) *h_cutCells = 0;
        return CIECU_OK;
    }
    EmbeddedArgs A{};
    A.dim = P->dim;
    A.order = P->order;
    A.nb = nb;
    A.q1 = P->q1;
    A.nq = P->nq;
    A.maxDepth = maxDepth;
    for (int d = 0; d < 3; ++d) {
        A.cells[d] = d < P->dim ? h_cells[d] : 1;
        A.origin[d] = d < P->dim ? h_origin[d] : 0.0;
        A.h[d] = d < P->dim ? h_cellSize[d] : 1.0;
        A.center[d] = d < P->dim ? h_center[d] : 0.0;
    }
    for (int i = 0; i < P->q1; ++i) {
        A.gn[i] = P->gn[i];
        A.gw[i] = P->gw[i];
    }
    A.radius2 = radius * radius;
    A.alpha = alpha;
    double f[3];
    convention_factors(P->dim, h_cellSize, convention, A.scale, f);
    for (int d = 0; d < 3; ++d) A.f[d] = f[d];
    const int nstart = maxDepth >= 1 ? (1 << P->dim) : 1;
    // batches of cut cells whose partial matrices fit in 512 MB
    const long perCut = static_cast<long>(nstart) * nb2 * static_cast<long>(sizeof(V));
    const long batchCap = std::max<long>(1, (512L << 20) / perCut);
    // work: K1 (FP64 and V), cut flags, their prefix sum, cut list, sides, scan work
    const long scanWork = scan_work(ncells);
    const size_t bytes = sizeof(double) * nb2 + sizeof(V) * nb2 +
                         sizeof(int) * (3 * static_cast<size_t>(ncells) + 1 + static_cast<size_t>(scanWork)) +
                         static_cast<size_t>(ncells) + 256;
    unsigned char* work = nullptr;
    CIECU_CUDA(cudaMalloc(&work, bytes));
    V* partial = nullptr;
    auto done = [&](int status) {
        cudaFree(partial);
        cudaFree(work);
        return status;
    };
    double* K1 = reinterpret_cast<double*>(work);
    V* K1v = reinterpret_cast<V*>(K1 + nb2);
    int* cut = reinterpret_cast<int*>(work + ((sizeof(double) * nb2 + sizeof(V) * nb2 + 15) & ~size_t(15)));
    int* index = cut + ncells;       // ncells + 1
    int* cutCells = index + ncells + 1;
    int* scan = cutCells + ncells;
    signed char* side = reinterpret_cast<signed char*>(scan + scanWork);
    int status = unit_element(P, A.scale, f, K1, st);
    if (status != CIECU_OK) return done(status);
    if constexpr (F64) {
        cudaError_t e = cudaMemcpyAsync(K1v, K1, sizeof(double) * nb2, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return done(cuda_fail(e, "assemble_embedded"));
    } else {
        to_float_kernel<<<(nb2 + 255) / 256, 256, 0, st>>>(nb2, K1, K1v);
        count_launch();
    }
    fc_classify_kernel<<<grid_for(ncells * 32, 256, 8), 256, 0, st>>>(A, ncells, cut, side);
    count_launch();
    status = exclusive_scan(cut, index, ncells, scan, st);
    if (status != CIECU_OK) return done(status);
    fc_compact_kernel<<<grid_for(ncells, 256, 8), 256, 0, st>>>(ncells, cut, index, cutCells);
    count_launch();
    int ncut = 0;
    cudaError_t e = cudaMemcpyAsync(&ncut, index + ncells, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(e, "assemble_embedded: classification"));
    const long batch = std::min<long>(std::max(ncut, 1), batchCap);
    if (ncut > 0) {
        e = cudaMalloc(&partial, static_cast<size_t>(batch * perCut));
        if (e != cudaSuccess) return done(cuda_fail(e, "assemble_embedded: partial matrices"));
    }
    V* val = static_cast<V*>(d_entries);
    for (long b0 = 0; b0 < std::max<long>(ncut, 1); b0 += batch) {
        const long b1 = std::min<long>(ncut, b0 + batch);
        if (b1 > b0) {
            fc_partial_kernel<F64><<<static_cast<unsigned>((b1 - b0) * nstart), kFcThreads, 0, st>>>(
                A, cutCells, static_cast<int>(b0), nstart, partial);
            count_launch();
        }
        for (size_t c = 0; c + 1 < P->colorOffsets.size(); ++c) {
            const long begin = P->colorOffsets[c], count = P->colorOffsets[c + 1] - begin;
            if (count == 0) continue;
            fc_scatter_kernel<V><<<grid_for(count * nb2, 256, 8), 256, 0, st>>>(
                count, nb, P->d_cellOrder + begin, cut, index, side, K1v, partial, nstart, static_cast<int>(b0),
                static_cast<int>(b1), b0 == 0 ? 1 : 0, d_kappa, alpha, A.scale, P->d_slots, val);
            count_launch();
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return done(cuda_fail(e, "assemble_embedded"));
    }
    e = cudaStreamSynchronize(st);  // the work buffers are in use until here
    if (e != cudaSuccess) return done(cuda_fail(e, "assemble_embedded"));
    if (h_cutCells) *h_cutCells = ncut;
    return done(CIECU_OK);
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_assemble_embedded(ciecu_assembly P, const double* d_kappa, const double* h_cellSize, const int32_t* h_cells,
                            const double* h_origin, const double* h_center, double radius, double alpha, int maxDepth,
                            int convention, int accumulate, double* d_entries, double* d_work, int64_t* h_cutCells) {
    CIECU_REQUIRE(d_work, "assemble_embedded: null argument");
    return assemble_finite_cell<true>(P, d_kappa, h_cellSize, h_cells, h_origin, h_center, radius, alpha, maxDepth,
                                      convention, accumulate, d_entries, h_cutCells);
}

int ciecu_assemble_embedded_f32(ciecu_assembly P, const double* d_kappa, const double* h_cellSize,
                                const int32_t* h_cells, const double* h_origin, const double* h_center, double radius,
                                double alpha, int maxDepth, int convention, int accumulate, float* d_entries32,
                                int64_t* h_cutCells) {
    return assemble_finite_cell<false>(P, d_kappa, h_cellSize, h_cells, h_origin, h_center, radius, alpha, maxDepth,
                                       convention, accumulate, d_entries32, h_cutCells);
}

}  // extern "C"
