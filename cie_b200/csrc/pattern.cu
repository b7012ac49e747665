// Sparsity pattern of a DoF map on the device: Assembler::makeCSRMatrix
// (fem/packages/graph/src/Assembler.cpp:55-175), whose row i is the sorted,
// distinct union of the DoF lists of the cells that contain DoF i.
//
//   1. cells per DoF (atomic counts), their prefix sum, the cell lists;
//   2. one warp per row gathers the DoFs of the row's cells into shared memory,
//      sorts them (bitonic), and counts (first call) or writes (second call) the
//      distinct ones;
//   3. the prefix sum of the row counts gives the row extents.
// The order of the cells inside a DoF's list depends on atomics, but the row is
// sorted, so the pattern does not.
#include "ciecu_graph.h"
#include "sortscan.cuh"
#include "space.cuh"

#include <algorithm>
#include <string>

namespace ciecu {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kT = 32 * kWarpsPerBlock;

__global__ void cell_count_kernel(long entries, const int* __restrict__ dofmap, int ndofs, int* __restrict__ count,
                                  int* __restrict__ bad) {
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < entries;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int d = dofmap[t];
        if (static_cast<unsigned>(d) < static_cast<unsigned>(ndofs))
            atomicAdd(count + d, 1);
        else
            atomicExch(bad, 1);
    }
}

__global__ void cell_fill_kernel(long ncells, int nb, const int* __restrict__ dofmap, const int* __restrict__ start,
                                 int* __restrict__ cursor, int* __restrict__ cells) {
    const long entries = ncells * nb;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < entries;
         t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int d = dofmap[t];
        cells[start[d] + atomicAdd(cursor + d, 1)] = static_cast<int>(t / nb);
    }
}

// Row i: the distinct DoFs of its cells, counted (col == nullptr) or written
// from rowptr[i] on.  Candidates beyond the sort buffer are flagged, not read.
__global__ void __launch_bounds__(kT) row_union_kernel(int ndofs, int nb, const int* __restrict__ dofmap,
                                                       const int* __restrict__ start, const int* __restrict__ cells,
                                                       int* __restrict__ rowCount, const int* __restrict__ rowptr,
                                                       int* __restrict__ col, int* __restrict__ tooLong) {
    __shared__ unsigned long long s_keys[kWarpsPerBlock][CIECU_GRAPH_MAX_ROW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long* keys = s_keys[w];
    const int warps = gridDim.x * kWarpsPerBlock;
    for (int i = blockIdx.x * kWarpsPerBlock + w; i < ndofs; i += warps) {
        const int c0 = start[i], nc = start[i + 1] - c0;
        const int m = nc * nb;
        if (m > CIECU_GRAPH_MAX_ROW) {
            if (lane == 0) {
                atomicExch(tooLong, 1);
                if (!col) rowCount[i] = 0;
            }
            continue;
        }
        for (int j = lane; j < m; j += 32) keys[j] = static_cast<unsigned>(dofmap[static_cast<long>(cells[c0 + j / nb]) * nb + j % nb]);
        __syncwarp();
        if (m > 1) warp_bitonic_sort(keys, m);
        // distinct entries: the first of each run of equal keys
        int base = 0;
        for (int j0 = 0; j0 < m; j0 += 32) {
            const int j = j0 + lane;
            const bool first = j < m && (j == 0 || keys[j] != keys[j - 1]);
            const unsigned ballot = __ballot_sync(0xffffffffu, first);
            if (col && first) col[rowptr[i] + base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<int>(keys[j]);
            base += __popc(ballot);
        }
        if (!col && lane == 0) rowCount[i] = base;
        __syncwarp();
    }
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_csr_pattern_device(ciecu_space space, int64_t ncells, int nb, const int32_t* d_dofmap, int32_t ndofs,
                             int32_t* d_rowExtents, int32_t* d_columnIndices, int64_t* h_nnz) {
    CIECU_REQUIRE(space && ncells >= 0 && nb >= 1 && ndofs >= 0 && d_rowExtents && (ncells == 0 || d_dofmap),
                  "csr_pattern_device: invalid arguments");
    // every row count is at most (cells of the DoF) x nb, so the int32 prefix sums
    // cannot overflow while ncells * nb * nb < 2^31
    CIECU_REQUIRE(ncells * nb * nb < (1LL << 31), "csr_pattern_device: ncells * nb^2 must stay below 2^31");
    cudaStream_t st = space->stream;
    const long entries = ncells * nb;
    const long scanWork = scan_work(ndofs + 1);
    int* work = nullptr;
    // count / cursor (ndofs), start (ndofs + 1), cells (entries), row counts
    // (ndofs), flags, scan work
    const size_t ints = 3 * static_cast<size_t>(ndofs) + 1 + static_cast<size_t>(entries) + 4 + scanWork;
    CIECU_CUDA(cudaMalloc(&work, sizeof(int) * ints));
    int* count = work;
    int* start = count + ndofs;
    int* cells = start + ndofs + 1;
    int* rowCount = cells + entries;
    int* flags = rowCount + ndofs;  // bad DoF index, row too long
    int* scan = flags + 4;
    auto done = [&](int status) {
        cudaFree(work);
        return status;
    };
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * static_cast<size_t>(ndofs), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, sizeof(int) * 4, st);
    if (e != cudaSuccess) return done(cuda_fail(e, "csr_pattern_device"));
    if (entries > 0) {
        cell_count_kernel<<<grid_for(entries, 256, 8), 256, 0, st>>>(entries, d_dofmap, ndofs, count, flags);
        count_launch();
    }
    int h_flags[2] = {0, 0};
    e = cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(e, "csr_pattern_device"));
    if (h_flags[0]) return done(fail(CIECU_ERR_ARGUMENT, "csr_pattern_device: DoF index out of range"));
    int status = exclusive_scan(count, start, ndofs, scan, st);
    if (status != CIECU_OK) return done(status);
    if (entries > 0) {
        e = cudaMemsetAsync(count, 0, sizeof(int) * static_cast<size_t>(ndofs), st);  // now the fill cursors
        if (e != cudaSuccess) return done(cuda_fail(e, "csr_pattern_device"));
        cell_fill_kernel<<<grid_for(entries, 256, 8), 256, 0, st>>>(ncells, nb, d_dofmap, start, count, cells);
        count_launch();
    }
    const long warps = ndofs;
    const long blocks = std::max<long>(1, std::min<long>((warps + kWarpsPerBlock - 1) / kWarpsPerBlock,
                                                         static_cast<long>(sm_count()) * 16));
    if (ndofs > 0) {
        row_union_kernel<<<static_cast<int>(blocks), kT, 0, st>>>(ndofs, nb, d_dofmap, start, cells, rowCount,
                                                                  d_rowExtents, d_columnIndices, flags + 1);
        count_launch();
    }
    if (!d_columnIndices) {
        status = exclusive_scan(rowCount, d_rowExtents, ndofs, scan, st);
        if (status != CIECU_OK) return done(status);
    }
    e = cudaMemcpyAsync(h_flags, flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st);
    int nnz = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nnz, d_rowExtents + ndofs, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(e, "csr_pattern_device"));
    if (h_flags[1])
        return done(fail(CIECU_ERR_ARGUMENT, "csr_pattern_device: the cells around a DoF hold more than " +
                                                 std::to_string(CIECU_GRAPH_MAX_ROW) + " DoF entries"));
    if (nnz < 0) return done(fail(CIECU_ERR_ARGUMENT, "csr_pattern_device: more than 2^31-1 entries"));
    if (h_nnz) *h_nnz = nnz;
    return done(CIECU_OK);
}

}  // extern "C"
