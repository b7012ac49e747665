// Cuthill-McKee reordering and the permutation of CSR matrices and vectors:
//   makeReordering   linalg/packages/utilities/src/reorder.cpp:23-173
//   reorder          linalg/packages/utilities/src/reorder.cpp:215-365 (CSR), :368-425 (vectors)
//
// The reference's traversal is a FIFO queue: a row is placed when it leaves the
// queue and queues its unqueued neighbours sorted by degree.  Breadth-first
// levels reproduce that order: every row of level L+1 is queued by the
// lowest-placed row of level L adjacent to it, rows queued by the same parent
// follow in (degree, index) order, and parents in placement order.  Each level
// is four kernels -- claim (atomicMin of the parent's position), count, a prefix
// sum of the counts, emit (a warp sorts its row's children in shared memory) --
// and the host reads back the next level's size.
#include "ciecu_graph.h"
#include "sortscan.cuh"
#include "space.cuh"

#include <climits>
#include <string>

struct ciecu_space_s;

namespace ciecu {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kT = 32 * kWarpsPerBlock;

__global__ void degree_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                              int* __restrict__ degree, int* __restrict__ pos, int* __restrict__ claim,
                              int* __restrict__ maxRow, int* __restrict__ bad) {
    const int stride = gridDim.x * blockDim.x;
    int longest = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int d = rowptr[i + 1] - rowptr[i];
        degree[i] = d;
        pos[i] = -1;
        claim[i] = INT_MAX;
        longest = d > longest ? d : longest;
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
            if (static_cast<unsigned>(col[e]) >= static_cast<unsigned>(n)) atomicExch(bad, 1);
    }
    longest = __reduce_max_sync(0xffffffffu, longest);
    if ((threadIdx.x & 31) == 0) atomicMax(maxRow, longest);
}

// Key (degree, index) of the least unplaced row, by atomicMin over 64-bit keys
// (the least degree, then the least index).
__global__ void least_unplaced_kernel(int n, const int* __restrict__ degree, const int* __restrict__ pos,
                                      unsigned long long* __restrict__ best) {
    const int stride = gridDim.x * blockDim.x;
    unsigned long long mine = ~0ULL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (pos[i] < 0) {
            const unsigned long long k = (static_cast<unsigned long long>(degree[i]) << 32) | static_cast<unsigned>(i);
            mine = k < mine ? k : mine;
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, mine, off);
        mine = o < mine ? o : mine;
    }
    if ((threadIdx.x & 31) == 0 && mine != ~0ULL) atomicMin(best, mine);
}

// Places the row named by *best at position `at` (a level of one row).
__global__ void place_start_kernel(const unsigned long long* __restrict__ best, int at, int* __restrict__ order,
                                   int* __restrict__ pos) {
    const int v = static_cast<int>(*best & 0xffffffffULL);
    order[at] = v;
    pos[v] = at;
}

// Every unplaced neighbour v of a level row at position k: claim[v] = min k.
__global__ void claim_kernel(int n, int begin, int end, const int* __restrict__ order, const int* __restrict__ rowptr,
                             const int* __restrict__ col, const int* __restrict__ pos, int* __restrict__ claim) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarpsPerBlock;
    for (int k = begin + blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); k < end; k += warps) {
        const int u = order[k];
        for (int e = rowptr[u] + lane; e < rowptr[u + 1]; e += 32) {
            const int v = col[e];
            if (static_cast<unsigned>(v) < static_cast<unsigned>(n) && pos[v] < 0) atomicMin(claim + v, k);
        }
    }
}

// count[k - begin] = children of the level row at position k.
__global__ void count_kernel(int n, int begin, int end, const int* __restrict__ order, const int* __restrict__ rowptr,
                             const int* __restrict__ col, const int* __restrict__ pos, const int* __restrict__ claim,
                             int* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarpsPerBlock;
    for (int k = begin + blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); k < end; k += warps) {
        const int u = order[k];
        int c = 0;
        for (int e = rowptr[u] + lane; e < rowptr[u + 1]; e += 32) {
            const int v = col[e];
            c += (static_cast<unsigned>(v) < static_cast<unsigned>(n) && pos[v] < 0 && claim[v] == k) ? 1 : 0;
        }
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) count[k - begin] = c;
    }
}

// The children of each level row, sorted by (degree, index), placed from
// end + offset[k - begin] on.
__global__ void __launch_bounds__(kT) emit_kernel(int n, int begin, int end, const int* __restrict__ order_in,
                                                  const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const int* __restrict__ degree, const int* __restrict__ claim,
                                                  const int* __restrict__ offset, int* __restrict__ order,
                                                  int* __restrict__ pos) {
    __shared__ unsigned long long s_keys[kWarpsPerBlock][CIECU_GRAPH_MAX_ROW];
    __shared__ int s_count[kWarpsPerBlock];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long* keys = s_keys[w];
    const int warps = gridDim.x * kWarpsPerBlock;
    // every warp runs the same number of rounds (no warp leaves early)
    for (int k0 = begin + blockIdx.x * kWarpsPerBlock; k0 < end; k0 += warps) {
        const int k = k0 + w;
        if (lane == 0) s_count[w] = 0;
        __syncwarp();
        if (k < end) {
            const int u = order_in[k];
            for (int e = rowptr[u] + lane; e < rowptr[u + 1]; e += 32) {
                const int v = col[e];
                // a row is claimed by one parent only, so no other warp places it
                if (static_cast<unsigned>(v) < static_cast<unsigned>(n) && claim[v] == k && pos[v] < 0) {
                    const int slot = atomicAdd(&s_count[w], 1);
                    keys[slot] = (static_cast<unsigned long long>(degree[v]) << 32) | static_cast<unsigned>(v);
                }
            }
        }
        __syncwarp();
        const int c = s_count[w];
        if (c > 1) warp_bitonic_sort(keys, c);
        __syncthreads();  // every warp has read pos[] of its neighbours before any row is placed
        if (k < end) {
            const int at = end + offset[k - begin];
            for (int i = lane; i < c; i += 32) {
                const int v = static_cast<int>(keys[i] & 0xffffffffULL);
                order[at + i] = v;
                pos[v] = at + i;
            }
        }
        __syncthreads();
    }
}

__global__ void reverse_kernel(int n, const int* __restrict__ in, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[n - 1 - i];
}

// ---- permutation -------------------------------------------------------------

__global__ void inverse_map_kernel(int n, const int* __restrict__ map, int* __restrict__ inverse,
                                   int* __restrict__ newLength, const int* __restrict__ rowptr, int* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int old = map[i];
        if (old < 0 || old >= n) {
            atomicExch(bad, 1);
            newLength[i] = 0;
            continue;
        }
        inverse[old] = i;
        newLength[i] = rowptr[old + 1] - rowptr[old];
    }
}

// One warp per new row: columns renamed, the row sorted by its new columns.
__global__ void __launch_bounds__(kT) permute_rows_kernel(int n, int* __restrict__ bad, const int* __restrict__ map,
                                                          const int* __restrict__ inverse,
                                                          const int* __restrict__ rowptr, const int* __restrict__ col,
                                                          const double* __restrict__ val,
                                                          const int* __restrict__ newRowptr, int* __restrict__ newCol,
                                                          double* __restrict__ newVal) {
    __shared__ unsigned long long s_keys[kWarpsPerBlock][CIECU_GRAPH_MAX_ROW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long* keys = s_keys[w];
    const int warps = gridDim.x * kWarpsPerBlock;
    for (int i = blockIdx.x * kWarpsPerBlock + w; i < n; i += warps) {
        const int old = map[i];
        const int b = rowptr[old], len = rowptr[old + 1] - b;
        for (int j = lane; j < len; j += 32) {
            const int c = col[b + j];
            unsigned renamed = 0xffffffffu;  // an out-of-range column sorts last and is flagged
            if (static_cast<unsigned>(c) < static_cast<unsigned>(n))
                renamed = static_cast<unsigned>(inverse[c]);
            else
                atomicExch(bad, 1);
            keys[j] = (static_cast<unsigned long long>(renamed) << 32) | static_cast<unsigned>(j);
        }
        __syncwarp();
        if (len > 1) warp_bitonic_sort(keys, len);
        const int nb = newRowptr[i];
        for (int j = lane; j < len; j += 32) {
            const unsigned long long key = keys[j];
            newCol[nb + j] = static_cast<int>(key >> 32);
            newVal[nb + j] = val[b + static_cast<int>(key & 0xffffffffULL)];
        }
        __syncwarp();
    }
}

__global__ void permute_vector_kernel(long n, const int* __restrict__ map, int reverse, const double* __restrict__ in,
                                      double* __restrict__ out) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        if (reverse)
            out[map[i]] = in[i];
        else
            out[i] = in[map[i]];
    }
}

__global__ void max_kernel(int n, const int* __restrict__ v, int* __restrict__ out) {
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = v[i] > m ? v[i] : m;
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

int blocks_for_warps(long warps) {
    const long need = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const long cap = static_cast<long>(sm_count()) * 16;
    return static_cast<int>(need < 1 ? 1 : (need < cap ? need : cap));
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_make_reordering(ciecu_space space, int32_t n, const int32_t* d_rowExtents, const int32_t* d_columnIndices,
                          int strategy, int32_t* d_map) {
    CIECU_REQUIRE(space && n >= 0, "make_reordering: invalid arguments");
    CIECU_REQUIRE(strategy == 1 || strategy == 2, "make_reordering: strategy must be 1 (Cuthill-McKee) or 2 (reverse)");
    if (n == 0) return CIECU_OK;
    CIECU_REQUIRE(d_rowExtents && d_columnIndices && d_map, "make_reordering: null array");
    cudaStream_t st = space->stream;
    // work: degree, pos, claim, count (n each), the prefix sums (n + 1), the
    // order (n), scan work, and the key / longest-row words
    const long scanWork = scan_work(n);
    int* work = nullptr;
    const size_t ints = 6 * static_cast<size_t>(n) + 1 + static_cast<size_t>(scanWork) + 8;
    CIECU_CUDA(cudaMalloc(&work, sizeof(int) * ints));
    int* degree = work;
    int* pos = degree + n;
    int* claim = pos + n;
    int* count = claim + n;
    int* offset = count + n;        // n + 1
    int* order = offset + n + 1;    // n
    int* scan = order + n;          // scanWork
    long tail = 6L * n + 1 + scanWork;  // first free int; the 64-bit key starts at an even one
    tail += tail & 1;
    unsigned long long* best = reinterpret_cast<unsigned long long*>(work + tail);
    int* maxRow = work + tail + 2;
    int* bad = maxRow + 1;
    auto done = [&](int status) {
        cudaFree(work);
        return status;
    };
    cudaError_t e = cudaMemsetAsync(maxRow, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return done(cuda_fail(e, "make_reordering"));
    const int gridN = grid_for(n, 256, 8);
    degree_kernel<<<gridN, 256, 0, st>>>(n, d_rowExtents, d_columnIndices, degree, pos, claim, maxRow, bad);
    count_launch();
    int flags[2] = {0, 0};  // longest row, out-of-range column
    e = cudaMemcpyAsync(flags, maxRow, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(e, "make_reordering: degrees"));
    const int longest = flags[0];
    if (flags[1]) return done(fail(CIECU_ERR_ARGUMENT, "make_reordering: a column index lies outside [0, n)"));
    if (longest > CIECU_GRAPH_MAX_ROW)
        return done(fail(CIECU_ERR_ARGUMENT, "make_reordering: a row holds " + std::to_string(longest) +
                                                 " entries, more than " + std::to_string(CIECU_GRAPH_MAX_ROW)));
    int placed = 0, begin = 0;
    while (placed < n) {
        if (placed == begin) {
            // the queue is empty: the least unplaced row starts a component
            e = cudaMemsetAsync(best, 0xff, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return done(cuda_fail(e, "make_reordering"));
            least_unplaced_kernel<<<gridN, 256, 0, st>>>(n, degree, pos, best);
            place_start_kernel<<<1, 1, 0, st>>>(best, placed, order, pos);
            count_launch(2);
            placed += 1;
        }
        const int end = placed;
        const int levelRows = end - begin;
        const int grid = blocks_for_warps(levelRows);
        claim_kernel<<<grid, kT, 0, st>>>(n, begin, end, order, d_rowExtents, d_columnIndices, pos, claim);
        count_kernel<<<grid, kT, 0, st>>>(n, begin, end, order, d_rowExtents, d_columnIndices, pos, claim, count);
        count_launch(2);
        const int status = exclusive_scan(count, offset, levelRows, scan, st);
        if (status != CIECU_OK) return done(status);
        emit_kernel<<<grid, kT, 0, st>>>(n, begin, end, order, d_rowExtents, d_columnIndices, degree, claim, offset,
                                         order, pos);
        count_launch();
        int added = 0;
        e = cudaMemcpyAsync(&added, offset + levelRows, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return done(cuda_fail(e, "make_reordering: level"));
        if (added < 0 || added > n - placed) return done(fail(CIECU_ERR_ARGUMENT, "make_reordering: inconsistent level"));
        begin = end;
        placed = end + added;
    }
    if (strategy == 2)
        reverse_kernel<<<gridN, 256, 0, st>>>(n, order, d_map);
    else
        e = cudaMemcpyAsync(d_map, order, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
    count_launch(strategy == 2 ? 1 : 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    return done(e == cudaSuccess ? CIECU_OK : cuda_fail(e, "make_reordering"));
}

int ciecu_reorder_csr(ciecu_space space, int32_t n, const int32_t* d_map, const int32_t* d_rowExtents,
                      const int32_t* d_columnIndices, const double* d_entries, int32_t* d_newRowExtents,
                      int32_t* d_newColumnIndices, double* d_newEntries) {
    CIECU_REQUIRE(space && n >= 0, "reorder_csr: invalid arguments");
    CIECU_REQUIRE(d_rowExtents && d_newRowExtents, "reorder_csr: null row extents");
    cudaStream_t st = space->stream;
    if (n == 0) {
        CIECU_CUDA(cudaMemsetAsync(d_newRowExtents, 0, sizeof(int), st));
        return CIECU_OK;
    }
    CIECU_REQUIRE(d_map, "reorder_csr: null map");
    const long scanWork = scan_work(n);
    int* work = nullptr;
    CIECU_CUDA(cudaMalloc(&work, sizeof(int) * (2 * static_cast<size_t>(n) + 2 + scanWork)));
    int* inverse = work;
    int* length = inverse + n;
    int* bad = length + n;
    int* scan = bad + 1;
    auto done = [&](int status) {
        cudaFree(work);
        return status;
    };
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), st);
    if (e != cudaSuccess) return done(cuda_fail(e, "reorder_csr"));
    inverse_map_kernel<<<grid_for(n, 256, 8), 256, 0, st>>>(n, d_map, inverse, length, d_rowExtents, bad);
    count_launch();
    int status = exclusive_scan(length, d_newRowExtents, n, scan, st);
    if (status != CIECU_OK) return done(status);
    int flags[2] = {0, 0};  // bad map, nnz
    e = cudaMemcpyAsync(&flags[0], bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flags[1], d_rowExtents + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(cuda_fail(e, "reorder_csr"));
    if (flags[0]) return done(fail(CIECU_ERR_ARGUMENT, "reorder_csr: the map holds a row index outside [0, n)"));
    if (flags[1] > 0) {
        if (!d_columnIndices || !d_entries || !d_newColumnIndices || !d_newEntries)
            return done(fail(CIECU_ERR_ARGUMENT, "reorder_csr: null column or value array"));
        // the longest row must fit the per-warp sort buffer
        int longest = 0;
        e = cudaMemsetAsync(bad, 0, sizeof(int), st);
        if (e == cudaSuccess) {
            max_kernel<<<grid_for(n, 256, 8), 256, 0, st>>>(n, length, bad);
            count_launch();
            e = cudaMemcpyAsync(&longest, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return done(cuda_fail(e, "reorder_csr"));
        if (longest > CIECU_GRAPH_MAX_ROW)
            return done(fail(CIECU_ERR_ARGUMENT, "reorder_csr: a row holds " + std::to_string(longest) +
                                                     " entries, more than " + std::to_string(CIECU_GRAPH_MAX_ROW)));
        permute_rows_kernel<<<blocks_for_warps(n), kT, 0, st>>>(n, bad, d_map, inverse, d_rowExtents,
                                                                d_columnIndices, d_entries, d_newRowExtents,
                                                                d_newColumnIndices, d_newEntries);
        count_launch();
        int outOfRange = 0;
        e = cudaMemcpyAsync(&outOfRange, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && outOfRange)
            return done(fail(CIECU_ERR_ARGUMENT, "reorder_csr: a column index lies outside [0, n)"));
    }
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    return done(e == cudaSuccess ? CIECU_OK : cuda_fail(e, "reorder_csr"));
}

int ciecu_reorder_vector(ciecu_space space, int64_t n, const int32_t* d_map, int reverse, const double* d_in,
                         double* d_out) {
    CIECU_REQUIRE(space && n >= 0 && (reverse == 0 || reverse == 1), "reorder_vector: invalid arguments");
    if (n == 0) return CIECU_OK;
    CIECU_REQUIRE(d_map && d_in && d_out && d_in != d_out, "reorder_vector: null or aliased vector");
    permute_vector_kernel<<<grid_for(n, 256, 8), 256, 0, space->stream>>>(n, d_map, reverse, d_in, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("permute_vector_kernel");
    return CIECU_OK;
}

}  // extern "C"
