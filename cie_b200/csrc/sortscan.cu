// Exclusive prefix sum over the grid: a block scan per tile of kScanTile items,
// the block totals scanned the same way (recursively), then the tile offsets
// added back.
#include "sortscan.cuh"
#include "space.cuh"

namespace ciecu {
namespace {

// Exclusive scan of one tile; tile total to sums[blockIdx.x].
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const int* __restrict__ in, int* __restrict__ out,
                                                                 long n, int* __restrict__ sums) {
    __shared__ int s_warp[32];
    const long base = static_cast<long>(blockIdx.x) * kScanTile + static_cast<long>(threadIdx.x) * kScanItems;
    int v[kScanItems];
    int local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        local += v[i];
    }
    // inclusive scan of the per-thread totals across the block
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = local;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = s_warp[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        s_warp[lane] = w;
    }
    __syncthreads();
    int running = x - local + (warp > 0 ? s_warp[warp - 1] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = running;
        running += v[i];
    }
    if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = running;
}

__global__ void scan_add_kernel(int* __restrict__ out, long n, const int* __restrict__ offsets) {
    const int add = offsets[blockIdx.x];
    const long base = static_cast<long>(blockIdx.x) * kScanTile;
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x)
        if (base + i < n) out[base + i] += add;
}

__global__ void scan_total_kernel(const int* __restrict__ in, int* __restrict__ out, long n) {
    // out[n] = out[n - 1] + in[n - 1] (n >= 1)
    out[n] = out[n - 1] + in[n - 1];
}

}  // namespace

int exclusive_scan(const int* d_in, int* d_out, long n, int* d_work, cudaStream_t st) {
    if (n <= 0) {
        CIECU_CUDA(cudaMemsetAsync(d_out, 0, sizeof(int), st));
        return CIECU_OK;
    }
    const long blocks = scan_blocks(n);
    int* sums = d_work;
    scan_tile_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, st>>>(d_in, d_out, n, sums);
    count_launch();
    CIECU_CHECK_LAUNCH("scan_tile_kernel");
    if (blocks > 1) {
        int* offsets = d_work + blocks + 1;  // scan of the block sums (blocks + 1 entries)
        CIECU_TRY(exclusive_scan(sums, offsets, blocks, offsets + blocks + 1, st));
        scan_add_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(d_out, n, offsets);
        count_launch();
        CIECU_CHECK_LAUNCH("scan_add_kernel");
    }
    scan_total_kernel<<<1, 1, 0, st>>>(d_in, d_out, n);
    count_launch();
    CIECU_CHECK_LAUNCH("scan_total_kernel");
    return CIECU_OK;
}

}  // namespace ciecu
