// CSR operator: handle, row-block schedule, autotuner and the product kernels of
// CSROperator::product (linalg/packages/solvers/src/CSROperator.cpp:33-111) and
// MaskedCSROperator::product (MaskedCSROperator.cpp:37-118).
#include "spmv.cuh"
#include "space.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace ciecu {

namespace {

// out = combine(inScale, out, outScale, A in); out is only read when inScale != 0.
template <typename T>
struct AxpbyOp {
    using Pre = T;
    T inScale, outScale;
    T* __restrict__ y;
    __device__ __forceinline__ T pre(int r) const { return inScale == T(0) ? T(0) : y[r]; }
    __device__ __forceinline__ void post(int r, T old, T sum) const { y[r] = combine(inScale, old, outScale, sum); }
};

template <int KERNEL, typename T, typename V, bool MASKED>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    spmv_kernel(CsrArgs<V> A, T inScale, const T* __restrict__ x, T outScale, T* __restrict__ y) {
    AxpbyOp<T> op{inScale, outScale, y};
    csr_rows<KERNEL, T, V, MASKED>(A, x, op);
}

// Row-block boundaries: greedy, at most kStreamTile entries and kStreamMaxRows
// rows per block; a row longer than the tile is a block of its own.
std::vector<int> make_row_blocks(const int* rowptr, int n) {
    std::vector<int> blocks{0};
    int r0 = 0;
    while (r0 < n) {
        int r1 = r0 + 1;
        if (rowptr[r1] - rowptr[r0] <= kStreamTile) {
            while (r1 < n && r1 - r0 < kStreamMaxRows && rowptr[r1 + 1] - rowptr[r0] <= kStreamTile) ++r1;
        }
        blocks.push_back(r1);
        r0 = r1;
    }
    return blocks;
}

// A page-locked host buffer, grown on demand and kept for the life of the
// process, through which csr_create reads the row extents back (a copy into
// pageable memory goes through a driver bounce buffer at a fraction of the
// rate).  The lock is held while the buffer is in use.
std::mutex g_stagingMutex;
void* g_staging = nullptr;
size_t g_stagingBytes = 0;

cudaError_t staging_reserve(size_t bytes) {
    if (bytes <= g_stagingBytes) return cudaSuccess;
    if (g_staging) cudaFreeHost(g_staging);
    g_staging = nullptr;
    g_stagingBytes = 0;
    const size_t grown = std::max(bytes, static_cast<size_t>(1) << 20);
    const cudaError_t e = cudaMallocHost(&g_staging, grown);
    if (e == cudaSuccess) g_stagingBytes = grown;
    return e;
}

// Column indices outside [0, ncols) are counted; csr_create refuses such a matrix
// so that no product ever reads outside the input vector.
__global__ void validate_columns_kernel(long nnz, const int* __restrict__ col, int ncols, unsigned* bad) {
    unsigned mine = 0;
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long k = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        const int c = col[k];
        mine |= (c < 0 || c >= ncols) ? 1u : 0u;
    }
    if (__any_sync(0xffffffffu, mine) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

// Tuned schedule per matrix shape and value type, shared across handles.
std::mutex g_tuneMutex;
std::map<std::tuple<int, long, int, int>, int> g_tuned;

template <typename T>
int launch_spmv(ciecu_csr_s* csr, int kernel, const uint16_t* mask, uint16_t threshold, T inScale, const T* x,
                T outScale, T* y) {
    const int grid = csr_grid(csr, kernel);
    return with_schedule(kernel, [&](auto k) -> int {
        constexpr int K = decltype(k)::value;
        if (mask)
            spmv_kernel<K, T, T, true><<<fit_grid(spmv_kernel<K, T, T, true>, csr_threads<K>(), grid),
                                         csr_threads<K>(), 0, csr->space->stream>>>(csr->args<T>(mask, threshold),
                                                                                    inScale, x, outScale, y);
        else
            spmv_kernel<K, T, T, false><<<fit_grid(spmv_kernel<K, T, T, false>, csr_threads<K>(), grid),
                                          csr_threads<K>(), 0, csr->space->stream>>>(csr->args<T>(), inScale, x,
                                                                                     outScale, y);
        count_launch();
        CIECU_CHECK_LAUNCH("spmv_kernel");
        return CIECU_OK;
    });
}

int candidates(const ciecu_csr_s* csr, std::vector<int>& out) {
    out.clear();
    out.push_back(1);
    for (int vs : {2, 4, 8, 16, 32})
        if (vs <= 2 * std::max(1.0, csr->avgRow) || vs == 32) out.push_back(vs);
    return CIECU_OK;
}

template <typename T>
int autotune(ciecu_csr_s* csr) {
    std::vector<int> cand;
    candidates(csr, cand);
    T* x = nullptr;
    T* y = nullptr;
    CIECU_CUDA(cudaMalloc(&x, sizeof(T) * std::max(1, csr->cols)));
    CIECU_CUDA(cudaMalloc(&y, sizeof(T) * std::max(1, csr->rows)));
    cudaStream_t s = csr->space->stream;
    CIECU_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * std::max(1, csr->cols), s));
    CIECU_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * std::max(1, csr->rows), s));
    cudaEvent_t e0, e1;
    CIECU_CUDA(cudaEventCreate(&e0));
    CIECU_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestKernel = 1;
    int status = CIECU_OK;
    for (int k : cand) {
        for (int rep = 0; rep < 2 && status == CIECU_OK; ++rep)
            status = launch_spmv<T>(csr, k, nullptr, 0, T(0), x, T(1), y);
        cudaEventRecord(e0, s);
        const int reps = 5;
        for (int rep = 0; rep < reps && status == CIECU_OK; ++rep)
            status = launch_spmv<T>(csr, k, nullptr, 0, T(0), x, T(1), y);
        cudaEventRecord(e1, s);
        if (status != CIECU_OK) break;
        cudaError_t err = cudaEventSynchronize(e1);
        if (err != cudaSuccess) {
            status = cuda_fail(err, "autotune");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            bestKernel = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(x);
    cudaFree(y);
    if (status != CIECU_OK) return status;
    csr->kernel = bestKernel;
    return CIECU_OK;
}

}  // namespace

// Blocks a CSR row pass needs for the schedule (callers cap it with fit_grid).
int csr_grid(const ciecu_csr_s* csr, int kernel) {
    if (kernel == 1) return std::max(1, csr->nblocks);
    const long rowsPerCta = static_cast<long>(kVectorThreads / 32) * (32 / kernel);
    return static_cast<int>(std::max(1L, (csr->rows + rowsPerCta - 1) / rowsPerCta));
}

int ensure_tuned(ciecu_csr_s* csr) {
    if (csr->kernel != 0) return CIECU_OK;
    const auto key = std::make_tuple(csr->rows, csr->nnz, csr->valueType, static_cast<int>(csr->aligned16));
    {
        std::lock_guard<std::mutex> lock(g_tuneMutex);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            csr->kernel = it->second;
            return CIECU_OK;
        }
    }
    const int status = csr->valueType == CIECU_F64 ? autotune<double>(csr) : autotune<float>(csr);
    if (status != CIECU_OK) return status;
    std::lock_guard<std::mutex> lock(g_tuneMutex);
    g_tuned[key] = csr->kernel;
    return CIECU_OK;
}

}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_csr_create(ciecu_space space, int32_t rowCount, int32_t columnCount, int64_t nnz,
                     const int32_t* d_rowExtents, const int32_t* d_columnIndices, const void* d_entries,
                     int valueType, ciecu_csr* out) {
    CIECU_REQUIRE(space && out, "csr_create: null space or output");
    CIECU_REQUIRE(rowCount >= 0 && columnCount >= 0 && nnz >= 0,
                  "expecting the row extents of a CSR matrix to have at least 1 entry, but it has none");
    CIECU_REQUIRE(d_rowExtents, "expecting the row extents of a CSR matrix to have at least 1 entry, but it has none");
    CIECU_REQUIRE(nnz == 0 || (d_columnIndices && d_entries),
                  "number of column indices is inconsistent with the number of entries in the provided CSR matrix");
    CIECU_REQUIRE(valueType == CIECU_F64 || valueType == CIECU_F32, "csr_create: unknown value type");
    CIECU_REQUIRE(nnz < (1LL << 31), "csr_create: int32 column indices limit nnz to 2^31-1");
    auto* csr = new ciecu_csr_s();
    csr->space = space;
    csr->rows = rowCount;
    csr->cols = columnCount;
    csr->nnz = nnz;
    csr->rowptr = d_rowExtents;
    csr->col = d_columnIndices;
    csr->val = d_entries;
    csr->valueType = valueType;
    csr->aligned16 = (reinterpret_cast<uintptr_t>(d_columnIndices) % 16 == 0) &&
                     (reinterpret_cast<uintptr_t>(d_entries) % 16 == 0);
    // Row extents come back to the host once (through the pinned staging buffer)
    // to check them (rowptr[0] == 0, monotone, rowptr[rows] == nnz), find the
    // longest row and build the row-block schedule.
    std::unique_lock<std::mutex> staging(g_stagingMutex);
    const size_t extentBytes = sizeof(int) * (static_cast<size_t>(rowCount) + 1);
    cudaError_t e = staging_reserve(extentBytes);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g_staging, d_rowExtents, extentBytes, cudaMemcpyDeviceToHost, space->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(space->stream);
    if (e != cudaSuccess) {
        delete csr;
        return cuda_fail(e, "csr_create: reading row extents");
    }
    const int* rowptr = static_cast<const int*>(g_staging);
    if (rowptr[0] != 0 || rowptr[rowCount] != nnz) {
        delete csr;
        return fail(CIECU_ERR_ARGUMENT, "number of column indices (" + std::to_string(nnz) +
                                            ") is inconsistent with the row extents of the provided CSR matrix");
    }
    int maxRow = 0;
    for (int r = 0; r < rowCount; ++r) {
        const int len = rowptr[r + 1] - rowptr[r];
        if (len < 0) {
            delete csr;
            return fail(CIECU_ERR_ARGUMENT, "row extents of the provided CSR matrix are not monotone at row " +
                                                std::to_string(r));
        }
        maxRow = std::max(maxRow, len);
    }
    csr->maxRow = maxRow;
    csr->avgRow = rowCount ? static_cast<double>(nnz) / rowCount : 0.0;
    const std::vector<int> blocks = make_row_blocks(rowptr, rowCount);
    staging.unlock();
    if (nnz > 0) {
        unsigned* d_bad = reinterpret_cast<unsigned*>(space->d_result);
        unsigned bad = 0;
        e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), space->stream);
        if (e == cudaSuccess) {
            validate_columns_kernel<<<grid_for(nnz, 256, 8), 256, 0, space->stream>>>(nnz, d_columnIndices, columnCount,
                                                                                    d_bad);
            count_launch();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, space->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(space->stream);
        if (e != cudaSuccess) {
            delete csr;
            return cuda_fail(e, "csr_create: validating column indices");
        }
        if (bad) {
            delete csr;
            return fail(CIECU_ERR_ARGUMENT, "column index out of range [0, " + std::to_string(columnCount) +
                                                ") in the provided CSR matrix");
        }
    }
    csr->nblocks = static_cast<int>(blocks.size()) - 1;
    e = pool_alloc(&csr->d_blocks, sizeof(int) * blocks.size(), space->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(csr->d_blocks, blocks.data(), sizeof(int) * blocks.size(), cudaMemcpyHostToDevice,
                            space->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(space->stream);
    if (e != cudaSuccess) {
        pool_release({csr->d_blocks});
        delete csr;
        return cuda_fail(e, "csr_create: row-block schedule");
    }
    *out = csr;
    return CIECU_OK;
}

int ciecu_csr_destroy(ciecu_csr csr) {
    if (!csr) return CIECU_OK;
    // No access to csr->space (it may already be gone); pool_release synchronises the device.
    pool_release({csr->d_blocks});
    delete csr;
    return CIECU_OK;
}

int ciecu_csr_set_kernel(ciecu_csr csr, int kernel) {
    CIECU_REQUIRE(csr, "csr_set_kernel: null matrix");
    CIECU_REQUIRE(kernel == 0 || kernel == 1 || kernel == 2 || kernel == 4 || kernel == 8 || kernel == 16 ||
                      kernel == 32,
                  "csr_set_kernel: kernel must be 0, 1, 2, 4, 8, 16 or 32");
    csr->kernel = kernel;
    return CIECU_OK;
}

int ciecu_csr_get_kernel(ciecu_csr csr, int* kernel) {
    CIECU_REQUIRE(csr && kernel, "csr_get_kernel: null argument");
    *kernel = csr->kernel;
    return CIECU_OK;
}

int ciecu_csr_autotune(ciecu_csr csr) {
    CIECU_REQUIRE(csr, "csr_autotune: null matrix");
    csr->kernel = 0;
    {
        std::lock_guard<std::mutex> lock(g_tuneMutex);
        g_tuned.erase(std::make_tuple(csr->rows, csr->nnz, csr->valueType, static_cast<int>(csr->aligned16)));
    }
    return ensure_tuned(csr);
}

static int spmv_checks(ciecu_csr csr, const void* in, const void* out, int valueType) {
    CIECU_REQUIRE(csr, "spmv: null matrix");
    CIECU_REQUIRE(csr->valueType == valueType, "spmv: matrix value type does not match the vector type");
    CIECU_REQUIRE((csr->rows == 0 || out) && (csr->cols == 0 || in), "spmv: null vector");
    return CIECU_OK;
}

int ciecu_csr_spmv_f64(ciecu_csr csr, double inScale, const double* d_in, double outScale, double* d_out) {
    CIECU_TRY(spmv_checks(csr, d_in, d_out, CIECU_F64));
    if (csr->rows == 0) return CIECU_OK;
    CIECU_TRY(ensure_tuned(csr));
    return launch_spmv<double>(csr, csr->kernel, nullptr, 0, inScale, d_in, outScale, d_out);
}

int ciecu_csr_spmv_f32(ciecu_csr csr, float inScale, const float* d_in, float outScale, float* d_out) {
    CIECU_TRY(spmv_checks(csr, d_in, d_out, CIECU_F32));
    if (csr->rows == 0) return CIECU_OK;
    CIECU_TRY(ensure_tuned(csr));
    return launch_spmv<float>(csr, csr->kernel, nullptr, 0, inScale, d_in, outScale, d_out);
}

int ciecu_csr_masked_spmv_f64(ciecu_csr csr, const uint16_t* d_mask, uint16_t threshold, double inScale,
                              const double* d_in, double outScale, double* d_out) {
    CIECU_TRY(spmv_checks(csr, d_in, d_out, CIECU_F64));
    CIECU_REQUIRE(d_mask, "masked_spmv: null mask");
    CIECU_REQUIRE(csr->rows == csr->cols, "masked_spmv: the mask indexes rows and columns, the matrix must be square");
    if (csr->rows == 0) return CIECU_OK;
    CIECU_TRY(ensure_tuned(csr));
    return launch_spmv<double>(csr, csr->kernel, d_mask, threshold, inScale, d_in, outScale, d_out);
}

}  // extern "C"
