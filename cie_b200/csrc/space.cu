// ciecu_space: stream, device memory, BLAS-1.
// Semantics of linalg/packages/solvers/src/DefaultSpace.cpp:50-187 and
// SYCLSpace.cpp:114-343; every op is one grid-stride kernel on the space's stream.
#include "space.cuh"

#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>

namespace ciecu {

std::atomic<long long> g_launches{0};

namespace {
thread_local std::string t_lastError;
}

void set_error(const std::string& message) { t_lastError = message; }

int fail(int status, const std::string& message) {
    t_lastError = message;
    return status;
}

int cuda_fail(cudaError_t error, const char* what) {
    t_lastError = std::string(what) + ": " + cudaGetErrorName(error) + " (" + cudaGetErrorString(error) + ")";
    return CIECU_ERR_CUDA;
}

int sm_count() {
    static int cached = [] {
        int device = 0, count = 0;
        if (cudaGetDevice(&device) != cudaSuccess) return kFallbackSMs;
        if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            return kFallbackSMs;
        return count > 0 ? count : kFallbackSMs;
    }();
    return cached;
}

namespace {
std::mutex g_poolMutex;
std::map<int, cudaMemPool_t> g_pools;

cudaError_t device_pool(cudaMemPool_t* pool) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_poolMutex);
    auto it = g_pools.find(device);
    if (it != g_pools.end()) {
        *pool = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t created = nullptr;
    e = cudaMemPoolCreate(&created, &props);
    if (e != cudaSuccess) return e;
    unsigned long long keep = kPoolKeepBytes;
    e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
        cudaMemPoolDestroy(created);
        return e;
    }
    g_pools[device] = created;
    *pool = created;
    return cudaSuccess;
}
}  // namespace

cudaError_t pool_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
    *ptr = nullptr;
    cudaMemPool_t pool = nullptr;
    const cudaError_t e = device_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(ptr, bytes == 0 ? 1 : bytes, pool, stream);
}

void pool_release(std::initializer_list<void*> ptrs) {
    bool any = false;
    for (void* p : ptrs) any = any || p;
    if (!any) return;
    cudaDeviceSynchronize();
    for (void* p : ptrs)
        if (p) cudaFreeAsync(p, cudaStreamLegacy);
    cudaStreamSynchronize(cudaStreamLegacy);  // the blocks are free for any stream from here
}

int resident_blocks(const void* kernel, int threads, size_t smem) {
    static std::mutex mutex;
    static std::map<std::tuple<const void*, int, size_t>, int> cache;
    const auto key = std::make_tuple(kernel, threads, smem);
    std::lock_guard<std::mutex> lock(mutex);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, threads, smem) != cudaSuccess || perSM < 1)
        perSM = 1;
    const int blocks = perSM * sm_count();
    cache[key] = blocks;
    return blocks;
}

// ---- kernels -----------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(kThreads) dot_kernel(long n, const T* __restrict__ a, const T* __restrict__ b,
                                                       double* partials, unsigned* counter, double* result) {
    double acc = 0.0;
    const long stride = static_cast<long>(gridDim.x) * kThreads;
    for (long i = static_cast<long>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
        acc = fma(static_cast<double>(a[i]), static_cast<double>(b[i]), acc);
    double mine[1] = {acc}, total[1];
    if (grid_reduce_last<1, kThreads>(mine, partials, counter, total) && threadIdx.x == 0) *result = total[0];
}

// t = alpha * t (.) s, special-cased like DefaultSpace::scale (:101-106)
template <typename T>
__global__ void scale_elementwise_kernel(long n, T* __restrict__ t, const T* __restrict__ s, T alpha) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const T l = t[i], r = s[i];
        t[i] = alpha == T(1) ? l * r : (alpha == T(-1) ? -l * r : alpha * l * r);
    }
}

template <typename T>
__global__ void scale_kernel(long n, T* __restrict__ v, T alpha) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) v[i] *= alpha;
}

// t = t + alpha * s, special-cased like DefaultSpace::add (:145-150)
template <typename T>
__global__ void add_kernel(long n, T* __restrict__ t, const T* __restrict__ s, T alpha) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const T l = t[i], r = s[i];
        t[i] = alpha == T(1) ? l + r : (alpha == T(-1) ? l - r : l + alpha * r);
    }
}

template <typename T>
__global__ void fill_kernel(long n, T* __restrict__ v, T value) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) v[i] = value;
}

template <typename TO, typename TI>
__global__ void convert_kernel(long n, TO* __restrict__ t, const TI* __restrict__ s) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        t[i] = static_cast<TO>(s[i]);
}

template <typename T>
int launch_dot(ciecu_space space, long n, const T* a, const T* b, double* d_result) {
    const int grid = dot_grid(n);
    dot_kernel<T><<<grid, kThreads, 0, space->stream>>>(n, a, b, space->d_partials, space->d_counter, d_result);
    count_launch();
    CIECU_CHECK_LAUNCH("dot_kernel");
    return CIECU_OK;
}

template int launch_dot<double>(ciecu_space, long, const double*, const double*, double*);
template int launch_dot<float>(ciecu_space, long, const float*, const float*, double*);

template <typename T>
int dot(ciecu_space space, int64_t n, const T* a, const T* b, double* h_result) {
    CIECU_REQUIRE(space && h_result && n >= 0, "dot: invalid arguments");
    if (n == 0) {
        *h_result = 0.0;
        return CIECU_OK;
    }
    CIECU_TRY(launch_dot(space, n, a, b, space->d_result));
    CIECU_CUDA(cudaMemcpyAsync(space->h_result, space->d_result, sizeof(double), cudaMemcpyDeviceToHost, space->stream));
    CIECU_CUDA(cudaStreamSynchronize(space->stream));
    *h_result = *space->h_result;
    return CIECU_OK;
}

template <typename Kernel, typename... Args>
int elementwise(ciecu_space space, int64_t n, const char* name, Kernel kernel, Args... args) {
    CIECU_REQUIRE(space && n >= 0, std::string(name) + ": invalid arguments");
    if (n == 0) return CIECU_OK;
    kernel<<<grid_for(n, kThreads, 8), kThreads, 0, space->stream>>>(static_cast<long>(n), args...);
    count_launch();
    CIECU_CHECK_LAUNCH(name);
    return CIECU_OK;
}

}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_last_error(char* h_buffer, int size) {
    const std::string& message = t_lastError;
    if (h_buffer && size > 0) {
        std::strncpy(h_buffer, message.c_str(), static_cast<size_t>(size) - 1);
        h_buffer[size - 1] = '\0';
    }
    return static_cast<int>(message.size());
}

int64_t ciecu_kernel_launch_count(void) { return g_launches.load(); }

int ciecu_device_info(int* smCount, int* ccMajor, int* ccMinor) {
    int device = 0;
    CIECU_CUDA(cudaGetDevice(&device));
    if (smCount) CIECU_CUDA(cudaDeviceGetAttribute(smCount, cudaDevAttrMultiProcessorCount, device));
    if (ccMajor) CIECU_CUDA(cudaDeviceGetAttribute(ccMajor, cudaDevAttrComputeCapabilityMajor, device));
    if (ccMinor) CIECU_CUDA(cudaDeviceGetAttribute(ccMinor, cudaDevAttrComputeCapabilityMinor, device));
    return CIECU_OK;
}

int ciecu_space_create(void* cudaStream, ciecu_space* out) {
    CIECU_REQUIRE(out, "space_create: null output");
    auto* space = new ciecu_space_s();
    int status = CIECU_OK;
    do {
        cudaError_t e = cudaGetDevice(&space->device);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaGetDevice"); break; }
        if (cudaStream) {
            space->stream = static_cast<cudaStream_t>(cudaStream);
        } else {
            e = cudaStreamCreateWithFlags(&space->stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) { status = cuda_fail(e, "cudaStreamCreate"); break; }
            space->ownsStream = true;
        }
        e = cudaMalloc(&space->d_partials, sizeof(double) * kMaxPartials * 4);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaMalloc(partials)"); break; }
        e = cudaMalloc(&space->d_counter, sizeof(unsigned) * 8);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaMalloc(counter)"); break; }
        e = cudaMemsetAsync(space->d_counter, 0, sizeof(unsigned) * 8, space->stream);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaMemset(counter)"); break; }
        e = cudaMalloc(&space->d_result, sizeof(double) * 8);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaMalloc(result)"); break; }
        e = cudaMallocHost(&space->h_result, sizeof(double) * 8);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaMallocHost(result)"); break; }
        e = cudaStreamSynchronize(space->stream);
        if (e != cudaSuccess) { status = cuda_fail(e, "space_create sync"); break; }
    } while (false);
    if (status != CIECU_OK) {
        ciecu_space_destroy(space);
        return status;
    }
    *out = space;
    return CIECU_OK;
}

int ciecu_space_destroy(ciecu_space space) {
    if (!space) return CIECU_OK;
    // Only a stream this space created is touched (a borrowed one may already be
    // gone); cudaFree synchronises the device.
    if (space->ownsStream && space->stream) cudaStreamSynchronize(space->stream);
    cudaFree(space->d_partials);
    cudaFree(space->d_counter);
    cudaFree(space->d_result);
    if (space->h_result) cudaFreeHost(space->h_result);
    if (space->ownsStream && space->stream) cudaStreamDestroy(space->stream);
    delete space;
    return CIECU_OK;
}

int ciecu_space_synchronize(ciecu_space space) {
    CIECU_REQUIRE(space, "space_synchronize: null space");
    CIECU_CUDA(cudaStreamSynchronize(space->stream));
    return CIECU_OK;
}

void* ciecu_space_stream(ciecu_space space) { return space ? space->stream : nullptr; }

int ciecu_alloc(ciecu_space space, size_t bytes, void** d_out) {
    CIECU_REQUIRE(space && d_out, "alloc: invalid arguments");
    *d_out = nullptr;
    if (bytes == 0) return CIECU_OK;
    CIECU_CUDA(cudaMalloc(d_out, bytes));
    return CIECU_OK;
}

int ciecu_free(ciecu_space space, void* d_ptr) {
    CIECU_REQUIRE(space, "free: null space");
    if (!d_ptr) return CIECU_OK;
    CIECU_CUDA(cudaStreamSynchronize(space->stream));
    CIECU_CUDA(cudaFree(d_ptr));
    return CIECU_OK;
}

int ciecu_memcpy_h2d(ciecu_space space, void* d_dst, const void* h_src, size_t bytes) {
    CIECU_REQUIRE(space, "memcpy_h2d: null space");
    if (bytes == 0) return CIECU_OK;
    CIECU_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, space->stream));
    CIECU_CUDA(cudaStreamSynchronize(space->stream));
    return CIECU_OK;
}

int ciecu_memcpy_d2h(ciecu_space space, void* h_dst, const void* d_src, size_t bytes) {
    CIECU_REQUIRE(space, "memcpy_d2h: null space");
    if (bytes == 0) return CIECU_OK;
    CIECU_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, space->stream));
    CIECU_CUDA(cudaStreamSynchronize(space->stream));
    return CIECU_OK;
}

int ciecu_memcpy_d2d(ciecu_space space, void* d_dst, const void* d_src, size_t bytes) {
    CIECU_REQUIRE(space, "memcpy_d2d: null space");
    if (bytes == 0) return CIECU_OK;
    CIECU_CUDA(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, space->stream));
    return CIECU_OK;
}

int ciecu_dot_f64(ciecu_space s, int64_t n, const double* a, const double* b, double* r) { return dot(s, n, a, b, r); }
int ciecu_dot_f32(ciecu_space s, int64_t n, const float* a, const float* b, double* r) { return dot(s, n, a, b, r); }

int ciecu_scale_elementwise_f64(ciecu_space s, int64_t n, double* t, const double* src, double alpha) {
    return elementwise(s, n, "scale_elementwise", scale_elementwise_kernel<double>, t, src, alpha);
}
int ciecu_scale_elementwise_f32(ciecu_space s, int64_t n, float* t, const float* src, float alpha) {
    return elementwise(s, n, "scale_elementwise", scale_elementwise_kernel<float>, t, src, alpha);
}
int ciecu_scale_f64(ciecu_space s, int64_t n, double* v, double alpha) {
    return elementwise(s, n, "scale", scale_kernel<double>, v, alpha);
}
int ciecu_scale_f32(ciecu_space s, int64_t n, float* v, float alpha) {
    return elementwise(s, n, "scale", scale_kernel<float>, v, alpha);
}
int ciecu_add_f64(ciecu_space s, int64_t n, double* t, const double* src, double alpha) {
    return elementwise(s, n, "add", add_kernel<double>, t, src, alpha);
}
int ciecu_add_f32(ciecu_space s, int64_t n, float* t, const float* src, float alpha) {
    return elementwise(s, n, "add", add_kernel<float>, t, src, alpha);
}
int ciecu_assign_f64(ciecu_space s, int64_t n, double* t, const double* src) {
    CIECU_REQUIRE(s && n >= 0, "assign: invalid arguments");
    return ciecu_memcpy_d2d(s, t, src, sizeof(double) * static_cast<size_t>(n));
}
int ciecu_assign_f32(ciecu_space s, int64_t n, float* t, const float* src) {
    CIECU_REQUIRE(s && n >= 0, "assign: invalid arguments");
    return ciecu_memcpy_d2d(s, t, src, sizeof(float) * static_cast<size_t>(n));
}
int ciecu_fill_f64(ciecu_space s, int64_t n, double* v, double value) {
    return elementwise(s, n, "fill", fill_kernel<double>, v, value);
}
int ciecu_fill_f32(ciecu_space s, int64_t n, float* v, float value) {
    return elementwise(s, n, "fill", fill_kernel<float>, v, value);
}
int ciecu_convert_f64_to_f32(ciecu_space s, int64_t n, float* t, const double* src) {
    return elementwise(s, n, "convert", convert_kernel<float, double>, t, src);
}
int ciecu_convert_f32_to_f64(ciecu_space s, int64_t n, double* t, const float* src) {
    return elementwise(s, n, "convert", convert_kernel<double, float>, t, src);
}

}  // extern "C"
