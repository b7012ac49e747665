// Diagonal operator, damped Jacobi, masked identity, Chebyshev smoother and the
// power iteration that bounds its spectrum.
//   makeDiagonalOperator / DiagonalOperator::product   linalg/packages/solvers/src/DiagonalOperator.cpp:37-88
//   JacobiOperator::product                            linalg/packages/solvers/src/JacobiOperator.cpp:36-62
//   MaskedIdentityOperator::product                    linalg/packages/solvers/src/MaskedIdentityOperator.cpp:14-74
// Each Jacobi / Chebyshev sweep is ONE kernel: the CSR row pass computes A x for
// the row and the epilogue applies the update, ping-ponging the iterate.
#include "spmv.cuh"
#include "space.cuh"

#include <cuda.h>

#include <mutex>
#include <string>

// Scratch of ciecu_jacobi_f64_static: the two Jacobi iterates of a matrix of at
// most CIECU_JACOBI_STATIC_MAX_ROWS rows (2 x 262144 doubles = 4 MiB), part of
// this library's device image, so using it needs no allocation.  One array per
// device, shared by every call on that device.
static __device__ __align__(256) double g_jacobiStaticScratch[2 * CIECU_JACOBI_STATIC_MAX_ROWS];

namespace ciecu {
namespace {

constexpr int kT = 256;

struct DiagError {
    int missingRow;
    int zeroRow;
};

// First diagonal entry of each row by linear scan (the CPU semantics of
// makeDiagonalOperator); failures are recorded as the smallest offending row.
__global__ void diag_inverse_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                    const double* __restrict__ val, double* __restrict__ dinv, DiagError* err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int k = rowptr[i];
        const int k1 = rowptr[i + 1];
        for (; k < k1; ++k)
            if (col[k] == i) break;
        if (k == k1) {
            atomicMin(&err->missingRow, i);
        } else if (val[k] == 0.0) {
            atomicMin(&err->zeroRow, i);
        } else {
            dinv[i] = 1.0 / val[k];
        }
    }
}

// DiagonalOperator::product: inScale == 0 -> out = in (.) D^-1 scaled by outScale;
// otherwise buffer = (in (.) D^-1) * outScale; out = inScale*out + buffer.
__global__ void diag_apply_kernel(long n, const double* __restrict__ dinv, double inScale,
                                  const double* __restrict__ in, double outScale, double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        // scale(t, s, a): a == 1 -> t*s; a == -1 -> -t*s; else a*t*s
        const double l = in[i], r = dinv[i];
        const double b = outScale == 1.0 ? l * r : (outScale == -1.0 ? -l * r : outScale * l * r);
        if (inScale == 0.0) {
            out[i] = b;
        } else {
            const double o = inScale == 1.0 ? out[i] : out[i] * inScale;
            out[i] = o + b;
        }
    }
}

__global__ void masked_identity_kernel(long n, const uint16_t* __restrict__ mask, uint16_t threshold,
                                       double inScale, const double* __restrict__ in, double outScale,
                                       double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = mask[i] < threshold ? in[i] : 0.0;
        out[i] = combine(inScale, out[i], outScale, v);
    }
}

// First Jacobi sweep from x0 = 0: A x0 = 0, so x1 = (w in) D^-1.
__global__ void jacobi_first_kernel(long n, const double* __restrict__ in, const double* __restrict__ dinv,
                                    double w, double* __restrict__ x) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double res = in[i] - 0.0;
        const double t = w == 1.0 ? res * dinv[i] : (w == -1.0 ? -res * dinv[i] : w * res * dinv[i]);
        x[i] = 0.0 + t;
    }
}

// One sweep: res = in - A x_old; x_new = x_old + (w res) D^-1.
struct JacobiOp {
    struct Pre {
        double in, d, xo;
    };
    const double* __restrict__ in;
    const double* __restrict__ dinv;
    const double* __restrict__ xold;
    double* __restrict__ xnew;
    double w;
    __device__ __forceinline__ Pre pre(int r) const { return Pre{in[r], dinv[r], xold[r]}; }
    __device__ __forceinline__ void post(int r, const Pre& p, double sum) const {
        const double res = p.in - sum;
        const double t = w == 1.0 ? res * p.d : (w == -1.0 ? -res * p.d : w * res * p.d);
        xnew[r] = p.xo + t;
    }
};

template <int KERNEL, bool MASKED>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    jacobi_sweep_kernel(CsrArgs<double> A, const double* __restrict__ in, const double* __restrict__ dinv, double w,
                        const double* __restrict__ xold, double* __restrict__ xnew) {
    JacobiOp op{in, dinv, xold, xnew, w};
    csr_rows<KERNEL, double, double, MASKED>(A, xold, op);
}

// out = x*outScale, then out += inScale*memory (scale(out,outScale); add(out,memory,inScale)).
__global__ void jacobi_output_kernel(long n, const double* __restrict__ x, double inScale, double outScale,
                                     double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double memory = out[i];
        const double sx = x[i] * outScale;
        out[i] = inScale == 1.0 ? sx + memory : (inScale == -1.0 ? sx - memory : sx + inScale * memory);
    }
}

// Chebyshev: d0 = D^-1 r0 / theta, x = d0.
__global__ void cheb_first_kernel(long n, const double* __restrict__ in, const double* __restrict__ dinv,
                                  double theta, double* __restrict__ r, double* __restrict__ d,
                                  double* __restrict__ x) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double ri = in[i];
        r[i] = ri;
        const double di = dinv[i] * ri / theta;
        d[i] = di;
        x[i] = 0.0 + di;
    }
}

// Chebyshev step: r -= A d_old; d_new = c1 d_old + c2 D^-1 r; x += d_new.
struct ChebOp {
    struct Pre {
        double r, d, dinv, x;
    };
    const double* __restrict__ dinv;
    double c1, c2;
    double* __restrict__ r;
    const double* __restrict__ dold;
    double* __restrict__ dnew;
    double* __restrict__ x;
    __device__ __forceinline__ Pre pre(int i) const { return Pre{r[i], dold[i], dinv[i], x[i]}; }
    __device__ __forceinline__ void post(int i, const Pre& p, double sum) const {
        const double ri = p.r - sum;
        r[i] = ri;
        const double di = c1 * p.d + c2 * p.dinv * ri;
        dnew[i] = di;
        x[i] = p.x + di;
    }
};

template <int KERNEL>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    cheb_step_kernel(CsrArgs<double> A, const double* __restrict__ dinv, double c1, double c2,
                     double* __restrict__ r, const double* __restrict__ dold, double* __restrict__ dnew,
                     double* __restrict__ x) {
    ChebOp op{dinv, c1, c2, r, dold, dnew, x};
    csr_rows<KERNEL, double, double, false>(A, dold, op);
}

__global__ void combine_kernel(long n, double inScale, const double* __restrict__ v, double outScale,
                               double* __restrict__ out) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = combine(inScale, out[i], outScale, v[i]);
}

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t index) {
    uint64_t z = seed + (index + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void power_init_kernel(long n, uint64_t seed, double* __restrict__ v) {
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        v[i] = static_cast<double>(splitmix_at(seed, static_cast<uint64_t>(i)) >> 11) * 0x1.0p-53 + 0.5;
}

// v <- v / ||v|| with the norm read from the device.
__global__ void power_normalize_kernel(long n, double* __restrict__ v, const double* __restrict__ norm2) {
    const double inv = 1.0 / sqrt(*norm2);
    const long stride = static_cast<long>(gridDim.x) * blockDim.x;
    for (long i = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) v[i] *= inv;
}

struct PowerOp {
    using Pre = double;
    const double* __restrict__ dinv;
    double* __restrict__ w;
    __device__ __forceinline__ double pre(int i) const { return dinv[i]; }
    __device__ __forceinline__ void post(int i, double d, double sum) const { w[i] = sum * d; }
};

template <int KERNEL>
__global__ void __launch_bounds__(csr_threads<KERNEL>())
    power_apply_kernel(CsrArgs<double> A, const double* __restrict__ dinv, const double* __restrict__ v,
                       double* __restrict__ w) {
    PowerOp op{dinv, w};
    csr_rows<KERNEL, double, double, false>(A, v, op);
}

// Device address of g_jacobiStaticScratch on `device` (which must be current),
// looked up on the first call for that device and remembered together with the
// identity of the current context.  A reset of the device (cudaDeviceReset or a
// primary-context reset) loads the library's device image again, possibly at
// another address; the new context has another identity, so the address is
// looked up again.  Allocates nothing.
constexpr int kStaticScratchDevices = 64;

// The two driver calls are fetched through the runtime, so the library keeps no
// link-time dependency on the driver library.
int current_context_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent getCurrent = nullptr;
    static GetId getId = nullptr;
    *id = 0;
    if (!getCurrent || !getId) {
        void* f = nullptr;
        void* g = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) != cudaSuccess || !f ||
            cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, nullptr) != cudaSuccess || !g)
            return 0;
        getCurrent = reinterpret_cast<GetCurrent>(f);
        getId = reinterpret_cast<GetId>(g);
    }
    CUcontext ctx = nullptr;
    if (getCurrent(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    return getId(ctx, id) == CUDA_SUCCESS ? 1 : 0;
}

int jacobi_static_scratch(int device, double** out) {
    struct Entry {
        unsigned long long context;
        double* address;
    };
    static std::mutex mutex;
    static Entry table[kStaticScratchDevices] = {};
    if (device < 0 || device >= kStaticScratchDevices)
        return fail(CIECU_ERR_ARGUMENT, "jacobi_f64_static: device ordinal " + std::to_string(device) +
                                            " is beyond the " + std::to_string(kStaticScratchDevices) +
                                            " devices this entry point supports");
    std::lock_guard<std::mutex> lock(mutex);
    unsigned long long context = 0;
    const int known = current_context_id(&context);
    if (!table[device].address || !known || table[device].context != context) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_jacobiStaticScratch);
        if (e != cudaSuccess) return cuda_fail(e, "jacobi_f64_static: cudaGetSymbolAddress(static scratch)");
        current_context_id(&context);  // the lookup made the device's context current
        table[device] = Entry{context, static_cast<double*>(p)};
    }
    *out = table[device].address;
    return CIECU_OK;
}

// Row schedule for a matrix whose SpMV schedule was never tuned (tuning
// allocates): lanes per row from the mean row length.
int untuned_schedule(const ciecu_csr_s* csr) {
    const double avg = csr->rows > 0 ? static_cast<double>(csr->nnz) / csr->rows : 0.0;
    return avg < 6.0 ? 2 : avg < 12.0 ? 4 : avg < 24.0 ? 8 : avg < 48.0 ? 16 : 32;
}

}  // namespace
}  // namespace ciecu

using namespace ciecu;

extern "C" {

int ciecu_diagonal_inverse_f64(ciecu_csr csr, double* d_inverse) {
    CIECU_REQUIRE(csr && (csr->rows == 0 || d_inverse), "diagonal_inverse: null argument");
    CIECU_REQUIRE(csr->valueType == CIECU_F64, "diagonal_inverse: FP64 matrix expected");
    if (csr->rows == 0) return CIECU_OK;
    cudaStream_t st = csr->space->stream;
    DiagError* d_err = reinterpret_cast<DiagError*>(csr->space->d_result);
    DiagError init{0x7fffffff, 0x7fffffff};
    CIECU_CUDA(cudaMemcpyAsync(d_err, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    diag_inverse_kernel<<<grid_for(csr->rows, kT, 8), kT, 0, st>>>(
        csr->rows, csr->rowptr, csr->col, static_cast<const double*>(csr->val), d_inverse, d_err);
    count_launch();
    CIECU_CHECK_LAUNCH("diag_inverse_kernel");
    DiagError err{};
    CIECU_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    if (err.missingRow != 0x7fffffff || err.zeroRow != 0x7fffffff) {
        if (err.zeroRow < err.missingRow)
            return fail(CIECU_ERR_DIAGONAL, "row " + std::to_string(err.zeroRow) + " has an explicit zero on its diagonal");
        return fail(CIECU_ERR_DIAGONAL, "row " + std::to_string(err.missingRow) + " has no diagonal entry");
    }
    return CIECU_OK;
}

int ciecu_diagonal_apply_f64(ciecu_space space, int64_t n, const double* d_inverse, double inScale, const double* d_in,
                             double outScale, double* d_out) {
    CIECU_REQUIRE(space && n >= 0, "diagonal_apply: invalid arguments");
    if (n == 0) return CIECU_OK;
    diag_apply_kernel<<<grid_for(n, kT, 8), kT, 0, space->stream>>>(n, d_inverse, inScale, d_in, outScale, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("diag_apply_kernel");
    return CIECU_OK;
}

int ciecu_masked_identity_f64(ciecu_space space, int64_t n, const uint16_t* d_mask, uint16_t threshold, double inScale,
                              const double* d_in, double outScale, double* d_out) {
    CIECU_REQUIRE(space && n >= 0 && (n == 0 || (d_mask && d_in && d_out)), "masked_identity: invalid arguments");
    if (n == 0) return CIECU_OK;
    masked_identity_kernel<<<grid_for(n, kT, 8), kT, 0, space->stream>>>(n, d_mask, threshold, inScale, d_in,
                                                                          outScale, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("masked_identity_kernel");
    return CIECU_OK;
}

int ciecu_jacobi_f64(ciecu_csr csr, const double* d_inverse, const uint16_t* d_mask, uint16_t threshold,
                     int64_t iterations, double relaxation, double inScale, const double* d_in, double outScale,
                     double* d_out, double* d_work) {
    CIECU_REQUIRE(csr && csr->valueType == CIECU_F64, "jacobi: FP64 matrix expected");
    CIECU_REQUIRE(csr->rows == csr->cols, "inconsistent input vector sizes");
    CIECU_REQUIRE(iterations >= 0, "jacobi: negative iteration count");
    const long n = csr->rows;
    if (n == 0) return CIECU_OK;
    CIECU_REQUIRE(d_inverse && d_in && d_out && d_work, "jacobi: null vector");
    CIECU_TRY(ensure_tuned(csr));
    cudaStream_t st = csr->space->stream;
    double* xa = d_work;
    double* xb = d_work + n;
    const int gridV = grid_for(n, kT, 8);
    if (iterations == 0) {
        CIECU_CUDA(cudaMemsetAsync(xa, 0, sizeof(double) * n, st));
    } else {
        jacobi_first_kernel<<<gridV, kT, 0, st>>>(n, d_in, d_inverse, relaxation, xa);
        count_launch();
        const int grid = csr_grid(csr, csr->kernel);
        for (int64_t s = 1; s < iterations; ++s) {
            CIECU_TRY(with_schedule(csr->kernel, [&](auto k) -> int {
                constexpr int K = decltype(k)::value;
                if (d_mask)
                    jacobi_sweep_kernel<K, true><<<fit_grid(jacobi_sweep_kernel<K, true>, csr_threads<K>(), grid),
                                                   csr_threads<K>(), 0, st>>>(
                        csr->args<double>(d_mask, threshold), d_in, d_inverse, relaxation, xa, xb);
                else
                    jacobi_sweep_kernel<K, false><<<fit_grid(jacobi_sweep_kernel<K, false>, csr_threads<K>(), grid),
                                                    csr_threads<K>(), 0, st>>>(
                        csr->args<double>(), d_in, d_inverse, relaxation, xa, xb);
                return CIECU_OK;
            }));
            count_launch();
            std::swap(xa, xb);
        }
    }
    jacobi_output_kernel<<<gridV, kT, 0, st>>>(n, xa, inScale, outScale, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("jacobi");
    return CIECU_OK;
}

int ciecu_chebyshev_f64(ciecu_csr csr, const double* d_inverse, int degree, double lambdaMin, double lambdaMax,
                        double inScale, const double* d_in, double outScale, double* d_out, double* d_work) {
    CIECU_REQUIRE(csr && csr->valueType == CIECU_F64 && csr->rows == csr->cols, "chebyshev: square FP64 matrix expected");
    CIECU_REQUIRE(degree >= 1, "chebyshev: degree must be at least 1");
    CIECU_REQUIRE(lambdaMax > lambdaMin && lambdaMin > 0.0, "chebyshev: need 0 < lambdaMin < lambdaMax");
    const long n = csr->rows;
    if (n == 0) return CIECU_OK;
    CIECU_REQUIRE(d_inverse && d_in && d_out && d_work, "chebyshev: null vector");
    CIECU_TRY(ensure_tuned(csr));
    cudaStream_t st = csr->space->stream;
    double* r = d_work;
    double* da = d_work + n;
    double* db = d_work + 2 * n;
    double* x = d_work + 3 * n;
    const double theta = 0.5 * (lambdaMax + lambdaMin);
    const double delta = 0.5 * (lambdaMax - lambdaMin);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    const int gridV = grid_for(n, kT, 8);
    cheb_first_kernel<<<gridV, kT, 0, st>>>(n, d_in, d_inverse, theta, r, da, x);
    count_launch();
    const int grid = csr_grid(csr, csr->kernel);
    for (int k = 1; k < degree; ++k) {
        const double rhoNew = 1.0 / (2.0 * sigma - rho);
        const double c1 = rhoNew * rho;
        const double c2 = 2.0 * rhoNew / delta;
        CIECU_TRY(with_schedule(csr->kernel, [&](auto kk) -> int {
            constexpr int K = decltype(kk)::value;
            cheb_step_kernel<K><<<fit_grid(cheb_step_kernel<K>, csr_threads<K>(), grid), csr_threads<K>(), 0, st>>>(csr->args<double>(), d_inverse, c1, c2, r, da, db, x);
            return CIECU_OK;
        }));
        count_launch();
        std::swap(da, db);
        rho = rhoNew;
    }
    combine_kernel<<<gridV, kT, 0, st>>>(n, inScale, x, outScale, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("chebyshev");
    return CIECU_OK;
}

int ciecu_power_lambda_max_f64(ciecu_csr csr, const double* d_inverse, int iterations, uint64_t seed, double* d_work,
                               double* h_lambda) {
    CIECU_REQUIRE(csr && csr->valueType == CIECU_F64 && csr->rows == csr->cols, "power: square FP64 matrix expected");
    CIECU_REQUIRE(iterations >= 1 && h_lambda && d_work && d_inverse, "power: invalid arguments");
    const long n = csr->rows;
    if (n == 0) {
        *h_lambda = 0.0;
        return CIECU_OK;
    }
    CIECU_TRY(ensure_tuned(csr));
    ciecu_space space = csr->space;
    cudaStream_t st = space->stream;
    double* v = d_work;
    double* w = d_work + n;
    const int gridV = grid_for(n, kT, 8);
    const int grid = csr_grid(csr, csr->kernel);
    power_init_kernel<<<gridV, kT, 0, st>>>(n, seed, v);
    count_launch();
    for (int it = 0; it < iterations; ++it) {
        CIECU_TRY(launch_dot<double>(space, n, v, v, space->d_result + 2));
        power_normalize_kernel<<<gridV, kT, 0, st>>>(n, v, space->d_result + 2);
        count_launch();
        CIECU_TRY(with_schedule(csr->kernel, [&](auto kk) -> int {
            constexpr int K = decltype(kk)::value;
            power_apply_kernel<K><<<fit_grid(power_apply_kernel<K>, csr_threads<K>(), grid), csr_threads<K>(), 0, st>>>(csr->args<double>(), d_inverse, v, w);
            return CIECU_OK;
        }));
        count_launch();
        CIECU_TRY(launch_dot<double>(space, n, v, w, space->d_result + 3));
        CIECU_CUDA(cudaMemcpyAsync(v, w, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    CIECU_CUDA(cudaMemcpyAsync(space->h_result + 3, space->d_result + 3, sizeof(double), cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    *h_lambda = space->h_result[3];
    CIECU_CHECK_LAUNCH("power");
    return CIECU_OK;
}

int ciecu_jacobi_f64_static(ciecu_csr csr, const double* d_inverse, const uint16_t* d_mask, uint16_t threshold,
                            int64_t iterations, double relaxation, double inScale, const double* d_in,
                            double outScale, double* d_out) {
    CIECU_REQUIRE(csr && csr->valueType == CIECU_F64, "jacobi_f64_static: FP64 matrix expected");
    CIECU_REQUIRE(csr->rows == csr->cols, "inconsistent input vector sizes");
    CIECU_REQUIRE(iterations >= 0, "jacobi_f64_static: negative iteration count");
    const long n = csr->rows;
    if (n > CIECU_JACOBI_STATIC_MAX_ROWS)
        return fail(CIECU_ERR_ARGUMENT, "jacobi_f64_static: " + std::to_string(n) +
                                            " rows exceed the static scratch of " +
                                            std::to_string(CIECU_JACOBI_STATIC_MAX_ROWS) +
                                            " rows; use ciecu_jacobi_f64 with caller-provided scratch");
    if (n == 0) return CIECU_OK;
    CIECU_REQUIRE(d_inverse && d_in && d_out, "jacobi_f64_static: null vector");
    int device = -1;
    CIECU_CUDA(cudaGetDevice(&device));
    CIECU_REQUIRE(device == csr->space->device, "jacobi_f64_static: the matrix's device must be the current device");
    double* scratch = nullptr;
    CIECU_TRY(jacobi_static_scratch(device, &scratch));
    cudaStream_t st = csr->space->stream;
    double* xa = scratch;
    double* xb = scratch + n;
    const int gridV = grid_for(n, kT, 8);
    if (iterations == 0) {
        CIECU_CUDA(cudaMemsetAsync(xa, 0, sizeof(double) * n, st));
    } else {
        jacobi_first_kernel<<<gridV, kT, 0, st>>>(n, d_in, d_inverse, relaxation, xa);
        count_launch();
        const int schedule = csr->kernel != 0 ? csr->kernel : untuned_schedule(csr);
        for (int64_t s = 1; s < iterations; ++s) {
            CIECU_TRY(with_schedule(schedule, [&](auto k) -> int {
                constexpr int K = decltype(k)::value;
                // no occupancy query: a fixed multiple of the SM count (the row
                // passes stride over the grid, so any grid size is correct)
                const long cap = static_cast<long>(sm_count()) * (2048 / csr_threads<K>());
                const int grid = static_cast<int>(std::min<long>(csr_grid(csr, K), cap));
                if (d_mask)
                    jacobi_sweep_kernel<K, true><<<grid, csr_threads<K>(), 0, st>>>(
                        csr->args<double>(d_mask, threshold), d_in, d_inverse, relaxation, xa, xb);
                else
                    jacobi_sweep_kernel<K, false><<<grid, csr_threads<K>(), 0, st>>>(
                        csr->args<double>(), d_in, d_inverse, relaxation, xa, xb);
                return CIECU_OK;
            }));
            count_launch();
            std::swap(xa, xb);
        }
    }
    jacobi_output_kernel<<<gridV, kT, 0, st>>>(n, xa, inScale, outScale, d_out);
    count_launch();
    CIECU_CHECK_LAUNCH("jacobi_f64_static");
    return CIECU_OK;
}

}  // extern "C"
