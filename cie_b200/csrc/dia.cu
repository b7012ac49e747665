// DIA copies of few-diagonal CSR matrices (dia.cuh): offset analysis and value
// fill.
#include "dia.cuh"
#include "space.cuh"

#include <algorithm>
#include <climits>

namespace ciecu {
namespace {

constexpr int kHashSlots = 128;  // power of two, > 2 * kMaxDiagonals
constexpr int kEmpty = INT_MIN;  // no offset c - r of an n < 2^31 matrix equals it

__device__ __forceinline__ unsigned hash_slot(int off) {
    return (static_cast<unsigned>(off) * 2654435761u) >> 25;  // top 7 bits
}

// Inserts every offset c - r into an open-addressing table (bounded probing).
// Sets *reject when the table is full, or when a row's columns are not strictly
// ascending (a DIA copy holds one entry per row and diagonal).
__global__ void dia_collect_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col, int* table,
                                   unsigned* reject) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int k1 = rowptr[r + 1];
        int prev = INT_MIN;
        for (int k = rowptr[r]; k < k1; ++k) {
            const int c = col[k];
            if (c <= prev) {
                atomicOr(reject, 1u);
                return;
            }
            prev = c;
            const int off = c - r;
            unsigned h = hash_slot(off);
            bool placed = false;
            for (int probe = 0; probe < kHashSlots; ++probe) {
                const int cur = *reinterpret_cast<volatile int*>(table + h);
                if (cur == off) {
                    placed = true;
                    break;
                }
                if (cur == kEmpty) {
                    const int was = atomicCAS(table + h, kEmpty, off);
                    if (was == kEmpty || was == off) {
                        placed = true;
                        break;
                    }
                }
                h = (h + 1) & (kHashSlots - 1);
            }
            if (!placed) {
                atomicOr(reject, 1u);
                return;
            }
        }
    }
}

template <typename V>
__global__ void dia_fill_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                const double* __restrict__ val, DiaArgs<V> a, V* __restrict__ out,
                                const double* __restrict__ sdiag) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int k1 = rowptr[r + 1];
        for (int k = rowptr[r]; k < k1; ++k) {
            const int c = col[k];
            const int off = c - r;
            int lo = 0, hi = a.ndiag - 1;  // the offset is in the table: the pattern was analysed
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (a.off[mid] < off) lo = mid + 1;
                else hi = mid;
            }
            if (a.off[lo] != off) continue;  // unreachable for the analysed pattern
            const double v = sdiag ? val[k] * sdiag[r] * sdiag[c] : val[k];
            out[static_cast<long>(lo) * a.ld + r] = static_cast<V>(v);
        }
    }
}

}  // namespace

int dia_offsets(ciecu_csr_s* csr, const std::vector<int>** out) {
    *out = &csr->diaOffsets;
    if (csr->diaState != 0) return CIECU_OK;
    csr->diaState = 2;
    csr->diaOffsets.clear();
    if (csr->rows != csr->cols || csr->rows == 0 || csr->nnz == 0) return CIECU_OK;
    cudaStream_t st = csr->space->stream;
    int* d_table = nullptr;
    CIECU_CUDA(pool_alloc(&d_table, sizeof(int) * (kHashSlots + 1), st));
    std::vector<int> h(kHashSlots + 1, kEmpty);
    h[kHashSlots] = 0;  // reject flag
    cudaError_t e = cudaMemcpyAsync(d_table, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        dia_collect_kernel<<<grid_for(csr->rows, 256, 8), 256, 0, st>>>(
            csr->rows, csr->rowptr, csr->col, d_table, reinterpret_cast<unsigned*>(d_table + kHashSlots));
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_table, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(d_table, st);  // back to the pool; the stream is idle here
    if (e != cudaSuccess) return cuda_fail(e, "dia: offset analysis");
    if (h[kHashSlots] != 0) return CIECU_OK;
    std::vector<int> offsets;
    for (int i = 0; i < kHashSlots; ++i)
        if (h[i] != kEmpty) offsets.push_back(h[i]);
    if (offsets.empty() || offsets.size() > static_cast<size_t>(kMaxDiagonals)) return CIECU_OK;
    const double fill = static_cast<double>(csr->nnz) / (static_cast<double>(offsets.size()) * csr->rows);
    if (fill < 0.6) return CIECU_OK;
    std::sort(offsets.begin(), offsets.end());
    csr->diaOffsets = offsets;
    csr->diaState = 1;
    return CIECU_OK;
}

int dia_fill_f64(const ciecu_csr_s* csr, const DiaArgs<double>& a, double* out, cudaStream_t st) {
    dia_fill_kernel<double><<<grid_for(csr->rows, 256, 8), 256, 0, st>>>(
        csr->rows, csr->rowptr, csr->col, static_cast<const double*>(csr->val), a, out, nullptr);
    count_launch();
    CIECU_CHECK_LAUNCH("dia_fill_kernel<double>");
    return CIECU_OK;
}

int dia_fill_f32(const ciecu_csr_s* csr, const DiaArgs<float>& a, float* out, const double* sdiag, cudaStream_t st) {
    dia_fill_kernel<float><<<grid_for(csr->rows, 256, 8), 256, 0, st>>>(
        csr->rows, csr->rowptr, csr->col, static_cast<const double*>(csr->val), a, out, sdiag);
    count_launch();
    CIECU_CHECK_LAUNCH("dia_fill_kernel<float>");
    return CIECU_OK;
}

// Counts the stored pairs (r, r + o), o > 0, whose mirror (r + o, r) differs in
// any bit: diagonal d (offset o) at row r against diagonal m (offset -o) at row
// r + o.
template <typename V>
__global__ void dia_symmetry_kernel(DiaArgs<V> a, unsigned* bad) {
    const int half = a.ndiag / 2;
    for (int k = 1; k <= half; ++k) {
        const int d = half + k, m = half - k;
        const int o = a.off[d];
        const V* up = a.val + static_cast<long>(d) * a.ld;
        const V* lo = a.val + static_cast<long>(m) * a.ld;
        for (long r = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; r + o < a.nrows;
             r += static_cast<long>(gridDim.x) * blockDim.x) {
            const bool same = sizeof(V) == 8 ? __double_as_longlong(static_cast<double>(up[r])) ==
                                                   __double_as_longlong(static_cast<double>(lo[r + o]))
                                             : __float_as_uint(static_cast<float>(up[r])) ==
                                                   __float_as_uint(static_cast<float>(lo[r + o]));
            if (!same) atomicAdd(bad, 1u);
        }
    }
}

template <typename V>
int dia_symmetric(const DiaArgs<V>& full, cudaStream_t st, unsigned* d_flag, bool* symmetric) {
    *symmetric = false;
    const int nd = full.ndiag;
    if (nd < 3 || nd % 2 == 0 || full.off[nd / 2] != 0) return CIECU_OK;
    for (int k = 1; k <= nd / 2; ++k)
        if (full.off[nd / 2 + k] != -full.off[nd / 2 - k]) return CIECU_OK;
    unsigned bad = 0;
    CIECU_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(unsigned), st));
    dia_symmetry_kernel<V><<<grid_for(full.nrows, 256, 8), 256, 0, st>>>(full, d_flag);
    count_launch();
    CIECU_CHECK_LAUNCH("dia_symmetry_kernel");
    CIECU_CUDA(cudaMemcpyAsync(&bad, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CIECU_CUDA(cudaStreamSynchronize(st));
    *symmetric = bad == 0;
    return CIECU_OK;
}
template int dia_symmetric<float>(const DiaArgs<float>&, cudaStream_t, unsigned*, bool*);
template int dia_symmetric<double>(const DiaArgs<double>&, cudaStream_t, unsigned*, bool*);

}  // namespace ciecu

extern "C" int ciecu_csr_diagonals(ciecu_csr csr, int* ndiag) {
    CIECU_REQUIRE(csr && ndiag, "csr_diagonals: null argument");
    const std::vector<int>* offsets = nullptr;
    CIECU_TRY(ciecu::dia_offsets(csr, &offsets));
    *ndiag = static_cast<int>(offsets->size());
    return CIECU_OK;
}
