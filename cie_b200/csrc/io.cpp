// MatrixMarket output of the linear system (cieutils/packages/io/src/MatrixMarket.cpp):
// the same text as the reference's stream writer, formatted in parallel.  A double
// printed by a C++ stream with the default flags and precision is printf "%g"
// (six significant digits), and an integer its decimal form, so each line is
// produced with snprintf into per-chunk buffers that are written in row order.
#include "ciecu_io.h"
#include "spmv.cuh"
#include "space.cuh"

#include <algorithm>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

namespace ciecu {
void set_error(const std::string& message);
int fail(int status, const std::string& message);
}  // namespace ciecu

namespace {

// Formats rows [a, b) of the CSR arrays into `out`.
void format_rows(int64_t a, int64_t b, const int32_t* rp, const int32_t* col, const double* val, std::string& out) {
    char line[96];
    for (int64_t i = a; i < b; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int len = std::snprintf(line, sizeof(line), "%lld %lld %g\n", static_cast<long long>(i + 1),
                                          static_cast<long long>(col[k]) + 1, val[k]);
            out.append(line, static_cast<size_t>(len));
        }
}

void format_values(int64_t a, int64_t b, const double* v, std::string& out) {
    char line[64];
    for (int64_t i = a; i < b; ++i) {
        const int len = std::snprintf(line, sizeof(line), "%g\n", v[i]);
        out.append(line, static_cast<size_t>(len));
    }
}

// Splits [0, n) into chunks, formats them on the host threads, writes in order.
template <typename F>
int write_chunked(std::FILE* f, int64_t n, int64_t weight, F&& format) {
    const unsigned threads = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const int64_t chunks = n <= 0 ? 0 : std::min<int64_t>(n, std::max<int64_t>(1, weight / 200000) * threads);
    std::vector<std::string> text(static_cast<size_t>(std::max<int64_t>(chunks, 1)));
    // rounds of `threads` chunks, each round written before the next is formatted
    for (int64_t first = 0; first < chunks; first += threads) {
        const int64_t last = std::min<int64_t>(chunks, first + threads);
        std::vector<std::thread> pool;
        for (int64_t c = first; c < last; ++c)
            pool.emplace_back([&, c] {
                text[c].clear();
                format(n * c / chunks, n * (c + 1) / chunks, text[c]);
            });
        for (auto& t : pool) t.join();
        for (int64_t c = first; c < last; ++c) {
            if (std::fwrite(text[c].data(), 1, text[c].size(), f) != text[c].size()) return 1;
            std::string().swap(text[c]);
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int ciecu_write_matrix_market_host(const char* path, int64_t rows, int64_t columns, const int32_t* h_rowExtents,
                                   const int32_t* h_columnIndices, const double* h_entries) {
    if (!path || rows < 0 || columns < 0 || !h_rowExtents)
        return ciecu::fail(CIECU_ERR_ARGUMENT, "write_matrix_market: invalid arguments");
    const int64_t nnz = h_rowExtents[rows];
    if (nnz > 0 && (!h_columnIndices || !h_entries))
        return ciecu::fail(CIECU_ERR_ARGUMENT, "write_matrix_market: null CSR arrays");
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return ciecu::fail(CIECU_ERR_ARGUMENT, std::string("write_matrix_market: cannot open ") + path);
    int bad = std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n",
                           static_cast<long long>(rows), static_cast<long long>(columns),
                           static_cast<long long>(nnz)) < 0;
    if (!bad)
        bad = write_chunked(f, rows, nnz, [&](int64_t a, int64_t b, std::string& out) {
            format_rows(a, b, h_rowExtents, h_columnIndices, h_entries, out);
        });
    bad |= std::fclose(f) != 0;
    return bad ? ciecu::fail(CIECU_ERR_ARGUMENT, std::string("write_matrix_market: write failed: ") + path) : CIECU_OK;
}

int ciecu_write_matrix_market_vector_host(const char* path, int64_t n, const double* h_values) {
    if (!path || n < 0 || (n > 0 && !h_values))
        return ciecu::fail(CIECU_ERR_ARGUMENT, "write_matrix_market_vector: invalid arguments");
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return ciecu::fail(CIECU_ERR_ARGUMENT, std::string("write_matrix_market_vector: cannot open ") + path);
    int bad = std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%lld 1\n", static_cast<long long>(n)) < 0;
    if (!bad)
        bad = write_chunked(f, n, n, [&](int64_t a, int64_t b, std::string& out) { format_values(a, b, h_values, out); });
    bad |= std::fclose(f) != 0;
    return bad ? ciecu::fail(CIECU_ERR_ARGUMENT, std::string("write_matrix_market_vector: write failed: ") + path)
               : CIECU_OK;
}

int ciecu_write_matrix_market(ciecu_csr csr, const char* path) {
    CIECU_REQUIRE(csr && path, "write_matrix_market: null argument");
    CIECU_REQUIRE(csr->valueType == CIECU_F64, "write_matrix_market: FP64 matrix expected");
    cudaStream_t st = csr->space->stream;
    std::vector<int32_t> rp(static_cast<size_t>(csr->rows) + 1), col(static_cast<size_t>(csr->nnz));
    std::vector<double> val(static_cast<size_t>(csr->nnz));
    CIECU_CUDA(cudaMemcpyAsync(rp.data(), csr->rowptr, sizeof(int32_t) * rp.size(), cudaMemcpyDeviceToHost, st));
    if (csr->nnz > 0) {
        CIECU_CUDA(cudaMemcpyAsync(col.data(), csr->col, sizeof(int32_t) * col.size(), cudaMemcpyDeviceToHost, st));
        CIECU_CUDA(cudaMemcpyAsync(val.data(), csr->val, sizeof(double) * val.size(), cudaMemcpyDeviceToHost, st));
    }
    CIECU_CUDA(cudaStreamSynchronize(st));
    return ciecu_write_matrix_market_host(path, csr->rows, csr->cols, rp.data(), col.data(), val.data());
}

int ciecu_write_matrix_market_vector(ciecu_space space, int64_t n, const double* d_values, const char* path) {
    CIECU_REQUIRE(space && path && n >= 0 && (n == 0 || d_values), "write_matrix_market_vector: invalid arguments");
    std::vector<double> v(static_cast<size_t>(n));
    if (n > 0) {
        CIECU_CUDA(cudaMemcpyAsync(v.data(), d_values, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, space->stream));
        CIECU_CUDA(cudaStreamSynchronize(space->stream));
    }
    return ciecu_write_matrix_market_vector_host(path, n, v.data());
}

}  // extern "C"
