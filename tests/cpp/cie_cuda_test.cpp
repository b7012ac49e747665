// Test program of the C++ host API (include/cie_cuda/linalg.hpp), written the way
// the reference's own driver uses its SYCL backend (executables/fem_examples/src/
// poisson2D/solver.cpp:238-288): matrix and vectors copied to the device through
// the space, a CSR operator, makeDiagonalOperator, ConjugateGradients.
// Results are checked against the C restatement in oracle/ (test infrastructure).
// Prints one line per check and "ALL OK" at the end; exit status 1 on a failure.
#include "cie_cuda/linalg.hpp"

#include "../../oracle/restate.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#ifdef CIE_CUDA_WITH_CIE_LINALG
#include "packages/solvers/inc/LinalgSpace.hpp"
static_assert(cie::linalg::LinalgSpaceLike<cie::cuda::CUDASpace<double>>);
static_assert(cie::linalg::LinalgSpaceLike<cie::cuda::CUDASpace<float>>);
#endif

namespace {

using namespace cie::cuda;
using Space = CUDASpace<double>;

int g_failures = 0;

void report(bool ok, const char* what, double value) {
    std::printf("%s %-58s %.3e\n", ok ? "ok  " : "FAIL", what, value);
    if (!ok) ++g_failures;
}

struct HostCSR {
    int n = 0;
    std::vector<int> rowptr, col;
    std::vector<double> val;
};

// Interior unknowns of the 5-point Laplacian on an m x m grid, diagonal scaled per
// row by a smooth positive coefficient (SPD, not a multiple of the identity).
HostCSR poisson5(int m) {
    HostCSR a;
    a.n = m * m;
    a.rowptr.push_back(0);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i) {
            const int r = j * m + i;
            const double c = 1.0 + 0.5 * std::sin(0.1 * r);
            if (j > 0) a.col.push_back(r - m), a.val.push_back(-1.0);
            if (i > 0) a.col.push_back(r - 1), a.val.push_back(-1.0);
            a.col.push_back(r), a.val.push_back(4.0 + c);
            if (i + 1 < m) a.col.push_back(r + 1), a.val.push_back(-1.0);
            if (j + 1 < m) a.col.push_back(r + m), a.val.push_back(-1.0);
            a.rowptr.push_back(static_cast<int>(a.col.size()));
        }
    return a;
}

std::vector<double> uniform(int n, unsigned seed) {
    std::vector<double> v(n);
    unsigned long long s = 0x9E3779B97F4A7C15ull ^ seed;
    for (auto& x : v) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        x = static_cast<double>(s >> 11) * 0x1.0p-53 * 2.0 - 1.0;
    }
    return v;
}

double rel_diff(const std::vector<double>& a, const std::vector<double>& b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i) num += (a[i] - b[i]) * (a[i] - b[i]), den += b[i] * b[i];
    return std::sqrt(num / (den > 0 ? den : 1.0));
}

double max_row_error(const HostCSR& a, const std::vector<double>& got, const std::vector<double>& want,
                     const std::vector<double>& in, const std::vector<double>& out0, double si, double so) {
    double worst = 0;
    for (int r = 0; r < a.n; ++r) {
        double scale = std::fabs(si * out0[r]);
        for (int k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) scale += std::fabs(so * a.val[k] * in[a.col[k]]);
        worst = std::fmax(worst, std::fabs(got[r] - want[r]) / (scale > 0 ? scale : 1.0));
    }
    return worst;
}

}  // namespace

int main() {
    try {
        const HostCSR a = poisson5(96);
        const int n = a.n;
        const std::vector<double> b = uniform(n, 1), x1 = uniform(n, 2), y0 = uniform(n, 3);

        // device copies through the spaces (solver.cpp:243-265)
        auto pSpace = std::make_shared<Space>();
        auto pIndexSpace = std::make_shared<CUDASpace<int>>(pSpace->sharedHandle());
        auto rowExtents = pIndexSpace->makeVector(a.rowptr.size());
        auto columnIndices = pIndexSpace->makeVector(a.col.size());
        auto entries = pSpace->makeVector(a.val.size());
        pIndexSpace->assign(CUDASpace<int>::view(rowExtents), std::span<const int>(a.rowptr));
        pIndexSpace->assign(CUDASpace<int>::view(columnIndices), std::span<const int>(a.col));
        pSpace->assign(Space::view(entries), std::span<const double>(a.val));
        DeviceCSR<double, int> deviceLHS{static_cast<size_t>(n), static_cast<size_t>(n), a.val.size(),
                                         rowExtents.get(), columnIndices.get(), entries.get()};
        auto rhs = pSpace->makeVector(n), in = pSpace->makeVector(n), out = pSpace->makeVector(n);
        pSpace->assign(Space::view(rhs), std::span<const double>(b));
        pSpace->assign(Space::view(in), std::span<const double>(x1));

        // SpMV with the reference's scale cases, (-1,-1) included
        auto pLhs = std::make_shared<CUDACSROperator<int, double>>(deviceLHS, pSpace);
        const double scales[][2] = {{0, 1}, {1, -1}, {-1, -1}, {2.0, 0.5}};
        for (auto& s : scales) {
            pSpace->assign(Space::view(out), std::span<const double>(y0));
            pLhs->product(s[0], Space::view(std::as_const(in)), s[1], Space::view(out));
            std::vector<double> got(n), want = y0;
            pSpace->assign(std::span<double>(got), Space::view(std::as_const(out)));
            ora_spmv(n, a.rowptr.data(), a.col.data(), a.val.data(), s[0], x1.data(), s[1], want.data());
            char what[96];
            std::snprintf(what, sizeof(what), "CSROperator::product (%g, %g) max row error", s[0], s[1]);
            report(max_row_error(a, got, want, x1, y0, s[0], s[1]) <= 1e-13, what,
                   max_row_error(a, got, want, x1, y0, s[0], s[1]));
        }

        // space operations
        {
            const double dot = pSpace->innerProduct(Space::view(std::as_const(in)), Space::view(std::as_const(rhs)));
            const double want = ora_dot(n, x1.data(), b.data());
            report(std::fabs(dot - want) <= 1e-12 * std::fabs(want) + 1e-12, "CUDASpace::innerProduct", dot - want);
        }

        // reference PCG (restatement) on the same system
        std::vector<double> xref(n, 0.0);
        double rstats[3] = {0, 0, 0};
        ora_pcg(n, a.rowptr.data(), a.col.data(), a.val.data(), b.data(), xref.data(), 5000, 0.0, 1e-10, 1, rstats);

        auto pPreconditioner = std::make_shared<DiagonalOperator<Space>>(
            makeDiagonalOperator<double, int, double>(*pLhs, std::const_pointer_cast<const Space>(pSpace)));
        ConjugateGradients<Space>::Statistics settings{5000, 0.0, 1e-10};
        {
            ConjugateGradients<Space> solver(pLhs, pSpace, pPreconditioner, settings);
            pSpace->fill(Space::view(out), 0.0);
            solver.product(0, Space::view(std::as_const(rhs)), 1, Space::view(out));
            std::vector<double> x(n);
            pSpace->assign(std::span<double>(x), Space::view(std::as_const(out)));
            const auto st = solver.getStats().value();
            report(solver.fused(), "ConjugateGradients: fused device solver selected", 0);
            report(rel_diff(x, xref) <= 1e-9, "ConjugateGradients (fused) vs reference PCG, rel diff", rel_diff(x, xref));
            report(std::llabs(static_cast<long long>(st.iterationCount) - static_cast<long long>(rstats[0])) <= 2,
                   "ConjugateGradients (fused) iterations - reference", st.iterationCount - rstats[0]);
        }
        {
            // a Jacobi operator of one sweep at relaxation 1 from x0 = 0 is D^-1 r: the
            // generic composition runs the same preconditioned iteration
            auto pJacobi = std::make_shared<JacobiOperator<Space>>(pSpace, n, pLhs, pPreconditioner, 1, 1.0);
            ConjugateGradients<Space> solver(pLhs, pSpace, pJacobi, settings);
            pSpace->fill(Space::view(out), 0.0);
            solver.product(0, Space::view(std::as_const(rhs)), 1, Space::view(out));
            std::vector<double> x(n);
            pSpace->assign(std::span<double>(x), Space::view(std::as_const(out)));
            const auto st = solver.getStats().value();
            report(!solver.fused(), "ConjugateGradients: generic composition selected", 0);
            report(rel_diff(x, xref) <= 1e-9, "ConjugateGradients (generic) vs reference PCG, rel diff",
                   rel_diff(x, xref));
            report(std::llabs(static_cast<long long>(st.iterationCount) - static_cast<long long>(rstats[0])) <= 2,
                   "ConjugateGradients (generic) iterations - reference", st.iterationCount - rstats[0]);
        }
        {
            // damped Jacobi, 6 sweeps at 2/3 (the p-multigrid smoother of solver.cpp:190-196)
            JacobiOperator<Space> jacobi(pSpace, n, pLhs, pPreconditioner, 6, 2.0 / 3.0);
            pSpace->assign(Space::view(out), std::span<const double>(y0));
            jacobi.product(1.0, Space::view(std::as_const(rhs)), -0.5, Space::view(out));
            std::vector<double> got(n), want = y0, dinv(n);
            pSpace->assign(std::span<double>(got), Space::view(std::as_const(out)));
            ora_diag_inverse(n, a.rowptr.data(), a.col.data(), a.val.data(), dinv.data());
            ora_jacobi(n, a.rowptr.data(), a.col.data(), a.val.data(), dinv.data(), 6, 2.0 / 3.0, 1.0, b.data(), -0.5,
                       want.data());
            report(rel_diff(got, want) <= 1e-13, "JacobiOperator (fused) vs restatement, rel diff", rel_diff(got, want));
        }
        {
            MixedPrecisionCG solver(pLhs, pPreconditioner, settings);
            pSpace->fill(Space::view(out), 0.0);
            solver.product(0, Space::view(std::as_const(rhs)), 1, Space::view(out));
            std::vector<double> x(n);
            pSpace->assign(std::span<double>(x), Space::view(std::as_const(out)));
            report(rel_diff(x, xref) <= 1e-9, "MixedPrecisionCG vs reference PCG, rel diff", rel_diff(x, xref));
            report(solver.getStats()->relativeResidual <= 1e-10, "MixedPrecisionCG true relative residual",
                   solver.getStats()->relativeResidual);
        }
        {
            // size mismatch is an exception, as CIE_CHECK is in the reference
            bool thrown = false;
            auto shorter = pSpace->makeVector(n - 1);
            try {
                pLhs->product(0, Space::view(std::as_const(in)), 1, Space::view(shorter));
            } catch (const Exception& e) {
                thrown = e.status() == CIECU_ERR_ARGUMENT;
            }
            report(thrown, "CSROperator::product size mismatch throws", 0);
            // a zero diagonal entry makes makeDiagonalOperator throw
            std::vector<double> broken = a.val;
            broken[a.rowptr[7] + 1] = 0.0;  // row 7 (first grid row, i > 0): its diagonal is entry 1
            auto brokenEntries = pSpace->makeVector(broken.size());
            pSpace->assign(Space::view(brokenEntries), std::span<const double>(broken));
            DeviceCSR<double, int> brokenLHS = deviceLHS;
            brokenLHS.entries = brokenEntries.get();
            thrown = false;
            try {
                auto d = makeDiagonalOperator<double, int, double>(brokenLHS, std::const_pointer_cast<const Space>(pSpace));
            } catch (const Exception& e) {
                thrown = e.status() == CIECU_ERR_DIAGONAL;
            }
            report(thrown, "makeDiagonalOperator on a zero diagonal throws", 0);
        }
        pSpace->synchronize();
    } catch (const std::exception& e) {
        std::printf("FAIL unexpected exception: %s\n", e.what());
        return 1;
    }
    if (g_failures) {
        std::printf("%d FAILED\n", g_failures);
        return 1;
    }
    std::printf("ALL OK\n");
    return 0;
}
