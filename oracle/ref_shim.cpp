// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// A C-ABI wrapper, written for this project, around the reference's own CPU
// linear-algebra classes (kelofm/cie `libraries/linalg/packages/solvers`).  It is
// compiled together with the reference's unmodified sources, in place, by
// oracle/Makefile into oracle/_ref/libcieref.so.  Only the parity tests, smoke()
// and the CPU-baseline leg of bench.py load it; the CUDA product never does.
//
// Every function below drives the reference classes exactly the way the
// reference's own driver does:
//   * cieref_pcg        -> executables/fem_examples/src/poisson2D/solver.cpp:82-108
//                          (CSROperator + makeDiagonalOperator + ConjugateGradients)
//   * cieref_spmv       -> linalg/packages/solvers/src/CSROperator.cpp:33-111
//   * cieref_masked_spmv-> linalg/packages/solvers/src/MaskedCSROperator.cpp:37-118
//   * cieref_diag_inverse-> linalg/packages/solvers/src/DiagonalOperator.cpp:56-88
//   * cieref_jacobi     -> linalg/packages/solvers/src/JacobiOperator.cpp:36-62
//   * cieref_pmg        -> executables/fem_examples/src/poisson2D/solver.cpp:111-232
//   * cieref_space_*    -> linalg/packages/solvers/src/DefaultSpace.cpp:50-187
//   * cieref_gauss_legendre -> fem/packages/numeric/src/GaussLegendreQuadrature.cpp:82-175
//   * cieref_make_reordering -> linalg/packages/utilities/src/reorder.cpp:23-173 (serial: no pool)
//   * cieref_reorder    -> linalg/packages/utilities/src/reorder.cpp:215-365
//   * cieref_matrix_market[_vector] -> cieutils/packages/io/src/MatrixMarket.cpp
//   * cieref_lagrange   -> fem/packages/maths/src/LagrangePolynomial.cpp:18-72 (coefficients),
//                          fem/packages/maths/impl/Polynomial_impl.hpp (Horner evaluation,
//                          makeDerivative)
#include "packages/solvers/inc/ConjugateGradients.hpp"
#include "packages/solvers/inc/CSROperator.hpp"
#include "packages/solvers/inc/MaskedCSROperator.hpp"
#include "packages/solvers/inc/DiagonalOperator.hpp"
#include "packages/solvers/inc/JacobiOperator.hpp"
#include "packages/solvers/inc/MaskedIdentityOperator.hpp"
#include "packages/solvers/inc/NestedProductOperator.hpp"
#include "packages/solvers/inc/DefaultSpace.hpp"
#include "packages/concurrency/inc/ThreadPoolBase.hpp"
#include "packages/numeric/inc/GaussLegendreQuadrature.hpp"
#include "packages/maths/inc/LagrangePolynomial.hpp"
#include "packages/utilities/inc/reorder.hpp"
#include "packages/io/inc/MatrixMarket.hpp"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <fstream>
#include <memory>
#include <span>
#include <string>
#include <vector>

using namespace cie;

namespace {

thread_local std::string g_lastError;

int fail(const std::exception& e) {
    g_lastError = e.what();
    return 1;
}

using Space = linalg::DefaultSpace<double>;
using View = linalg::CSRView<const double, const int>;

View makeView(int nrows, int ncols, const int* rowptr, const int* col, const double* val) {
    const std::size_t nnz = static_cast<std::size_t>(rowptr[nrows]);
    return View(static_cast<std::size_t>(ncols),
                std::span<const int>(rowptr, static_cast<std::size_t>(nrows) + 1),
                std::span<const int>(col, nnz),
                std::span<const double>(val, nnz));
}

} // namespace

extern "C" {

int cieref_last_error(char* buffer, int size) {
    if (buffer && size > 0) {
        std::strncpy(buffer, g_lastError.c_str(), static_cast<std::size_t>(size) - 1);
        buffer[size - 1] = '\0';
    }
    return static_cast<int>(g_lastError.size());
}

int cieref_max_threads() {
    return static_cast<int>(mp::ThreadPoolBase::maxNumberOfThreads());
}

// Opaque thread pool handle (mp::ThreadPoolBase), so that timed calls exclude
// thread creation like the reference driver, which builds its pool once.
void* cieref_pool_create(int threads) {
    try {
        return new mp::ThreadPoolBase(static_cast<Size>(threads));
    } catch (const std::exception& e) {
        fail(e);
        return nullptr;
    }
}

void cieref_pool_destroy(void* pool) {
    delete static_cast<mp::ThreadPoolBase*>(pool);
}

int cieref_spmv(void* pool, int nrows, int ncols, const int* rowptr, const int* col,
                const double* val, double inScale, const double* in, double outScale,
                double* out) {
    try {
        auto view = makeView(nrows, ncols, rowptr, col, val);
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) threads = *static_cast<mp::ThreadPoolBase*>(pool);
        linalg::CSROperator<int, double> op(view, threads);
        op.product(inScale, std::span<const double>(in, static_cast<std::size_t>(ncols)), outScale,
                   std::span<double>(out, static_cast<std::size_t>(nrows)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_spmv_f32(void* pool, int nrows, int ncols, const int* rowptr, const int* col,
                    const float* val, float inScale, const float* in, float outScale, float* out) {
    try {
        const std::size_t nnz = static_cast<std::size_t>(rowptr[nrows]);
        linalg::CSRView<const float, const int> view(
            static_cast<std::size_t>(ncols), std::span<const int>(rowptr, static_cast<std::size_t>(nrows) + 1),
            std::span<const int>(col, nnz), std::span<const float>(val, nnz));
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) threads = *static_cast<mp::ThreadPoolBase*>(pool);
        linalg::CSROperator<int, float> op(view, threads);
        op.product(inScale, std::span<const float>(in, static_cast<std::size_t>(ncols)), outScale,
                   std::span<float>(out, static_cast<std::size_t>(nrows)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_masked_spmv(void* pool, int nrows, int ncols, const int* rowptr, const int* col,
                       const double* val, const std::uint16_t* mask, std::uint16_t threshold,
                       double inScale, const double* in, double outScale, double* out) {
    try {
        auto view = makeView(nrows, ncols, rowptr, col, val);
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) threads = *static_cast<mp::ThreadPoolBase*>(pool);
        linalg::MaskedCSROperator<int, double, double, std::uint16_t> op(
            view, std::span<const std::uint16_t>(mask, static_cast<std::size_t>(ncols)), threshold, threads);
        op.product(inScale, std::span<const double>(in, static_cast<std::size_t>(ncols)), outScale,
                   std::span<double>(out, static_cast<std::size_t>(nrows)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_diag_inverse(int nrows, const int* rowptr, const int* col, const double* val,
                        double* inverseDiagonal) {
    try {
        auto view = makeView(nrows, nrows, rowptr, col, val);
        auto pSpace = std::make_shared<Space>();
        auto diag = linalg::makeDiagonalOperator<double, int, double>(view, pSpace);
        // Read the stored inverse diagonal back through the operator: D^-1 * ones.
        std::vector<double> ones(static_cast<std::size_t>(nrows), 1.0);
        diag.product(0.0, ones, 1.0, std::span<double>(inverseDiagonal, static_cast<std::size_t>(nrows)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Jacobi-preconditioned CG exactly as solveCG builds it.  stats_out receives
// {iterationCount, absoluteResidual, relativeResidual}; seconds_out the
// steady_clock time of ConjugateGradients::product alone.
int cieref_pcg(void* pool, int n, const int* rowptr, const int* col, const double* val,
               const double* b, double* x, long maxIterations, double absoluteTolerance,
               double relativeTolerance, int precondition, int verbosity, double* stats_out,
               double* seconds_out) {
    try {
        auto view = makeView(n, n, rowptr, col, val);
        std::shared_ptr<Space> pSpace;
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) {
            threads = *static_cast<mp::ThreadPoolBase*>(pool);
            pSpace = std::make_shared<Space>(*static_cast<mp::ThreadPoolBase*>(pool));
        } else {
            pSpace = std::make_shared<Space>();
        }
        auto pLhs = std::make_shared<linalg::CSROperator<int, double>>(view, threads);
        std::shared_ptr<linalg::LinearOperator<Space>> pPrecond;
        if (precondition)
            pPrecond = std::make_shared<linalg::DiagonalOperator<Space>>(
                linalg::makeDiagonalOperator<double, int, double>(view, pSpace));
        linalg::ConjugateGradients<Space>::Statistics settings{
            .iterationCount = static_cast<std::size_t>(maxIterations),
            .absoluteResidual = absoluteTolerance,
            .relativeResidual = relativeTolerance};
        linalg::ConjugateGradients<Space> solver(pLhs, pSpace, pPrecond, settings, verbosity);
        const auto t0 = std::chrono::steady_clock::now();
        solver.product(0.0, std::span<const double>(b, static_cast<std::size_t>(n)), 1.0,
                       std::span<double>(x, static_cast<std::size_t>(n)));
        const auto t1 = std::chrono::steady_clock::now();
        const auto stats = solver.getStats().value();
        if (stats_out) {
            stats_out[0] = static_cast<double>(stats.iterationCount);
            stats_out[1] = stats.absoluteResidual;
            stats_out[2] = stats.relativeResidual;
        }
        if (seconds_out) *seconds_out = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// JacobiOperator over a CSROperator with the diagonal preconditioner as its
// inverse diagonal (the smoother configuration of solveMultigrid).
int cieref_jacobi(void* pool, int n, const int* rowptr, const int* col, const double* val,
                  long iterations, double relaxation, double inScale, const double* in,
                  double outScale, double* out) {
    try {
        auto view = makeView(n, n, rowptr, col, val);
        std::shared_ptr<Space> pSpace;
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) {
            threads = *static_cast<mp::ThreadPoolBase*>(pool);
            pSpace = std::make_shared<Space>(*static_cast<mp::ThreadPoolBase*>(pool));
        } else {
            pSpace = std::make_shared<Space>();
        }
        auto pLhs = std::make_shared<linalg::CSROperator<int, double>>(view, threads);
        auto pDiag = std::make_shared<linalg::DiagonalOperator<Space>>(
            linalg::makeDiagonalOperator<double, int, double>(view, pSpace));
        linalg::JacobiOperator<Space> op(pSpace, static_cast<std::size_t>(n), pLhs, pDiag,
                                         static_cast<std::size_t>(iterations), relaxation);
        op.product(inScale, std::span<const double>(in, static_cast<std::size_t>(n)), outScale,
                   std::span<double>(out, static_cast<std::size_t>(n)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// The p-multigrid cycle of solveMultigrid (solver.cpp:111-232) over an
// externally supplied ansatz mask.  levels = polynomial order p; grid 0 is CG on
// the masked (threshold 2) operator with relative tolerance 0.5, grids 2..p are
// 6 sweeps of damped Jacobi (omega = 2/3) on the masked (threshold k+1)
// operator.  Stops when ||r|| <= tolerance * ||r0||; cycles_out receives the
// number of V-cycles, relres_out the final ||r||/||r0||.
int cieref_pmg(void* pool, int n, const int* rowptr, const int* col, const double* val,
               const std::uint16_t* mask, int polynomialOrder, const double* b, double* x,
               double tolerance, long maxCycles, long* cycles_out, double* relres_out) {
    try {
        auto view = makeView(n, n, rowptr, col, val);
        using Operator = linalg::LinearOperator<Space>;
        using MaskSpace = linalg::DefaultSpace<std::uint16_t>;
        std::shared_ptr<Space> pSpace;
        OptionalRef<mp::ThreadPoolBase> threads;
        if (pool) {
            threads = *static_cast<mp::ThreadPoolBase*>(pool);
            pSpace = std::make_shared<Space>(*static_cast<mp::ThreadPoolBase*>(pool));
        } else {
            pSpace = std::make_shared<Space>();
        }
        auto pMaskSpace = std::make_shared<MaskSpace>();
        const std::span<const std::uint16_t> maskView(mask, static_cast<std::size_t>(n));
        const std::span<const double> rhs(b, static_cast<std::size_t>(n));
        const std::span<double> solution(x, static_cast<std::size_t>(n));

        auto residual = pSpace->makeVector(static_cast<std::size_t>(n));
        pSpace->assign(residual, rhs);
        // The reference starts from the residual of the zero guess; the input x is
        // expected to be zero (it is accumulated into, like the reference).
        const double initialResidualNorm = std::sqrt(pSpace->innerProduct(residual, residual));

        struct Grid {
            std::shared_ptr<Operator> pOperator, pRestriction, pLhs;
        };
        std::vector<Grid> grids;
        auto pInverseDiagonal = std::make_shared<linalg::DiagonalOperator<Space>>(
            linalg::makeDiagonalOperator<double, int, double>(view, pSpace));
        {
            const std::uint16_t threshold = 2;
            auto pGridLhs = std::make_shared<linalg::MaskedCSROperator<int, double, double, std::uint16_t>>(
                view, maskView, threshold, threads);
            linalg::ConjugateGradients<Space>::Statistics settings{
                .iterationCount = 5000, .absoluteResidual = 0, .relativeResidual = 5e-1};
            auto pOperator = std::make_shared<linalg::ConjugateGradients<Space>>(
                pGridLhs, pSpace, pInverseDiagonal, settings, 0);
            auto pRestriction = std::make_shared<linalg::MaskedIdentityOperator<Space, MaskSpace>>(
                pSpace, pMaskSpace, maskView, threshold);
            grids.push_back(Grid{pOperator, pRestriction, pGridLhs});
        }
        for (int order = 2; order < polynomialOrder + 1; ++order) {
            const std::uint16_t threshold = static_cast<std::uint16_t>(order + 1);
            auto pGridLhs = std::make_shared<linalg::MaskedCSROperator<int, double, double, std::uint16_t>>(
                view, maskView, threshold, threads);
            auto pMask = std::make_shared<linalg::MaskedIdentityOperator<Space, MaskSpace>>(
                pSpace, pMaskSpace, maskView, threshold);
            auto pSmoother = std::make_shared<linalg::JacobiOperator<Space>>(
                pSpace, static_cast<std::size_t>(n), pGridLhs, pInverseDiagonal, 6, 2.0 / 3.0);
            auto pOperator = std::make_shared<linalg::NestedProductOperator<Space>>(
                pSpace, pSmoother, pMask, static_cast<std::size_t>(n));
            grids.push_back(Grid{pOperator, pMask, pGridLhs});
        }

        double residualNorm = initialResidualNorm;
        auto gridResidual = pSpace->makeVector(static_cast<std::size_t>(n));
        auto solutionUpdate = pSpace->makeVector(static_cast<std::size_t>(n));
        long cycles = 0;
        while (tolerance * initialResidualNorm < residualNorm && cycles < maxCycles) {
            auto visit = [&](Grid& grid) {
                grid.pRestriction->product(0, residual, 1, gridResidual);
                pSpace->fill(solutionUpdate, 0);
                grid.pOperator->product(0, gridResidual, 1, solutionUpdate);
                pSpace->add(solution, solutionUpdate, 1);
                grid.pLhs->product(1, solutionUpdate, -1, residual);
            };
            for (auto it = grids.rbegin(); it != grids.rend(); ++it) visit(*it);
            for (auto it = grids.begin() + 1; it != grids.end(); ++it) visit(*it);
            residualNorm = std::sqrt(pSpace->innerProduct(residual, residual));
            ++cycles;
        }
        if (cycles_out) *cycles_out = cycles;
        if (relres_out) *relres_out = initialResidualNorm > 0 ? residualNorm / initialResidualNorm : 0.0;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_space_dot(void* pool, long n, const double* a, const double* b, double* out) {
    try {
        Space space = pool ? Space(*static_cast<mp::ThreadPoolBase*>(pool)) : Space();
        *out = space.innerProduct(std::span<const double>(a, static_cast<std::size_t>(n)),
                                  std::span<const double>(b, static_cast<std::size_t>(n)));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// op: 0 scale(t, s, alpha) [t = alpha * t (.) s]; 1 scale(t, alpha); 2 add(t, s, alpha);
//     3 assign(t, s); 4 fill(t, alpha)
int cieref_space_op(void* pool, int op, long n, double* target, const double* source, double alpha) {
    try {
        Space space = pool ? Space(*static_cast<mp::ThreadPoolBase*>(pool)) : Space();
        std::span<double> t(target, static_cast<std::size_t>(n));
        std::span<const double> s(source, source ? static_cast<std::size_t>(n) : 0u);
        switch (op) {
            case 0: space.scale(t, s, alpha); break;
            case 1: space.scale(t, alpha); break;
            case 2: space.add(t, s, alpha); break;
            case 3: space.assign(t, s); break;
            case 4: space.fill(t, alpha); break;
            default: g_lastError = "unknown space op"; return 1;
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_gauss_legendre(int order, double* nodes, double* weights) {
    try {
        fem::GaussLegendreQuadrature<double> quadrature(static_cast<Size>(order));
        for (int i = 0; i < order; ++i) {
            nodes[i] = quadrature.nodes()[static_cast<std::size_t>(i)];
            weights[i] = quadrature.weights()[static_cast<std::size_t>(i)];
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// The 1-D Lagrange basis polynomial of node iBase on the given nodes, built by the
// reference's LagrangePolynomial: its ascending monomial coefficients (count of
// them), and its value and derivative (Polynomial::evaluate of the polynomial and
// of makeDerivative()) at each of the npts points.
int cieref_lagrange(int count, const double* nodes, int iBase, int npts, const double* points,
                    double* coefficients, double* values, double* derivatives) {
    try {
        const fem::maths::LagrangePolynomial<double> basis(std::span<const double>(nodes, static_cast<std::size_t>(count)),
                                                           static_cast<Size>(iBase));
        const auto c = basis.coefficients();
        for (std::size_t k = 0; k < c.size(); ++k) coefficients[k] = c[k];
        const auto derivative = basis.makeDerivative();
        for (int i = 0; i < npts; ++i) {
            double in[1] = {points[i]}, out[1] = {0.0};
            basis.evaluate(std::span<const double>(in, 1), std::span<double>(out, 1), {});
            values[i] = out[0];
            derivative.evaluate(std::span<const double>(in, 1), std::span<double>(out, 1), {});
            derivatives[i] = out[0];
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// makeReordering<int,double> without a thread pool (the pool's minimum-degree
// search combines per-thread minima, which can pick another start row among
// equal degrees): map[new row] = old row.  strategy 1: Cuthill-McKee, 2: reverse.
int cieref_make_reordering(int n, const int* rowptr, const int* col, const double* val, int strategy, int* map) {
    try {
        const std::size_t nnz = static_cast<std::size_t>(rowptr[n]);
        makeReordering<int, double>(std::span<int>(map, static_cast<std::size_t>(n)),
                                    std::span<const int>(rowptr, static_cast<std::size_t>(n) + 1),
                                    std::span<const int>(col, nnz), std::span<const double>(val, nnz),
                                    strategy == 2 ? ReorderingStrategy::ReverseCuthillMcKee
                                                  : ReorderingStrategy::CuthillMcKee,
                                    {});
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// reorder<int,double,false>: the CSR matrix permuted in place, new row i = old row
// map[i], columns renumbered and sorted within each row.
int cieref_reorder(int n, const int* map, int* rowptr, int* col, double* val) {
    try {
        const std::size_t nnz = static_cast<std::size_t>(rowptr[n]);
        reorder<int, double, false>(std::span<const int>(map, static_cast<std::size_t>(n)),
                                    std::span<int>(rowptr, static_cast<std::size_t>(n) + 1), std::span<int>(col, nnz),
                                    std::span<double>(val, nnz), {});
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_matrix_market(const char* path, int rows, int columns, const int* rowptr, const int* col,
                         const double* val) {
    try {
        std::ofstream file(path);
        io::MatrixMarket::Output out(file);
        out(rows, columns, rowptr[rows], rowptr, col, val);
        return file.good() ? 0 : 1;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int cieref_matrix_market_vector(const char* path, long n, const double* values) {
    try {
        std::ofstream file(path);
        io::MatrixMarket::Output out(file);
        out(values, static_cast<std::size_t>(n));
        return file.good() ? 0 : 1;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

} // extern "C"
