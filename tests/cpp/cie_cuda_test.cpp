// Test program of the C++ host API (include/cie_cuda/linalg.hpp, solvers.hpp,
// fem.hpp), written the way the reference's own driver uses its SYCL backend
// (executables/fem_examples/src/poisson2D/solver.cpp:238-288): matrix and vectors
// copied to the device through the space, a CSR operator, makeDiagonalOperator,
// ConjugateGradients; then the batched, multi-RHS and two-level solvers, the
// reordering, and the assembly processor with the adjoint gradient.
// Results are checked against the C restatement in oracle/ (test infrastructure).
// Prints one line per check and "ALL OK" at the end; exit status 1 on a failure.
#include "cie_cuda/fem.hpp"
#include "cie_cuda/linalg.hpp"
#include "cie_cuda/solvers.hpp"

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

// Device copies of a host CSR matrix kept alive together.
struct DeviceMatrix {
    CUDAVector<int> rowExtents, columnIndices;
    CUDAVector<double> entries;
    DeviceCSR<double, int> view;
};

DeviceMatrix upload(const std::shared_ptr<Space>& pSpace, const HostCSR& a) {
    CUDASpace<int> indexSpace(pSpace->sharedHandle());
    DeviceMatrix m;
    m.rowExtents = indexSpace.makeVector(a.rowptr.size());
    m.columnIndices = indexSpace.makeVector(a.col.size());
    m.entries = pSpace->makeVector(a.val.size());
    indexSpace.assign(CUDASpace<int>::view(m.rowExtents), std::span<const int>(a.rowptr));
    indexSpace.assign(CUDASpace<int>::view(m.columnIndices), std::span<const int>(a.col));
    pSpace->assign(Space::view(m.entries), std::span<const double>(a.val));
    m.view = DeviceCSR<double, int>{static_cast<size_t>(a.n), static_cast<size_t>(a.n), a.val.size(),
                                    m.rowExtents.get(), m.columnIndices.get(), m.entries.get()};
    return m;
}

std::vector<double> download(const std::shared_ptr<Space>& pSpace, const Space::Vector& v) {
    std::vector<double> h(v.size());
    pSpace->assign(std::span<double>(h), Space::view(v));
    return h;
}

std::vector<double> reference_solve(const HostCSR& a, const std::vector<double>& b, double* iterations = nullptr) {
    std::vector<double> x(a.n, 0.0);
    double st[3] = {0, 0, 0};
    ora_pcg(a.n, a.rowptr.data(), a.col.data(), a.val.data(), b.data(), x.data(), 20000, 0.0, 1e-10, 1, st);
    if (iterations) *iterations = st[0];
    return x;
}

// The solvers without a single reference class, each checked system by system /
// column by column against the restated reference CG.
void solver_classes(const std::shared_ptr<Space>& pSpace) {
    using Stats = ConjugateGradients<Space>::Statistics;
    const Stats settings{20000, 0.0, 1e-10};
    {
        // two systems in one block-diagonal matrix
        const HostCSR s0 = poisson5(20), s1 = poisson5(31);
        HostCSR bd;
        bd.n = s0.n + s1.n;
        bd.rowptr = s0.rowptr;
        bd.col = s0.col;
        bd.val = s0.val;
        for (int r = 0; r < s1.n; ++r) {
            for (int k = s1.rowptr[r]; k < s1.rowptr[r + 1]; ++k) bd.col.push_back(s1.col[k] + s0.n), bd.val.push_back(s1.val[k]);
            bd.rowptr.push_back(static_cast<int>(bd.col.size()));
        }
        auto dm = upload(pSpace, bd);
        auto pA = std::make_shared<CUDACSROperator<int, double>>(dm.view, pSpace);
        auto pD = std::make_shared<DiagonalOperator<Space>>(
            makeDiagonalOperator<double, int, double>(*pA, std::const_pointer_cast<const Space>(pSpace)));
        BatchedConjugateGradients batch(pA, {0, s0.n, s0.n + s1.n}, pD, settings);
        const std::vector<double> b = uniform(bd.n, 7);
        auto rhs = pSpace->makeVector(bd.n), x = pSpace->makeVector(bd.n);
        pSpace->assign(Space::view(rhs), std::span<const double>(b));
        pSpace->fill(Space::view(x), 0.0);
        batch.product(0, Space::view(std::as_const(rhs)), 1, Space::view(x));
        const std::vector<double> xh = download(pSpace, x);
        const std::vector<double> x0 = reference_solve(s0, std::vector<double>(b.begin(), b.begin() + s0.n));
        const std::vector<double> x1 = reference_solve(s1, std::vector<double>(b.begin() + s0.n, b.end()));
        const double e0 = rel_diff(std::vector<double>(xh.begin(), xh.begin() + s0.n), x0);
        const double e1 = rel_diff(std::vector<double>(xh.begin() + s0.n, xh.end()), x1);
        report(e0 <= 1e-9 && e1 <= 1e-9 && batch.getStats().size() == 2,
               "BatchedConjugateGradients per system vs reference PCG", std::fmax(e0, e1));
        // FP32 iterations with FP64 reliable updates: same bar
        batch.setReliableUpdates(0.1);
        pSpace->fill(Space::view(x), 0.0);
        batch.product(0, Space::view(std::as_const(rhs)), 1, Space::view(x));
        const std::vector<double> xr = download(pSpace, x);
        const double f0 = rel_diff(std::vector<double>(xr.begin(), xr.begin() + s0.n), x0);
        const double f1 = rel_diff(std::vector<double>(xr.begin() + s0.n, xr.end()), x1);
        const auto reps = batch.refinements();
        report(f0 <= 1e-9 && f1 <= 1e-9 && reps[0] > 0 && reps[1] > 0,
               "BatchedConjugateGradients reliable updates vs reference PCG", std::fmax(f0, f1));
    }
    const HostCSR a = poisson5(40);
    auto dm = upload(pSpace, a);
    auto pA = std::make_shared<CUDACSROperator<int, double>>(dm.view, pSpace);
    auto pD = std::make_shared<DiagonalOperator<Space>>(
        makeDiagonalOperator<double, int, double>(*pA, std::const_pointer_cast<const Space>(pSpace)));
    const std::vector<double> b = uniform(a.n, 9);
    const std::vector<double> xref = reference_solve(a, b);
    {
        // three right-hand sides b, 2b, -b (row-major n x 3)
        const int k = 3;
        std::vector<double> B(static_cast<size_t>(a.n) * k);
        for (int i = 0; i < a.n; ++i) B[i * k] = b[i], B[i * k + 1] = 2.0 * b[i], B[i * k + 2] = -b[i];
        auto rhs = pSpace->makeVector(B.size()), X = pSpace->makeVector(B.size());
        pSpace->assign(Space::view(rhs), std::span<const double>(B));
        pSpace->fill(Space::view(X), 0.0);
        MultiRHSConjugateGradients multi(pA, k, pD, settings);
        multi.product(0, Space::view(std::as_const(rhs)), 1, Space::view(X));
        const std::vector<double> Xh = download(pSpace, X);
        double worst = 0.0;
        const double factor[3] = {1.0, 2.0, -1.0};
        for (int c = 0; c < k; ++c) {
            std::vector<double> col(a.n), want(a.n);
            for (int i = 0; i < a.n; ++i) col[i] = Xh[i * k + c], want[i] = factor[c] * xref[i];
            worst = std::fmax(worst, rel_diff(col, want));
        }
        report(worst <= 1e-9, "MultiRHSConjugateGradients per column vs reference PCG", worst);
        // the FP32-refined form from zero: same bar
        multi.setRefinement(0.1);
        pSpace->fill(Space::view(X), 0.0);
        multi.product(0, Space::view(std::as_const(rhs)), 1, Space::view(X));
        const std::vector<double> Xr = download(pSpace, X);
        double worstR = 0.0;
        for (int c = 0; c < k; ++c) {
            std::vector<double> col(a.n), want(a.n);
            for (int i = 0; i < a.n; ++i) col[i] = Xr[i * k + c], want[i] = factor[c] * xref[i];
            worstR = std::fmax(worstR, rel_diff(col, want));
        }
        const auto refinements = multi.refinements();
        report(worstR <= 1e-9 && refinements[0] > 0, "MultiRHSConjugateGradients FP32-refined vs reference PCG",
               worstR);
    }
    {
        // two levels with the identity transfer and the fine matrix as coarse matrix
        HostCSR eye;
        eye.n = a.n;
        for (int i = 0; i <= a.n; ++i) eye.rowptr.push_back(i);
        for (int i = 0; i < a.n; ++i) eye.col.push_back(i), eye.val.push_back(1.0);
        auto de = upload(pSpace, eye);
        auto pEye = std::make_shared<CUDACSROperator<int, double>>(de.view, pSpace);
        TwoLevelConjugateGradients mg(pA, pD, pEye, pEye, pA, pD, settings, ciecu_mg_options{2, 0.0, 30.0, 10, 1});
        auto rhs = pSpace->makeVector(a.n), x = pSpace->makeVector(a.n);
        pSpace->assign(Space::view(rhs), std::span<const double>(b));
        pSpace->fill(Space::view(x), 0.0);
        mg.product(0, Space::view(std::as_const(rhs)), 1, Space::view(x));
        const double e = rel_diff(download(pSpace, x), xref);
        report(e <= 1e-9 && mg.getStats()->relativeResidual < 1e-10, "TwoLevelConjugateGradients vs reference PCG", e);
    }
    {
        // reverse Cuthill-McKee on the device, the permuted solve mapped back
        CUDASpace<int> indexSpace(pSpace->sharedHandle());
        auto map = indexSpace.makeVector(a.n);
        makeReordering(*pSpace, CUDASpace<int>::view(map), dm.view, ReorderingStrategy::ReverseCuthillMcKee);
        std::vector<int> mapH(a.n), mapRef(a.n);
        indexSpace.assign(std::span<int>(mapH), CUDASpace<int>::view(std::as_const(map)));
        ora_cuthill_mckee(a.n, a.rowptr.data(), a.col.data(), 2, mapRef.data());
        report(mapH == mapRef, "makeReordering (RCM) vs restated sequential order", 0);
        auto rp = indexSpace.makeVector(a.n + 1), cl = indexSpace.makeVector(a.col.size());
        auto vl = pSpace->makeVector(a.val.size());
        const CUDAView<const int> mapView = CUDASpace<int>::view(std::as_const(map));
        reorder(*pSpace, mapView, dm.view, CUDASpace<int>::view(rp), CUDASpace<int>::view(cl), Space::view(vl));
        DeviceCSR<double, int> permuted{static_cast<size_t>(a.n), static_cast<size_t>(a.n), a.val.size(), rp.get(),
                                        cl.get(), vl.get()};
        auto pB = std::make_shared<CUDACSROperator<int, double>>(permuted, pSpace);
        auto pDB = std::make_shared<DiagonalOperator<Space>>(
            makeDiagonalOperator<double, int, double>(*pB, std::const_pointer_cast<const Space>(pSpace)));
        auto rhs = pSpace->makeVector(a.n), bp = pSpace->makeVector(a.n), xp = pSpace->makeVector(a.n);
        auto x = pSpace->makeVector(a.n);
        pSpace->assign(Space::view(rhs), std::span<const double>(b));
        reorder(*pSpace, mapView, Space::view(std::as_const(rhs)), Space::view(bp));
        ConjugateGradients<Space> solver(pB, pSpace, pDB, settings);
        pSpace->fill(Space::view(xp), 0.0);
        solver.product(0, Space::view(std::as_const(bp)), 1, Space::view(xp));
        reorder(*pSpace, mapView, Space::view(std::as_const(xp)), Space::view(x), true);
        const double e = rel_diff(download(pSpace, x), xref);
        report(e <= 1e-9, "reordered solve mapped back vs reference PCG", e);
    }
}

// The assembly processor on a 2D Q2 grid: device pattern, stiffness, elimination,
// solve and adjoint gradient against the restatement.
void assembly_classes(const std::shared_ptr<Space>& pSpace) {
    StructuredGrid grid(2, 2, {8, 6, 1});
    const int nb = grid.basisSize();
    const long ncells = grid.cellCount();
    CUDASpace<int> indexSpace(pSpace->sharedHandle());
    auto dofmap = indexSpace.makeVector(grid.dofmap.size());
    indexSpace.assign(CUDASpace<int>::view(dofmap), std::span<const int>(grid.dofmap));
    CUDAVector<int> rowExtents, columnIndices;
    makeCSRPattern(indexSpace, ncells, nb, CUDASpace<int>::view(std::as_const(dofmap)), grid.ndofs, rowExtents,
                   columnIndices);
    HostCSR a;
    a.n = grid.ndofs;
    a.rowptr.resize(a.n + 1);
    const long nnz = ora_csr_pattern(ncells, nb, grid.dofmap.data(), a.n, a.rowptr.data(), nullptr);
    a.col.resize(nnz);
    ora_csr_pattern(ncells, nb, grid.dofmap.data(), a.n, a.rowptr.data(), a.col.data());
    std::vector<int> rpH(a.n + 1), colH(columnIndices.size());
    indexSpace.assign(std::span<int>(rpH), CUDASpace<int>::view(std::as_const(rowExtents)));
    indexSpace.assign(std::span<int>(colH), CUDASpace<int>::view(std::as_const(columnIndices)));
    report(rpH == a.rowptr && colH == a.col, "makeCSRPattern (device) vs Assembler::makeCSRMatrix restatement", 0);
    auto entries = pSpace->makeVector(a.col.size());
    DeviceCSR<double, int> m{static_cast<size_t>(a.n), static_cast<size_t>(a.n), a.col.size(), rowExtents.get(),
                             columnIndices.get(), entries.get()};
    auto pA = std::make_shared<CUDACSROperator<int, double>>(m, pSpace);
    CUDAIntegrandProcessor processor(pA, grid, CUDASpace<int>::view(std::as_const(dofmap)));
    std::vector<double> kappa(ncells);
    for (long e = 0; e < ncells; ++e) kappa[e] = 1.0 + 0.25 * std::sin(0.7 * e);
    auto kappaD = pSpace->makeVector(ncells);
    pSpace->assign(Space::view(kappaD), std::span<const double>(kappa));
    processor.stiffness(Space::view(std::as_const(kappaD)), Space::view(entries));
    // restatement: element matrices kappa_e K1 at the tensor Gauss points, scattered
    std::vector<double> gn(3), gw(3), pts(9 * 2), wts(9), K1(static_cast<size_t>(nb) * nb);
    ora_gauss_legendre(3, gn.data(), gw.data());
    for (int q = 0; q < 9; ++q) pts[2 * q] = gn[q % 3], pts[2 * q + 1] = gn[q / 3], wts[q] = gw[q % 3] * gw[q / 3];
    ora_element_stiffness(2, 2, 9, pts.data(), wts.data(), 1.0, grid.cellSize.data(), 0, K1.data());
    std::vector<double> Ke(static_cast<size_t>(ncells) * nb * nb);
    for (long e = 0; e < ncells; ++e)
        for (int k = 0; k < nb * nb; ++k) Ke[e * nb * nb + k] = kappa[e] * K1[k];
    a.val.assign(a.col.size(), 0.0);
    ora_assemble(ncells, nb, grid.dofmap.data(), Ke.data(), a.rowptr.data(), a.col.data(), a.val.data());
    const std::vector<double> got = download(pSpace, entries);
    double worst = 0.0, scale = 0.0;
    for (size_t k = 0; k < got.size(); ++k) worst = std::fmax(worst, std::fabs(got[k] - a.val[k])), scale = std::fmax(scale, std::fabs(a.val[k]));
    report(worst <= 1e-13 * scale, "CUDAIntegrandProcessor::stiffness vs restatement", worst / scale);
    // homogeneous Dirichlet by elimination, solve, adjoint gradient of J = |u|^2 / 2
    std::vector<uint8_t> bnd(a.n);
    check(ciecu_structured_boundary(2, 2, grid.cells.data(), bnd.data()));
    CUDASpace<uint8_t> byteSpace(pSpace->sharedHandle());
    auto bndD = byteSpace.makeVector(a.n);
    byteSpace.assign(CUDASpace<uint8_t>::view(bndD), std::span<const uint8_t>(bnd));
    std::vector<double> b = uniform(a.n, 13);
    auto rhs = pSpace->makeVector(a.n);
    pSpace->assign(Space::view(rhs), std::span<const double>(b));
    processor.eliminate(CUDASpace<uint8_t>::view(std::as_const(bndD)), Space::view(entries), Space::view(rhs));
    ora_dirichlet_eliminate(a.n, a.rowptr.data(), a.col.data(), a.val.data(), bnd.data(), b.data());
    auto pD = std::make_shared<DiagonalOperator<Space>>(
        makeDiagonalOperator<double, int, double>(*pA, std::const_pointer_cast<const Space>(pSpace)));
    ConjugateGradients<Space> solver(pA, pSpace, pD, ConjugateGradients<Space>::Statistics{20000, 0.0, 1e-10});
    auto u = pSpace->makeVector(a.n);
    pSpace->fill(Space::view(u), 0.0);
    solver.product(0, Space::view(std::as_const(rhs)), 1, Space::view(u));
    auto lambda = pSpace->makeVector(a.n), grad = pSpace->makeVector(ncells);
    adjointGradient(solver, processor, CUDASpace<uint8_t>::view(std::as_const(bndD)), Space::view(std::as_const(u)),
                    Space::view(std::as_const(u)), Space::view(lambda), Space::view(grad));
    std::vector<double> uh = download(pSpace, u);
    const std::vector<double> uref = reference_solve(a, b);
    std::vector<double> pu = uref;
    for (int i = 0; i < a.n; ++i) if (bnd[i]) pu[i] = 0.0;
    std::vector<double> lref = reference_solve(a, pu);
    for (int i = 0; i < a.n; ++i) if (bnd[i]) lref[i] = 0.0;
    std::vector<double> gref(ncells);
    ora_element_gradient(ncells, nb, grid.dofmap.data(), K1.data(), lref.data(), pu.data(), gref.data());
    const double eg = rel_diff(download(pSpace, grad), gref);
    report(rel_diff(uh, uref) <= 1e-9, "assembled system solve vs reference PCG", rel_diff(uh, uref));
    report(eg <= 1e-8, "adjointGradient dJ/dkappa vs restated adjoint", eg);
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
            // one kernel per inner iteration over the diagonal copy (fuseDirection 2)
            MixedPrecisionCG solver(pLhs, pPreconditioner, settings, ciecu_mixed_options{0, 0.1, 1, -2, 0, 2});
            pSpace->fill(Space::view(out), 0.0);
            solver.product(0, Space::view(std::as_const(rhs)), 1, Space::view(out));
            std::vector<double> x(n);
            pSpace->assign(std::span<double>(x), Space::view(std::as_const(out)));
            report(solver.kernelsPerIteration() == 1, "MixedPrecisionCG single pass: kernels per inner iteration",
                   solver.kernelsPerIteration());
            report(rel_diff(x, xref) <= 1e-9, "MixedPrecisionCG single pass vs reference PCG, rel diff",
                   rel_diff(x, xref));
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
        solver_classes(pSpace);
        assembly_classes(pSpace);
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
