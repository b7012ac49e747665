// cie_cuda/fem.hpp -- C++ host API of the assembly side of the B200 path, over the
// ciecu C-ABI, in the style of cie_cuda/linalg.hpp.
//
//   reference (fem/packages)                     here (namespace cie::cuda)
//   IntegrandProcessor / SYCLIntegrandProcessor  CUDAIntegrandProcessor: the stiffness integrand
//     (utilities/inc/IntegrandProcessor.hpp:138-158) of a structured Q_p grid integrated on the
//     TransformedIntegrand<LinearIsotropic-        device and scattered into a device CSR matrix
//     StiffnessIntegrand>                          (stiffness, finiteCell, finiteCellF32)
//   KDTreeQuadraturePointFactory +               finiteCell: cut-cell tree and material scaling
//     ScaledMultiMaterialIntegrand
//   DirichletPenaltyIntegrand                    penalty: weak Dirichlet terms on the box faces
//   symmetric Dirichlet elimination              eliminate (fem/test/test_1d.cpp:291-313)
//     (fem/test/test_1d.cpp:291-313)
//   Assembler::makeCSRMatrix                     makeCSRPattern (on the device)
//   (python optcontrol/adjointmodel.py)          adjointGradient: transposed PCG solve + element gradient
#pragma once

#include "cie_cuda/linalg.hpp"
#include "ciecu_assembly.h"
#include "ciecu_graph.h"
#include "ciecu_host.h"

#include <array>
#include <vector>

namespace cie::cuda {

// A uniform grid of cells[0] x ... Q_order Lagrange cells with edge lengths
// cellSize, its DoF map (first axis fastest) on the device, and the cell colours.
struct StructuredGrid {
    int dim = 0, order = 0;
    std::array<int32_t, 3> cells{1, 1, 1};
    std::array<double, 3> cellSize{1.0, 1.0, 1.0};
    int32_t ndofs = 0;
    std::vector<int32_t> dofmap, colors;  // host copies

    StructuredGrid(int dim_, int order_, std::array<int32_t, 3> cells_) : dim(dim_), order(order_), cells(cells_) {
        long ncells = 1;
        int nb = 1;
        for (int d = 0; d < dim; ++d) {
            ncells *= cells[d];
            nb *= order + 1;
            cellSize[d] = 1.0 / cells[d];
        }
        dofmap.resize(static_cast<std::size_t>(ncells) * nb);
        colors.resize(static_cast<std::size_t>(ncells));
        check(ciecu_structured_dofmap(dim, order, cells.data(), dofmap.data(), &ndofs));
        check(ciecu_structured_colors(dim, cells.data(), colors.data()));
    }
    long cellCount() const noexcept { return static_cast<long>(colors.size()); }
    int basisSize() const noexcept {
        int nb = 1;
        for (int d = 0; d < dim; ++d) nb *= order + 1;
        return nb;
    }
};

// Assembler::makeCSRMatrix on the device: row extents and columns of the grid's pattern.
inline void makeCSRPattern(const CUDASpace<int>& space, long ncells, int nb, CUDAView<const int> dofmap, int32_t ndofs,
                           CUDAVector<int>& rowExtents, CUDAVector<int>& columnIndices) {
    rowExtents = space.makeVector(static_cast<std::size_t>(ndofs) + 1);
    int64_t nnz = 0;
    check(ciecu_csr_pattern_device(space.handle(), ncells, nb, dofmap.data(), ndofs, rowExtents.get(), nullptr, &nnz));
    columnIndices = space.makeVector(static_cast<std::size_t>(nnz));
    check(ciecu_csr_pattern_device(space.handle(), ncells, nb, dofmap.data(), ndofs, rowExtents.get(),
                                   columnIndices.get(), &nnz));
}

// The device integrand processor of one grid and one CSR pattern: a plan built
// once (element -> CSR-entry map; colours for the atomic-free scatter), then any
// number of assemblies into value arrays of that pattern.
class CUDAIntegrandProcessor {
public:
    using Space = CUDASpace<double>;

    CUDAIntegrandProcessor(std::shared_ptr<CUDACSROperator<int, double>> pPattern, const StructuredGrid& grid,
                           CUDAView<const int> deviceDofmap, int quadratureOrder = 0)
        : _pPattern(std::move(pPattern)), _grid(grid) {
        ciecu_assembly raw = nullptr;
        check(ciecu_assembly_create(_pPattern->handle(), grid.dim, grid.order,
                                    quadratureOrder ? quadratureOrder : grid.order + 1, grid.cellCount(),
                                    deviceDofmap.data(), grid.colors.data(), &raw));
        _plan = std::shared_ptr<ciecu_assembly_s>(raw, [](ciecu_assembly a) { ciecu_assembly_destroy(a); });
        _work = _pPattern->space()->makeVector(static_cast<std::size_t>(grid.basisSize()) * grid.basisSize());
    }

    // entries (+)= sum_e kappa_e K_e (convention 0: the reference's parametric
    // gradients with |det J^-1|; 1: physical gradients).
    void stiffness(CUDAView<const double> kappa, CUDAView<double> entries, int convention = 0,
                   bool accumulate = false) {
        check(ciecu_assemble_stiffness(_plan.get(), kappa.data(), _grid.cellSize.data(), convention,
                                       accumulate ? 1 : 0, entries.data()));
    }
    // Finite-cell stiffness of the sphere |x - center| < radius (factor alpha
    // outside, cut cells on a depth-maxDepth tree); returns the cut-cell count.
    int64_t finiteCell(std::array<double, 3> center, double radius, double alpha, int maxDepth,
                       CUDAView<double> entries, CUDAView<const double> kappa = {}, bool accumulate = false) {
        int64_t cut = 0;
        const std::array<double, 3> origin{0.0, 0.0, 0.0};
        check(ciecu_assemble_embedded(_plan.get(), kappa.data(), _grid.cellSize.data(), _grid.cells.data(),
                                      origin.data(), center.data(), radius, alpha, maxDepth, 0, accumulate ? 1 : 0,
                                      entries.data(), _work.get(), &cut));
        return cut;
    }
    // The same matrix in FP32 with the contraction on the tensor cores.
    int64_t finiteCellF32(std::array<double, 3> center, double radius, double alpha, int maxDepth,
                          CUDAView<float> entries32, CUDAView<const double> kappa = {}, bool accumulate = false) {
        int64_t cut = 0;
        const std::array<double, 3> origin{0.0, 0.0, 0.0};
        check(ciecu_assemble_embedded_f32(_plan.get(), kappa.data(), _grid.cellSize.data(), _grid.cells.data(),
                                          origin.data(), center.data(), radius, alpha, maxDepth, 0,
                                          accumulate ? 1 : 0, entries32.data(), &cut));
        return cut;
    }
    // Weak Dirichlet condition by penalty on the box faces of faceMask (0: all);
    // boundaryValues (nodal, may be empty) add their terms to rhs.
    void penalty(double penaltyFactor, CUDAView<double> entries, CUDAView<const double> boundaryValues = {},
                 CUDAView<double> rhs = {}, int faceMask = 0) {
        check(ciecu_assemble_dirichlet_penalty(_plan.get(), _grid.cells.data(), _grid.cellSize.data(), penaltyFactor,
                                               faceMask, 0, boundaryValues.data(), entries.data(), rhs.data()));
    }
    // Symmetric elimination of the flagged DoFs (rhs may be empty).
    void eliminate(CUDAView<const uint8_t> isBoundary, CUDAView<double> entries, CUDAView<double> rhs = {}) {
        check(ciecu_dirichlet_eliminate(_pPattern->handle(), isBoundary.data(), entries.data(), rhs.data()));
    }
    // dJ/dkappa_e = -lambda_e^T K_e(kappa = 1) u_e.
    void elementGradient(CUDAView<const double> lambda, CUDAView<const double> u, CUDAView<double> gradient,
                         int convention = 0) {
        check(ciecu_element_gradient(_plan.get(), _grid.cellSize.data(), convention, lambda.data(), u.data(),
                                     gradient.data(), _work.get()));
    }

    ciecu_assembly handle() const noexcept { return _plan.get(); }
    const StructuredGrid& grid() const noexcept { return _grid; }
    const std::shared_ptr<Space>& space() const noexcept { return _pPattern->space(); }

private:
    std::shared_ptr<CUDACSROperator<int, double>> _pPattern;
    StructuredGrid _grid;
    std::shared_ptr<ciecu_assembly_s> _plan;
    CUDAVector<double> _work;
};

// Adjoint sensitivities of J(u), u = A(kappa)^-1 P b (ciecu_adjoint_gradient):
// lambda = A^-1 P dJ/du by the solver's fused PCG (A is symmetric), dJ/db =
// lambda, and dJ/dkappa.  isBoundary may be empty (nothing eliminated).
inline SolverStatistics<double> adjointGradient(ConjugateGradients<CUDASpace<double>>& solver,
                                                CUDAIntegrandProcessor& processor, CUDAView<const uint8_t> isBoundary,
                                                CUDAView<const double> u, CUDAView<const double> dJdu,
                                                CUDAView<double> lambda, CUDAView<double> dJdkappa) {
    require(solver.fused(), "adjointGradient: the solver must be the fused device PCG (CSR operator + diagonal)");
    const int nb = processor.grid().basisSize();
    auto buffer = processor.space()->makeVector(2 * u.size() + static_cast<std::size_t>(nb) * nb);
    ciecu_statistics s{};
    check(ciecu_adjoint_gradient(solver.handle(), processor.handle(), processor.grid().cellSize.data(), 0,
                                 isBoundary.data(), u.data(), dJdu.data(), lambda.data(), dJdkappa.data(),
                                 buffer.get(), &s));
    return SolverStatistics<double>{static_cast<std::size_t>(s.iterationCount), s.absoluteResidual,
                                    s.relativeResidual};
}

}  // namespace cie::cuda
