// cie_cuda/solvers.hpp -- C++ classes for the solvers of the B200 path that have no
// single reference class, over the ciecu C-ABI, in the style of cie_cuda/linalg.hpp
// (same product semantics out <- inScale * out + outScale * x, same statistics,
// non-zero statuses thrown as cie::cuda::Exception):
//
//   BatchedConjugateGradients   many independent systems in one block-diagonal CSR
//                               matrix, one solve (ciecu_batch_*)
//   MultiRHSConjugateGradients  k right-hand sides of one matrix as SpMM-CG (ciecu_multi_*)
//   TwoLevelConjugateGradients  CG preconditioned by a two-level cycle, on the device (ciecu_mgcg_*)
//   makeReordering / reorder    Cuthill-McKee maps and permutations on the device
//                               (linalg/packages/utilities/src/reorder.cpp:23-425, ciecu_graph.h)
// Each solver is the reference's ConjugateGradients algorithm
// (linalg/packages/solvers/impl/ConjugateGradients_impl.hpp:49-201) applied per
// system / per column / with another preconditioner.
#pragma once

#include "cie_cuda/linalg.hpp"
#include "ciecu_batch.h"
#include "ciecu_graph.h"
#include "ciecu_mg.h"
#include "ciecu_multi.h"

#include <vector>

namespace cie::cuda {

// Independent systems s = 0..S-1 in rows [rowOffsets[s], rowOffsets[s+1]) of one
// block-diagonal matrix (no entry may couple two systems); each has its own
// scalars and stopping decision.  Statistics per system.
class BatchedConjugateGradients {
public:
    using Space = CUDASpace<double>;
    using Statistics = SolverStatistics<double>;

    BatchedConjugateGradients(std::shared_ptr<CUDACSROperator<int, double>> pLhs, std::vector<int64_t> rowOffsets,
                              std::shared_ptr<DiagonalOperator<Space>> pPreconditioner, Statistics settings)
        : _pLhs(std::move(pLhs)), _pPreconditioner(std::move(pPreconditioner)), _offsets(std::move(rowOffsets)) {
        require(_offsets.size() >= 2, "BatchedConjugateGradients: at least one system");
        ciecu_batch raw = nullptr;
        check(ciecu_batch_create(_pLhs->handle(), static_cast<int64_t>(_offsets.size() - 1), _offsets.data(),
                                 _pPreconditioner->inverseDiagonal().data(), detail::to_c(settings), &raw));
        _solver = std::shared_ptr<ciecu_batch_s>(raw, [](ciecu_batch b) { ciecu_batch_destroy(b); });
    }

    // FP32 inner solves with FP64 refinement per system (innerTolerance: the drop of
    // the FP32 residual per refinement step; 0 returns to FP64).
    void setRefinement(double innerTolerance) { check(ciecu_batch_set_refinement(_solver.get(), innerTolerance)); }
    // delta in (0, 1): FP32 iterations per system with FP64 reliable updates
    // (ciecu_batch_set_reliable_updates); 0: off.
    void setReliableUpdates(double delta) { check(ciecu_batch_set_reliable_updates(_solver.get(), delta)); }
    std::vector<int64_t> refinements() const {
        std::vector<int64_t> out(systems());
        check(ciecu_batch_refinements(_solver.get(), out.data()));
        return out;
    }

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) {
        require(in.size() == out.size() && out.size() == _pLhs->matrix().rowCount,
                "BatchedConjugateGradients::product: incompatible vector sizes");
        std::vector<ciecu_statistics> s(_offsets.size() - 1);
        const int status = ciecu_batch_product(_solver.get(), inScale, in.data(), outScale, out.data(), s.data());
        _stats.clear();
        for (const auto& e : s)
            _stats.push_back(Statistics{static_cast<std::size_t>(e.iterationCount), e.absoluteResidual,
                                        e.relativeResidual});
        check(status);
    }
    const std::vector<Statistics>& getStats() const noexcept { return _stats; }
    std::size_t systems() const noexcept { return _offsets.size() - 1; }

private:
    std::shared_ptr<CUDACSROperator<int, double>> _pLhs;
    std::shared_ptr<DiagonalOperator<Space>> _pPreconditioner;
    std::vector<int64_t> _offsets;
    std::shared_ptr<ciecu_batch_s> _solver;
    std::vector<Statistics> _stats;
};

// k right-hand sides of one matrix: in / out are n x k row-major (entry (i, c) at
// i * k + c); column c is solved exactly as ConjugateGradients solves it alone.
class MultiRHSConjugateGradients {
public:
    using Space = CUDASpace<double>;
    using Statistics = SolverStatistics<double>;

    MultiRHSConjugateGradients(std::shared_ptr<CUDACSROperator<int, double>> pLhs, int rhsCount,
                               std::shared_ptr<DiagonalOperator<Space>> pPreconditioner, Statistics settings)
        : _pLhs(std::move(pLhs)), _pPreconditioner(std::move(pPreconditioner)), _k(rhsCount) {
        ciecu_multi raw = nullptr;
        check(ciecu_multi_create(_pLhs->handle(), rhsCount, _pPreconditioner->inverseDiagonal().data(),
                                 detail::to_c(settings), &raw));
        _solver = std::shared_ptr<ciecu_multi_s>(raw, [](ciecu_multi m) { ciecu_multi_destroy(m); });
    }

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) {
        require(in.size() == out.size() && out.size() == _pLhs->matrix().rowCount * static_cast<std::size_t>(_k),
                "MultiRHSConjugateGradients::product: vectors must hold n x k entries");
        std::vector<ciecu_statistics> s(static_cast<std::size_t>(_k));
        const int status = ciecu_multi_product(_solver.get(), inScale, in.data(), outScale, out.data(), s.data());
        _stats.clear();
        for (const auto& e : s)
            _stats.push_back(Statistics{static_cast<std::size_t>(e.iterationCount), e.absoluteResidual,
                                        e.relativeResidual});
        check(status);
    }
    const std::vector<Statistics>& getStats() const noexcept { return _stats; }
    int rhsCount() const noexcept { return _k; }
    // delta in (0, 1): FP32 iterations per column with FP64 reliable updates
    // (ciecu_multi_set_refinement); 0: FP64 iterations.
    void setRefinement(double delta) { check(ciecu_multi_set_refinement(_solver.get(), delta)); }
    std::vector<int64_t> refinements() const {
        std::vector<int64_t> out(static_cast<std::size_t>(_k));
        check(ciecu_multi_refinements(_solver.get(), out.data()));
        return out;
    }

private:
    std::shared_ptr<CUDACSROperator<int, double>> _pLhs;
    std::shared_ptr<DiagonalOperator<Space>> _pPreconditioner;
    int _k;
    std::shared_ptr<ciecu_multi_s> _solver;
    std::vector<Statistics> _stats;
};

// CG preconditioned by z = S r; z += P C(R (r - A z)); z += S (r - A z) on the
// device (ciecu_mgcg_create documents the cycle).  pSmoother32: optional FP32 copy
// of the fine matrix for single-precision smoothing.
class TwoLevelConjugateGradients : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    using Statistics = SolverStatistics<double>;

    TwoLevelConjugateGradients(std::shared_ptr<CUDACSROperator<int, double>> pFine,
                               std::shared_ptr<DiagonalOperator<Space>> pFineDiagonal,
                               std::shared_ptr<CUDACSROperator<int, double>> pProlongation,
                               std::shared_ptr<CUDACSROperator<int, double>> pRestriction,
                               std::shared_ptr<CUDACSROperator<int, double>> pCoarse,
                               std::shared_ptr<DiagonalOperator<Space>> pCoarseDiagonal, Statistics settings,
                               ciecu_mg_options options = ciecu_mg_options{2, 0.0, 30.0, 8, 1},
                               std::shared_ptr<CUDACSROperator<int, float>> pSmoother32 = nullptr)
        : _keep{pFine, pProlongation, pRestriction, pCoarse},
          _diagonals{pFineDiagonal, pCoarseDiagonal},
          _pSmoother32(std::move(pSmoother32)),
          _n(pFine->matrix().rowCount) {
        ciecu_mgcg raw = nullptr;
        check(ciecu_mgcg_create(pFine->handle(), pFineDiagonal->inverseDiagonal().data(),
                                _pSmoother32 ? _pSmoother32->handle() : nullptr, pProlongation->handle(),
                                pRestriction->handle(), pCoarse->handle(), pCoarseDiagonal->inverseDiagonal().data(),
                                options, detail::to_c(settings), &raw));
        _solver = std::shared_ptr<ciecu_mgcg_s>(raw, [](ciecu_mgcg m) { ciecu_mgcg_destroy(m); });
    }

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size() && out.size() == _n,
                "TwoLevelConjugateGradients::product: incompatible vector sizes");
        ciecu_statistics s{};
        const int status = ciecu_mgcg_product(_solver.get(), inScale, in.data(), outScale, out.data(), &s);
        _stats = Statistics{static_cast<std::size_t>(s.iterationCount), s.absoluteResidual, s.relativeResidual};
        check(status);
    }
    std::optional<Statistics> getStats() const noexcept { return _stats; }

private:
    std::vector<std::shared_ptr<CUDACSROperator<int, double>>> _keep;
    std::vector<std::shared_ptr<DiagonalOperator<Space>>> _diagonals;
    std::shared_ptr<CUDACSROperator<int, float>> _pSmoother32;
    std::size_t _n;
    std::shared_ptr<ciecu_mgcg_s> _solver;
    std::optional<Statistics> _stats;
};

enum class ReorderingStrategy { CuthillMcKee = 1, ReverseCuthillMcKee = 2 };

// makeReordering on the device: map[k] = the row placed at position k (any space
// of the matrix's stream).
template <class TSpace>
void makeReordering(const TSpace& space, CUDAView<int> map, const DeviceCSR<double, int>& m,
                    ReorderingStrategy strategy = ReorderingStrategy::CuthillMcKee) {
    require(map.size() == m.rowCount, "makeReordering: the map must hold one entry per row");
    check(ciecu_make_reordering(space.handle(), static_cast<int32_t>(m.rowCount), m.rowExtents, m.columnIndices,
                                static_cast<int>(strategy), map.data()));
}

// reorder<int,double,false> out of place: out holds rowCount + 1 row extents and
// nnz columns and entries.
inline void reorder(const CUDASpace<double>& space, CUDAView<const int> map, const DeviceCSR<double, int>& in,
                    CUDAView<int> outRowExtents, CUDAView<int> outColumnIndices, CUDAView<double> outEntries) {
    require(map.size() == in.rowCount && outRowExtents.size() == in.rowCount + 1 &&
                outColumnIndices.size() == in.nnz && outEntries.size() == in.nnz,
            "reorder: output sizes do not match the matrix");
    check(ciecu_reorder_csr(space.handle(), static_cast<int32_t>(in.rowCount), map.data(), in.rowExtents,
                            in.columnIndices, in.entries, outRowExtents.data(), outColumnIndices.data(),
                            outEntries.data()));
}

// reorder (out[i] = in[map[i]]) and reverseReorder (out[map[i]] = in[i]) of a vector.
inline void reorder(const CUDASpace<double>& space, CUDAView<const int> map, CUDAView<const double> in,
                    CUDAView<double> out, bool reverse = false) {
    require(map.size() == in.size() && in.size() == out.size(), "reorder: size mismatch");
    check(ciecu_reorder_vector(space.handle(), static_cast<int64_t>(in.size()), map.data(), reverse ? 1 : 0,
                               in.data(), out.data()));
}

}  // namespace cie::cuda
