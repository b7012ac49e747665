// cie_cuda/linalg.hpp -- C++ host API of the B200 linear-solve path, header-only,
// over the ciecu C-ABI (libciecu.so).  It mirrors the reference's linalg classes
// so that code written against them (e.g. executables/fem_examples/src/poisson2D/
// solver.cpp:238-288, solveSYCLCG) runs on the GPU with the space type swapped:
//
//   reference (linalg/packages/solvers)          here (namespace cie::cuda)
//   LinalgSpaceLike / SYCLSpace<T>               CUDASpace<T>, CUDAVector<T>, CUDAView<T>
//     (inc/LinalgSpace.hpp:10-35, inc/SYCLSpace.hpp:66-131)
//   LinearOperator<TSpace> (inc/LinearOperator.hpp:10-34)
//                                                LinearOperator<TSpace> (the reference's own
//                                                class when CIE_CUDA_WITH_CIE_LINALG is defined)
//   SYCLCSROperator<TI,TV> (src/SYCLCSROperator.cpp:32-89)
//                                                CUDACSROperator<TI,TV,TMV>
//   MaskedCSROperator (src/MaskedCSROperator.cpp:37-118)
//                                                CUDAMaskedCSROperator<TI,TV,TMask>
//   DiagonalOperator / makeDiagonalOperator (src/DiagonalOperator.cpp:37-88)
//                                                DiagonalOperator<CUDASpace<T>>, makeDiagonalOperator
//   JacobiOperator (src/JacobiOperator.cpp:36-62)
//                                                JacobiOperator<CUDASpace<T>>
//   ConjugateGradients (impl/ConjugateGradients_impl.hpp:49-201)
//                                                ConjugateGradients<CUDASpace<T>>
//   MaskedIdentityOperator (src/MaskedIdentityOperator.cpp:14-74)
//                                                MaskedIdentityOperator<CUDASpace<T>>
//   NestedProductOperator (impl/NestedProductOperator_impl.hpp:24-32)
//                                                NestedProductOperator<TSpace>
//   (no counterpart)                             MixedPrecisionCG: FP32-inner CG, FP64 reliable updates
//
// Semantics of every product: out <- inScale * out + outScale * Op(in).  A non-zero
// ciecu status becomes a cie::cuda::Exception carrying ciecu_last_error's message
// (the role of CIE_CHECK / CIE_THROW, cieutils/packages/macros/inc/checks.hpp:17-23).
// Operators are not re-entrant (they own scratch vectors), as in the reference.
// Arithmetic is provided for double (the whole path) and float (space operations
// and SpMV); index spaces (int, uint16_t) provide storage and copies only.
#pragma once

#include "ciecu.h"
#include "ciecu_mixed.h"

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#ifdef CIE_CUDA_WITH_CIE_LINALG
#include "packages/solvers/inc/LinearOperator.hpp"
#endif

namespace cie::cuda {

// ---- errors ----------------------------------------------------------------------

class Exception : public std::runtime_error {
public:
    Exception(int status, const std::string& message)
        : std::runtime_error(message + " (ciecu status " + std::to_string(status) + ")"), _status(status) {}
    int status() const noexcept { return _status; }

private:
    int _status;
};

inline void check(int status) {
    if (status == CIECU_OK) return;
    char buffer[1024] = {0};
    ciecu_last_error(buffer, static_cast<int>(sizeof(buffer)));
    throw Exception(status, buffer);
}

inline void require(bool condition, const char* message) {
    if (!condition) throw Exception(CIECU_ERR_ARGUMENT, message);
}

// ---- space, vectors and views ----------------------------------------------------

using SpaceHandle = std::shared_ptr<ciecu_space_s>;

// A ciecu space bound to `cudaStream` (nullptr: a stream the space creates and owns).
inline SpaceHandle makeSpaceHandle(void* cudaStream = nullptr) {
    ciecu_space raw = nullptr;
    check(ciecu_space_create(cudaStream, &raw));
    return SpaceHandle(raw, [](ciecu_space s) { ciecu_space_destroy(s); });
}

// Owning device vector (the role of SYCLVector / DeviceMemory, cieutils
// packages/concurrency/inc/sycl.hpp:33-71).  Move-only.
template <class T>
class CUDAVector {
public:
    CUDAVector() noexcept = default;
    CUDAVector(SpaceHandle space, std::size_t size) : _space(std::move(space)), _size(size) {
        if (_size) {
            void* p = nullptr;
            check(ciecu_alloc(_space.get(), sizeof(T) * _size, &p));
            _data = static_cast<T*>(p);
        }
    }
    CUDAVector(const CUDAVector&) = delete;
    CUDAVector& operator=(const CUDAVector&) = delete;
    CUDAVector(CUDAVector&& other) noexcept { swap(other); }
    CUDAVector& operator=(CUDAVector&& other) noexcept {
        if (this != &other) {
            CUDAVector tmp(std::move(other));
            swap(tmp);
        }
        return *this;
    }
    ~CUDAVector() {
        if (_data) ciecu_free(_space.get(), _data);
    }
    T* get() noexcept { return _data; }
    const T* get() const noexcept { return _data; }
    std::size_t size() const noexcept { return _size; }

private:
    void swap(CUDAVector& other) noexcept {
        std::swap(_space, other._space);
        std::swap(_data, other._data);
        std::swap(_size, other._size);
    }
    SpaceHandle _space;
    T* _data = nullptr;
    std::size_t _size = 0;
};

// Non-owning device view; CUDAView<T> converts to CUDAView<const T>.
template <class T>
class CUDAView {
public:
    CUDAView() noexcept = default;
    CUDAView(T* data, std::size_t size) noexcept : _data(data), _size(size) {}
    template <class U, class = std::enable_if_t<std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
    CUDAView(CUDAView<U> other) noexcept : _data(other.data()), _size(other.size()) {}
    T* data() const noexcept { return _data; }
    std::size_t size() const noexcept { return _size; }

private:
    T* _data = nullptr;
    std::size_t _size = 0;
};

template <class T>
class CUDASpace {
public:
    using Value = T;
    using Vector = CUDAVector<T>;
    using VectorView = CUDAView<T>;
    using ConstVectorView = CUDAView<const T>;

    // A space on a new stream owned by the space, or on the caller's stream.
    explicit CUDASpace(void* cudaStream = nullptr) : _handle(makeSpaceHandle(cudaStream)) {}
    // Share the stream of another space (value and index spaces of one solve,
    // like the shared queue of solver.cpp:243-244).
    explicit CUDASpace(SpaceHandle handle) : _handle(std::move(handle)) {}

    static VectorView view(Vector& v) noexcept { return VectorView(v.get(), v.size()); }
    static ConstVectorView view(const Vector& v) noexcept { return ConstVectorView(v.get(), v.size()); }
    static std::size_t size(ConstVectorView v) noexcept { return v.size(); }

    Vector makeVector(std::size_t size) const { return Vector(_handle, size); }

    Value innerProduct(ConstVectorView left, ConstVectorView right) const {
        require(left.size() == right.size(), "innerProduct: size mismatch");
        double result = 0.0;
        if constexpr (std::is_same_v<T, double>)
            check(ciecu_dot_f64(h(), n(left), left.data(), right.data(), &result));
        else if constexpr (std::is_same_v<T, float>)
            check(ciecu_dot_f32(h(), n(left), left.data(), right.data(), &result));
        else
            static_assert(sizeof(T) == 0, "innerProduct: double or float spaces only");
        return static_cast<Value>(result);
    }
    // target <- scale * target (.) source  (elementwise; DefaultSpace.cpp:81-106)
    void scale(VectorView target, ConstVectorView source, Value scale) const {
        require(target.size() == source.size(), "scale: size mismatch");
        if constexpr (std::is_same_v<T, double>)
            check(ciecu_scale_elementwise_f64(h(), n(target), target.data(), source.data(), scale));
        else
            check(ciecu_scale_elementwise_f32(h(), n(target), target.data(), source.data(), scale));
    }
    void scale(VectorView v, Value value) const {
        if constexpr (std::is_same_v<T, double>)
            check(ciecu_scale_f64(h(), n(v), v.data(), value));
        else
            check(ciecu_scale_f32(h(), n(v), v.data(), value));
    }
    // target <- target + scale * source
    void add(VectorView target, ConstVectorView source, Value scale) const {
        require(target.size() == source.size(), "add: size mismatch");
        if constexpr (std::is_same_v<T, double>)
            check(ciecu_add_f64(h(), n(target), target.data(), source.data(), scale));
        else
            check(ciecu_add_f32(h(), n(target), target.data(), source.data(), scale));
    }
    void assign(VectorView target, ConstVectorView source) const {
        require(target.size() == source.size(), "assign: size mismatch");
        check(ciecu_memcpy_d2d(h(), target.data(), source.data(), sizeof(T) * target.size()));
    }
    // host -> device and device -> host (SYCLSpace::assign overloads)
    void assign(VectorView target, std::span<const T> source) const {
        require(target.size() == source.size(), "assign: size mismatch");
        check(ciecu_memcpy_h2d(h(), target.data(), source.data(), sizeof(T) * target.size()));
    }
    void assign(std::span<T> target, ConstVectorView source) const {
        require(target.size() == source.size(), "assign: size mismatch");
        check(ciecu_memcpy_d2h(h(), target.data(), source.data(), sizeof(T) * source.size()));
    }
    void fill(VectorView v, Value value) const {
        if constexpr (std::is_same_v<T, double>)
            check(ciecu_fill_f64(h(), n(v), v.data(), value));
        else if constexpr (std::is_same_v<T, float>)
            check(ciecu_fill_f32(h(), n(v), v.data(), value));
        else
            static_assert(sizeof(T) == 0, "fill: double or float spaces only");
    }

    void synchronize() const { check(ciecu_space_synchronize(h())); }
    ciecu_space handle() const noexcept { return _handle.get(); }
    const SpaceHandle& sharedHandle() const noexcept { return _handle; }

private:
    ciecu_space h() const noexcept { return _handle.get(); }
    static int64_t n(ConstVectorView v) noexcept { return static_cast<int64_t>(v.size()); }
    SpaceHandle _handle;
};

// ---- operators -------------------------------------------------------------------

#ifdef CIE_CUDA_WITH_CIE_LINALG
template <class TSpace>
using LinearOperator = ::cie::linalg::LinearOperator<TSpace>;
#else
// out <- inScale * out + outScale * Op(in)  (LinearOperator.hpp:15-33)
template <class TSpace>
class LinearOperator {
public:
    virtual ~LinearOperator() = default;
    virtual void product(typename TSpace::Value inScale, typename TSpace::ConstVectorView in,
                         typename TSpace::Value outScale, typename TSpace::VectorView out) = 0;
};
#endif

// Device CSR arrays (the CSRView of the reference over device memory): row
// extents (rowCount + 1), column indices and entries, int32 indices.
template <class TValue, class TIndex = int>
struct DeviceCSR {
    std::size_t rowCount = 0, columnCount = 0, nnz = 0;
    const TIndex* rowExtents = nullptr;
    const TIndex* columnIndices = nullptr;
    const TValue* entries = nullptr;

    // From any CSRView-shaped object (rowCount(), columnCount(), rowExtents(),
    // columnIndices(), entries() spans) whose arrays live on the device.
    template <class TView>
    static DeviceCSR fromView(const TView& view) {
        DeviceCSR m;
        m.rowCount = view.rowCount();
        m.columnCount = view.columnCount();
        m.nnz = view.entries().size();
        m.rowExtents = view.rowExtents().data();
        m.columnIndices = view.columnIndices().data();
        m.entries = view.entries().data();
        return m;
    }
};

using CSRHandle = std::shared_ptr<ciecu_csr_s>;

template <class TValue, class TIndex>
CSRHandle makeCSRHandle(const DeviceCSR<TValue, TIndex>& m, const SpaceHandle& space) {
    static_assert(std::is_same_v<std::remove_const_t<TIndex>, int> || std::is_same_v<std::remove_const_t<TIndex>, int32_t>,
                  "CSR indices are int32");
    static_assert(std::is_same_v<std::remove_const_t<TValue>, double> || std::is_same_v<std::remove_const_t<TValue>, float>,
                  "CSR entries are double or float");
    require(m.rowCount <= static_cast<std::size_t>(std::numeric_limits<int32_t>::max()), "CSR: too many rows");
    ciecu_csr raw = nullptr;
    check(ciecu_csr_create(space.get(), static_cast<int32_t>(m.rowCount), static_cast<int32_t>(m.columnCount),
                           static_cast<int64_t>(m.nnz), m.rowExtents, m.columnIndices, m.entries,
                           std::is_same_v<std::remove_const_t<TValue>, double> ? CIECU_F64 : CIECU_F32, &raw));
    // a CSR handle may outlive nothing but its space: keep the space alive with it
    return CSRHandle(raw, [space](ciecu_csr c) { ciecu_csr_destroy(c); });
}

// SpMV over a device CSR matrix (CSROperator.cpp:33-111; scale special cases and
// the (-1,-1) -> A*in - out combination of :78-110 included).
template <class TIndex, class TValue, class TMatrixValue = TValue>
class CUDACSROperator : public LinearOperator<CUDASpace<TValue>> {
    static_assert(std::is_same_v<TValue, TMatrixValue>, "matrix and vector value types must match");

public:
    using Space = CUDASpace<TValue>;

    CUDACSROperator(const DeviceCSR<TMatrixValue, TIndex>& lhs, std::shared_ptr<Space> pSpace)
        : _lhs(lhs), _pSpace(std::move(pSpace)), _csr(makeCSRHandle(lhs, _pSpace->sharedHandle())) {}
    template <class TView, class = decltype(std::declval<const TView&>().rowExtents())>
    CUDACSROperator(const TView& deviceView, std::shared_ptr<Space> pSpace)
        : CUDACSROperator(DeviceCSR<TMatrixValue, TIndex>::fromView(deviceView), std::move(pSpace)) {}

    void product(TValue inScale, typename Space::ConstVectorView in, TValue outScale,
                 typename Space::VectorView out) override {
        require(in.size() == _lhs.columnCount && out.size() == _lhs.rowCount,
                "CSROperator::product: inconsistent input vector sizes");
        if constexpr (std::is_same_v<TValue, double>)
            check(ciecu_csr_spmv_f64(_csr.get(), inScale, in.data(), outScale, out.data()));
        else
            check(ciecu_csr_spmv_f32(_csr.get(), inScale, in.data(), outScale, out.data()));
    }

    const DeviceCSR<TMatrixValue, TIndex>& matrix() const noexcept { return _lhs; }
    ciecu_csr handle() const noexcept { return _csr.get(); }
    const std::shared_ptr<Space>& space() const noexcept { return _pSpace; }

private:
    DeviceCSR<TMatrixValue, TIndex> _lhs;
    std::shared_ptr<Space> _pSpace;
    CSRHandle _csr;
};

// SpMV restricted to rows / columns with mask < threshold; masked rows receive
// combine(inScale, out, outScale, 0) (MaskedCSROperator.cpp:37-118, CPU semantics).
template <class TIndex, class TValue, class TMask = uint16_t>
class CUDAMaskedCSROperator : public CUDACSROperator<TIndex, TValue> {
    static_assert(std::is_same_v<TMask, uint16_t>, "masks are uint16");
    static_assert(std::is_same_v<TValue, double>, "masked operators are FP64");

public:
    using Space = CUDASpace<TValue>;
    CUDAMaskedCSROperator(const DeviceCSR<TValue, TIndex>& lhs, CUDAView<const TMask> mask, TMask threshold,
                          std::shared_ptr<Space> pSpace)
        : CUDACSROperator<TIndex, TValue>(lhs, std::move(pSpace)), _mask(mask), _threshold(threshold) {
        require(mask.size() == lhs.rowCount, "MaskedCSROperator: mask size must equal the row count");
    }

    void product(TValue inScale, typename Space::ConstVectorView in, TValue outScale,
                 typename Space::VectorView out) override {
        require(in.size() == this->matrix().columnCount && out.size() == this->matrix().rowCount,
                "MaskedCSROperator::product: inconsistent input vector sizes");
        check(ciecu_csr_masked_spmv_f64(this->handle(), _mask.data(), _threshold, inScale, in.data(), outScale,
                                        out.data()));
    }
    CUDAView<const TMask> mask() const noexcept { return _mask; }
    TMask threshold() const noexcept { return _threshold; }

private:
    CUDAView<const TMask> _mask;
    TMask _threshold;
};

template <class TSpace>
class DiagonalOperator;

// out <- inScale * out + outScale * (in (.) D^-1)  (DiagonalOperator.cpp:37-53).
// Owns its inverse diagonal, like the reference (moved in, :27-34).
template <>
class DiagonalOperator<CUDASpace<double>> : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    DiagonalOperator(Space::Vector&& inverseDiagonal, std::shared_ptr<const Space> pSpace) noexcept
        : _inverseDiagonal(std::move(inverseDiagonal)), _pSpace(std::move(pSpace)) {}

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size() && out.size() == _inverseDiagonal.size(),
                "DiagonalOperator::product: inconsistent input vector sizes");
        check(ciecu_diagonal_apply_f64(_pSpace->handle(), static_cast<int64_t>(out.size()), _inverseDiagonal.get(),
                                       inScale, in.data(), outScale, out.data()));
    }
    Space::ConstVectorView inverseDiagonal() const noexcept { return Space::view(_inverseDiagonal); }

private:
    Space::Vector _inverseDiagonal;
    std::shared_ptr<const Space> _pSpace;
};

// makeDiagonalOperator (DiagonalOperator.cpp:56-88): throws, naming the first row,
// on a missing or zero diagonal entry.
template <class TValue, class TIndex, class TMatrixValue>
DiagonalOperator<CUDASpace<TValue>> makeDiagonalOperator(const CUDACSROperator<TIndex, TValue, TMatrixValue>& matrix,
                                                         std::shared_ptr<const CUDASpace<TValue>> pSpace) {
    auto inverse = pSpace->makeVector(matrix.matrix().rowCount);
    check(ciecu_diagonal_inverse_f64(matrix.handle(), inverse.get()));
    return DiagonalOperator<CUDASpace<TValue>>(std::move(inverse), std::move(pSpace));
}

template <class TValue, class TIndex, class TMatrixValue>
DiagonalOperator<CUDASpace<TValue>> makeDiagonalOperator(const DeviceCSR<TMatrixValue, TIndex>& matrix,
                                                         std::shared_ptr<const CUDASpace<TValue>> pSpace) {
    auto handle = makeCSRHandle(matrix, pSpace->sharedHandle());
    auto inverse = pSpace->makeVector(matrix.rowCount);
    check(ciecu_diagonal_inverse_f64(handle.get(), inverse.get()));
    return DiagonalOperator<CUDASpace<TValue>>(std::move(inverse), std::move(pSpace));
}

// out <- combine(inScale, out, outScale, mask < threshold ? in : 0)
// (MaskedIdentityOperator.cpp:14-74).
template <class TSpace>
class MaskedIdentityOperator;

template <>
class MaskedIdentityOperator<CUDASpace<double>> : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    MaskedIdentityOperator(std::shared_ptr<const Space> pSpace, CUDAView<const uint16_t> mask, uint16_t threshold)
        : _pSpace(std::move(pSpace)), _mask(mask), _threshold(threshold) {}
    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size() && out.size() == _mask.size(),
                "MaskedIdentityOperator::product: inconsistent input vector sizes");
        check(ciecu_masked_identity_f64(_pSpace->handle(), static_cast<int64_t>(out.size()), _mask.data(),
                                        _threshold, inScale, in.data(), outScale, out.data()));
    }

private:
    std::shared_ptr<const Space> _pSpace;
    CUDAView<const uint16_t> _mask;
    uint16_t _threshold;
};

// lhs(rhs(in)) through an owned intermediate of rowCount entries
// (NestedProductOperator_impl.hpp:24-32).
template <class TSpace>
class NestedProductOperator : public LinearOperator<TSpace> {
public:
    NestedProductOperator(std::shared_ptr<TSpace> pSpace, std::shared_ptr<LinearOperator<TSpace>> pLhs,
                          std::shared_ptr<LinearOperator<TSpace>> pRhs, std::size_t rowCount)
        : _pSpace(std::move(pSpace)), _pLhs(std::move(pLhs)), _pRhs(std::move(pRhs)),
          _buffer(_pSpace->makeVector(rowCount)) {
        _pSpace->fill(TSpace::view(_buffer), 0);
    }
    void product(typename TSpace::Value inScale, typename TSpace::ConstVectorView in, typename TSpace::Value outScale,
                 typename TSpace::VectorView out) override {
        _pRhs->product(0, in, 1, TSpace::view(_buffer));
        _pLhs->product(inScale, TSpace::view(std::as_const(_buffer)), outScale, out);
    }

private:
    std::shared_ptr<TSpace> _pSpace;
    std::shared_ptr<LinearOperator<TSpace>> _pLhs, _pRhs;
    typename TSpace::Vector _buffer;
};

// Damped Jacobi from x0 = 0 (JacobiOperator.cpp:36-62).  With a (masked) CSR
// operator and a DiagonalOperator each sweep is one fused kernel; any other pair
// runs the reference's composition of products and space operations.
template <class TSpace>
class JacobiOperator;

template <>
class JacobiOperator<CUDASpace<double>> : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    JacobiOperator(std::shared_ptr<Space> pSpace, std::size_t size, std::shared_ptr<LinearOperator<Space>> pLhs,
                   std::shared_ptr<LinearOperator<Space>> pInverseDiagonal, std::size_t iterations = 1,
                   double relaxation = 1)
        : _pSpace(std::move(pSpace)), _size(size), _pLhs(std::move(pLhs)),
          _pInverseDiagonal(std::move(pInverseDiagonal)), _iterations(iterations), _relaxation(relaxation),
          _work(_pSpace->makeVector(2 * size)) {}

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size() && out.size() == _size, "inconsistent input vector sizes");
        auto* csr = dynamic_cast<CUDACSROperator<int, double>*>(_pLhs.get());
        auto* masked = dynamic_cast<CUDAMaskedCSROperator<int, double>*>(_pLhs.get());
        auto* diagonal = dynamic_cast<DiagonalOperator<Space>*>(_pInverseDiagonal.get());
        if (csr && diagonal) {
            check(ciecu_jacobi_f64(csr->handle(), diagonal->inverseDiagonal().data(),
                                   masked ? masked->mask().data() : nullptr, masked ? masked->threshold() : 0,
                                   static_cast<int64_t>(_iterations), _relaxation, inScale, in.data(), outScale,
                                   out.data(), _work.get()));
            return;
        }
        auto memory = _pSpace->makeVector(_size), residual = _pSpace->makeVector(_size);
        _pSpace->assign(Space::view(memory), out);
        _pSpace->fill(out, 0);
        for (std::size_t k = 0; k < _iterations; ++k) {
            _pSpace->assign(Space::view(residual), in);
            _pLhs->product(1, out, -1, Space::view(residual));                   // in - A x  (the -1,-1 rule not used)
            _pInverseDiagonal->product(1, Space::view(std::as_const(residual)), _relaxation, out);
        }
        _pSpace->scale(out, outScale);
        _pSpace->add(out, Space::view(std::as_const(memory)), inScale);
    }

private:
    std::shared_ptr<Space> _pSpace;
    std::size_t _size;
    std::shared_ptr<LinearOperator<Space>> _pLhs, _pInverseDiagonal;
    std::size_t _iterations;
    double _relaxation;
    Space::Vector _work;
};

// Statistics of the iterative solvers (IterativeSolver.hpp:21-25).
template <class TValue>
struct SolverStatistics {
    std::size_t iterationCount = 0;
    TValue absoluteResidual = 0;
    TValue relativeResidual = 0;
};

namespace detail {
// utils::Comparison<double>::less with the default tolerances (Comparison_impl.hpp:32-63).
inline bool float_less(double a, double b) {
    const double norm = std::fmin(std::fabs(a) + std::fabs(b), std::numeric_limits<double>::max());
    const double tol = std::fmax(std::numeric_limits<double>::min(), std::numeric_limits<double>::epsilon() * norm);
    return a < b && !(std::fabs(a - b) < tol);
}
inline ciecu_statistics to_c(const SolverStatistics<double>& s) {
    return ciecu_statistics{static_cast<int64_t>(s.iterationCount), s.absoluteResidual, s.relativeResidual};
}
}  // namespace detail

// Preconditioned conjugate gradients (ConjugateGradients_impl.hpp:49-201).  A
// CUDACSROperator with a DiagonalOperator (or no) preconditioner runs the fused,
// device-resident solver; any other combination runs the reference algorithm
// composed of operator products and space operations, on the GPU.
template <class TSpace>
class ConjugateGradients;

template <>
class ConjugateGradients<CUDASpace<double>> : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    using Statistics = SolverStatistics<double>;

    ConjugateGradients(std::shared_ptr<LinearOperator<Space>> pLhs, std::shared_ptr<Space> pSpace,
                       std::shared_ptr<LinearOperator<Space>> pPreconditioner = nullptr, Statistics settings = {},
                       int verbosity = 0)
        : _pLhs(std::move(pLhs)), _pPreconditioner(std::move(pPreconditioner)), _pSpace(std::move(pSpace)),
          _settings(settings), _verbosity(verbosity) {
        rebuild();
    }

    void configure(Statistics settings) {
        _settings = settings;
        rebuild();
    }
    Statistics getConfiguration() const noexcept { return _settings; }
    std::optional<Statistics> getStats() const noexcept { return _stats; }
    bool fused() const noexcept { return static_cast<bool>(_solver); }
    // The fused device solver (null for the generic composition).
    ciecu_pcg handle() const noexcept { return _solver.get(); }

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size(), "ConjugateGradients::product: incompatible vector sizes");
        if (_solver) {
            ciecu_statistics s{};
            const int status = ciecu_pcg_product(_solver.get(), inScale, in.data(), outScale, out.data(), &s);
            _stats = Statistics{static_cast<std::size_t>(s.iterationCount), s.absoluteResidual, s.relativeResidual};
            check(status);
            return;
        }
        generic(inScale, in, outScale, out);
    }

private:
    void rebuild() {
        _solver.reset();
        auto* csr = dynamic_cast<CUDACSROperator<int, double>*>(_pLhs.get());
        auto* masked = dynamic_cast<CUDAMaskedCSROperator<int, double>*>(_pLhs.get());
        auto* diagonal = dynamic_cast<DiagonalOperator<Space>*>(_pPreconditioner.get());
        if (csr && !masked && (!_pPreconditioner || diagonal)) {
            ciecu_pcg raw = nullptr;
            check(ciecu_pcg_create(csr->handle(), diagonal ? diagonal->inverseDiagonal().data() : nullptr,
                                   detail::to_c(_settings), _verbosity, &raw));
            _solver = std::shared_ptr<ciecu_pcg_s>(raw, [](ciecu_pcg p) { ciecu_pcg_destroy(p); });
        }
    }

    void generic(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) {
        const Space& sp = *_pSpace;
        const std::size_t n = out.size();
        Statistics stats{0, std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
        auto solution = sp.makeVector(n);
        sp.assign(Space::view(solution), out);
        auto x = Space::view(solution);
        if (_settings.iterationCount) {
            auto search = sp.makeVector(n), searchProduct = sp.makeVector(n), residual = sp.makeVector(n);
            Space::Vector z;
            auto p = Space::view(search), q = Space::view(searchProduct), r = Space::view(residual);
            sp.fill(q, 0);
            sp.assign(r, in);
            _pLhs->product(1, x, -1, r);  // r = b - A x0
            double rr = sp.innerProduct(r, r);
            const double initial = std::sqrt(rr);
            stats.absoluteResidual = initial;
            stats.relativeResidual = 1.0;
            bool done = detail::float_less(stats.absoluteResidual, _settings.absoluteResidual) ||
                        detail::float_less(stats.relativeResidual, _settings.relativeResidual);
            double rz = rr;
            if (!done) {
                if (_pPreconditioner) {
                    z = sp.makeVector(n);
                    _pPreconditioner->product(0, r, 1, Space::view(z));
                    rz = sp.innerProduct(r, Space::view(std::as_const(z)));
                    sp.assign(p, Space::view(std::as_const(z)));
                    if (!(0 < rz)) throw Exception(CIECU_ERR_BREAKDOWN, "preconditioned norm vanished in iteration 0");
                } else {
                    sp.assign(p, r);
                    if (!(0 < rz)) throw Exception(CIECU_ERR_BREAKDOWN, "residual norm vanished in iteration 0");
                }
            }
            while (!done && stats.iterationCount < _settings.iterationCount) {
                _pLhs->product(0, p, 1, q);
                const double den = sp.innerProduct(p, q);
                if (!(0 < den)) {
                    _stats = stats;
                    throw Exception(CIECU_ERR_BREAKDOWN,
                                    "p^T A p vanished in iteration " + std::to_string(stats.iterationCount));
                }
                const double alpha = rz / den;
                sp.add(x, p, alpha);
                sp.add(r, q, -alpha);
                rr = sp.innerProduct(r, r);
                const double previous = rz;
                if (_pPreconditioner) {
                    _pPreconditioner->product(0, r, 1, Space::view(z));
                    rz = sp.innerProduct(r, Space::view(std::as_const(z)));
                } else {
                    rz = rr;
                }
                sp.scale(p, rz / previous);
                sp.add(p, _pPreconditioner ? Space::view(std::as_const(z)) : Space::ConstVectorView(r), 1);
                stats.absoluteResidual = std::sqrt(rr);
                stats.relativeResidual = stats.absoluteResidual / initial;
                if (detail::float_less(stats.absoluteResidual, _settings.absoluteResidual) ||
                    detail::float_less(stats.relativeResidual, _settings.relativeResidual))
                    break;
                ++stats.iterationCount;
            }
        }
        // out = inScale * out + outScale * x  (ConjugateGradients_impl.hpp:190-198)
        if (inScale == 1) {
            sp.add(out, x, outScale);
        } else if (inScale == 0) {
            sp.assign(out, x);
            sp.scale(out, outScale);
        } else {
            sp.scale(out, inScale);
            sp.add(out, x, outScale);
        }
        _stats = stats;
    }

    std::shared_ptr<LinearOperator<Space>> _pLhs, _pPreconditioner;
    std::shared_ptr<Space> _pSpace;
    Statistics _settings;
    int _verbosity;
    std::optional<Statistics> _stats;
    std::shared_ptr<ciecu_pcg_s> _solver;
};

// Mixed-precision PCG (no reference counterpart): FP32 inner CG over an FP32
// copy of the matrix (diagonal storage or SELL-32), FP64 reliable updates; stops
// on the true FP64 residual.  Same product semantics and statistics as
// ConjugateGradients.
class MixedPrecisionCG : public LinearOperator<CUDASpace<double>> {
public:
    using Space = CUDASpace<double>;
    using Statistics = SolverStatistics<double>;

    MixedPrecisionCG(std::shared_ptr<CUDACSROperator<int, double>> pLhs,
                     std::shared_ptr<DiagonalOperator<Space>> pPreconditioner, Statistics settings,
                     ciecu_mixed_options options = ciecu_mixed_options{0, 0.1, 1, 0, 0, 0})
        : _pLhs(std::move(pLhs)), _pPreconditioner(std::move(pPreconditioner)) {
        ciecu_mixed raw = nullptr;
        check(ciecu_mixed_create(_pLhs->handle(), _pPreconditioner->inverseDiagonal().data(),
                                 detail::to_c(settings), options, &raw));
        _solver = std::shared_ptr<ciecu_mixed_s>(raw, [](ciecu_mixed m) { ciecu_mixed_destroy(m); });
    }

    void product(double inScale, Space::ConstVectorView in, double outScale, Space::VectorView out) override {
        require(in.size() == out.size() && out.size() == _pLhs->matrix().rowCount,
                "MixedPrecisionCG::product: incompatible vector sizes");
        ciecu_mixed_statistics s{};
        const int status = ciecu_mixed_product(_solver.get(), inScale, in.data(), outScale, out.data(), &s);
        _stats = Statistics{static_cast<std::size_t>(s.iterationCount), s.absoluteResidual, s.relativeResidual};
        _refinements = static_cast<std::size_t>(s.refinements);
        check(status);
    }
    std::optional<Statistics> getStats() const noexcept { return _stats; }
    std::size_t refinements() const noexcept { return _refinements; }
    // Kernels per inner iteration of the solver's loop (3, 2 or 1; options.fuseDirection).
    int kernelsPerIteration() const {
        int k = 0;
        check(ciecu_mixed_form(_solver.get(), &k));
        return k;
    }

private:
    std::shared_ptr<CUDACSROperator<int, double>> _pLhs;
    std::shared_ptr<DiagonalOperator<Space>> _pPreconditioner;
    std::shared_ptr<ciecu_mixed_s> _solver;
    std::optional<Statistics> _stats;
    std::size_t _refinements = 0;
};

}  // namespace cie::cuda
