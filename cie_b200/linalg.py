"""Python mirror of the kelofm/cie linalg operator API over the CUDA backend.

Names, argument meaning and error behaviour follow the reference:
  LinearOperator.product(inScale, in, outScale, out):  out <- inScale*out + outScale*Op(in)
      (linalg/packages/solvers/inc/LinearOperator.hpp:10-34)
  CUDASpace satisfies LinalgSpaceLike (linalg/packages/solvers/inc/LinalgSpace.hpp:10-35)
  CSROperator, MaskedCSROperator, DiagonalOperator / makeDiagonalOperator,
  JacobiOperator, MaskedIdentityOperator, NestedProductOperator, ConjugateGradients.
Vectors are torch CUDA tensors (torch provides device memory and streams only);
every operation runs in the libciecu.so kernels.  Failures raise CiecuError,
the counterpart of cie::Exception.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import Statistics, MixedOptions, MixedStatistics, call, CiecuError

__all__ = [
    "CUDASpace", "CSRMatrix", "LinearOperator", "CSROperator", "MaskedCSROperator", "DiagonalOperator",
    "makeDiagonalOperator", "JacobiOperator", "MaskedIdentityOperator", "NestedProductOperator",
    "ChebyshevOperator", "ConjugateGradients", "MixedPrecisionCG", "Statistics", "CiecuError", "launch_count",
]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def launch_count():
    """Kernels launched by libciecu.so since it was loaded."""
    return int(_lib.load().ciecu_kernel_launch_count())


class CUDASpace:
    """Device vector space on one CUDA stream (the SYCLSpace counterpart)."""

    def __init__(self, dtype=torch.float64, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("CUDASpace needs a CUDA device (there is no CPU fallback)")
        _lib.load()
        self.dtype = dtype
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.stream = torch.cuda.Stream(self.device)
        handle = ctypes.c_void_p()
        call("ciecu_space_create", ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(handle))
        self.handle = handle
        self._sfx = "f64" if dtype == torch.float64 else "f32"

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                _lib.load().ciecu_space_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    # -- stream ordering with torch's current stream ---------------------------
    def enter(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))

    def leave(self):
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def synchronize(self):
        call("ciecu_space_synchronize", self.handle)

    # -- LinalgSpaceLike ---------------------------------------------------------
    @staticmethod
    def view(vector):
        return vector

    @staticmethod
    def size(view):
        return int(view.numel())

    def makeVector(self, size):
        return torch.empty(int(size), dtype=self.dtype, device=self.device)

    def _check(self, *vs):
        for v in vs:
            if not (v.is_cuda and v.dtype == self.dtype and v.is_contiguous()):
                raise CiecuError(1, "expected a contiguous %s CUDA vector" % self.dtype)

    def innerProduct(self, left, right):
        self._check(left, right)
        if left.numel() != right.numel():
            raise CiecuError(1, "incompatible vector sizes %d != %d" % (left.numel(), right.numel()))
        out = ctypes.c_double()
        self.enter()
        call("ciecu_dot_" + self._sfx, self.handle, left.numel(), _ptr(left), _ptr(right), ctypes.byref(out))
        return out.value

    def scale(self, target, source_or_value, scale=None):
        """scale(target, source, alpha): target = alpha * target (.) source (elementwise);
        scale(view, value): view *= value."""
        self.enter()
        if scale is None:
            self._check(target)
            call("ciecu_scale_" + self._sfx, self.handle, target.numel(), _ptr(target), float(source_or_value))
        else:
            self._check(target, source_or_value)
            call("ciecu_scale_elementwise_" + self._sfx, self.handle, target.numel(), _ptr(target),
                 _ptr(source_or_value), float(scale))
        self.leave()

    def add(self, target, source, scale):
        self._check(target, source)
        self.enter()
        call("ciecu_add_" + self._sfx, self.handle, target.numel(), _ptr(target), _ptr(source), float(scale))
        self.leave()

    def assign(self, target, source):
        """Device<-device, device<-host (numpy / CPU tensor) and host<-device."""
        self.enter()
        if isinstance(target, torch.Tensor) and target.is_cuda and isinstance(source, torch.Tensor) and source.is_cuda:
            self._check(target, source)
            call("ciecu_assign_" + self._sfx, self.handle, target.numel(), _ptr(target), _ptr(source))
        elif isinstance(target, torch.Tensor) and target.is_cuda:
            host = np.ascontiguousarray(np.asarray(source), dtype=np.float64 if self._sfx == "f64" else np.float32)
            call("ciecu_memcpy_h2d", self.handle, _ptr(target), host.ctypes.data_as(ctypes.c_void_p), host.nbytes)
        else:
            host = np.asarray(target)
            call("ciecu_memcpy_d2h", self.handle, host.ctypes.data_as(ctypes.c_void_p), _ptr(source),
                 source.numel() * source.element_size())
        self.leave()

    def fill(self, view, value):
        self._check(view)
        self.enter()
        call("ciecu_fill_" + self._sfx, self.handle, view.numel(), _ptr(view), float(value))
        self.leave()


class CSRMatrix:
    """Device CSR arrays (the storage a device CSRView points at,
    linalg/packages/utilities/inc/CSRView.hpp:11-86)."""

    def __init__(self, columnCount, rowExtents, columnIndices, entries):
        self.columnCount = int(columnCount)
        self.rowExtents = rowExtents
        self.columnIndices = columnIndices
        self.entries = entries

    @classmethod
    def from_host(cls, columnCount, rowExtents, columnIndices, entries, dtype=torch.float64, device="cuda"):
        return cls(columnCount,
                   torch.as_tensor(np.asarray(rowExtents, dtype=np.int32)).to(device),
                   torch.as_tensor(np.asarray(columnIndices, dtype=np.int32)).to(device),
                   torch.as_tensor(np.asarray(entries)).to(device=device, dtype=dtype))

    def rowCount(self):
        return int(self.rowExtents.numel()) - 1

    def nnz(self):
        return int(self.columnIndices.numel())

    def astype(self, dtype):
        return CSRMatrix(self.columnCount, self.rowExtents, self.columnIndices, self.entries.to(dtype))


class LinearOperator:
    def product(self, inScale, in_, outScale, out):
        raise NotImplementedError


class _CSRHandle:
    def __init__(self, matrix, space):
        if matrix.columnIndices.numel() != matrix.entries.numel():
            raise CiecuError(1, "number of column indices (%d) is inconsistent with the number of entries (%d) "
                                "in the provided CSR matrix" % (matrix.columnIndices.numel(), matrix.entries.numel()))
        if matrix.rowExtents.numel() < 1:
            raise CiecuError(1, "expecting the row extents of a CSR matrix to have at least 1 entry, but it has none")
        self.matrix = matrix
        self.space = space
        vt = 0 if matrix.entries.dtype == torch.float64 else 1
        h = ctypes.c_void_p()
        space.enter()
        call("ciecu_csr_create", space.handle, matrix.rowCount(), matrix.columnCount, matrix.nnz(),
             _ptr(matrix.rowExtents), _ptr(matrix.columnIndices), _ptr(matrix.entries), vt, ctypes.byref(h))
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                _lib.load().ciecu_csr_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def kernel(self):
        k = ctypes.c_int()
        call("ciecu_csr_get_kernel", self.handle, ctypes.byref(k))
        return k.value

    def set_kernel(self, k):
        call("ciecu_csr_set_kernel", self.handle, int(k))

    def diagonals(self):
        """Diagonals of the matrix's diagonal-storage copy (0: not a few-diagonal matrix)."""
        d = ctypes.c_int()
        call("ciecu_csr_diagonals", self.handle, ctypes.byref(d))
        return d.value


class CSROperator(LinearOperator):
    """CSROperator<int,T>::product (linalg/packages/solvers/src/CSROperator.cpp:33-111)."""

    def __init__(self, lhs, space):
        self.lhs = lhs
        self.space = space
        self.csr = _CSRHandle(lhs, space)

    def product(self, inScale, in_, outScale, out):
        rows, cols = self.lhs.rowCount(), self.lhs.columnCount
        if out.numel() != rows or in_.numel() != cols:
            raise CiecuError(1, "Incompatible matrix-vector product: [%dx%d] * [%d] = [%d]"
                             % (rows, cols, in_.numel(), out.numel()))
        self.space._check(in_, out)
        self.space.enter()
        if self.space._sfx == "f64":
            call("ciecu_csr_spmv_f64", self.csr.handle, float(inScale), _ptr(in_), float(outScale), _ptr(out))
        else:
            call("ciecu_csr_spmv_f32", self.csr.handle, float(inScale), _ptr(in_), float(outScale), _ptr(out))
        self.space.leave()


def _mask_tensor(mask, device):
    if isinstance(mask, torch.Tensor) and mask.is_cuda:
        return mask
    arr = np.ascontiguousarray(np.asarray(mask, dtype=np.uint16)).view(np.int16)
    return torch.as_tensor(arr).to(device)


class MaskedCSROperator(LinearOperator):
    """MaskedCSROperator<int,double,double,uint16_t> (MaskedCSROperator.cpp:37-118): rows and
    columns whose mask is >= threshold are excluded; masked rows get inScale*out."""

    def __init__(self, lhs, mask, threshold, space, csr_handle=None):
        self.lhs = lhs
        self.space = space
        self.mask = _mask_tensor(mask, space.device)
        self.threshold = int(threshold)
        self.csr = csr_handle if csr_handle is not None else _CSRHandle(lhs, space)

    def product(self, inScale, in_, outScale, out):
        rows, cols = self.lhs.rowCount(), self.lhs.columnCount
        if out.numel() != rows or in_.numel() != cols:
            raise CiecuError(1, "Incompatible masked matrix-vector product: [%dx%d] * [%d] = [%d]"
                             % (rows, cols, in_.numel(), out.numel()))
        self.space._check(in_, out)
        self.space.enter()
        call("ciecu_csr_masked_spmv_f64", self.csr.handle, _ptr(self.mask), self.threshold, float(inScale),
             _ptr(in_), float(outScale), _ptr(out))
        self.space.leave()


class DiagonalOperator(LinearOperator):
    """DiagonalOperator<CUDASpace> (DiagonalOperator.cpp:37-53); owns the inverse diagonal."""

    def __init__(self, inverseDiagonal, space):
        self.inverseDiagonal = inverseDiagonal
        self.space = space

    def product(self, inScale, in_, outScale, out):
        self.space._check(in_, out)
        self.space.enter()
        call("ciecu_diagonal_apply_f64", self.space.handle, out.numel(), _ptr(self.inverseDiagonal),
             float(inScale), _ptr(in_), float(outScale), _ptr(out))
        self.space.leave()


def makeDiagonalOperator(matrix, space, csr_handle=None):
    """makeDiagonalOperator (DiagonalOperator.cpp:56-88): raises on a missing or zero diagonal."""
    handle = csr_handle if csr_handle is not None else _CSRHandle(matrix, space)
    dinv = space.makeVector(matrix.rowCount())
    space.enter()
    call("ciecu_diagonal_inverse_f64", handle.handle, _ptr(dinv))
    space.leave()
    op = DiagonalOperator(dinv, space)
    op._csr = handle
    return op


class JacobiOperator(LinearOperator):
    """JacobiOperator (JacobiOperator.cpp:36-62).  With a (masked) CSR operator and a
    DiagonalOperator every sweep is one fused kernel; any other operator pair runs
    the reference's composition of products and space operations."""

    def __init__(self, space, size, lhs, inverseDiagonal, iterations=1, relaxation=1.0):
        self.space = space
        self.size = int(size)
        self.lhs = lhs
        self.inverseDiagonal = inverseDiagonal
        self.iterations = int(iterations)
        self.relaxation = float(relaxation)
        self._work = space.makeVector(2 * self.size)

    def product(self, inScale, in_, outScale, out):
        if in_.numel() != out.numel() or out.numel() != self.size:
            raise CiecuError(1, "inconsistent input vector sizes")
        fused = isinstance(self.lhs, (CSROperator, MaskedCSROperator)) and isinstance(
            self.inverseDiagonal, DiagonalOperator)
        sp = self.space
        if fused:
            mask = self.lhs.mask if isinstance(self.lhs, MaskedCSROperator) else None
            thr = self.lhs.threshold if mask is not None else 0
            sp.enter()
            call("ciecu_jacobi_f64", self.lhs.csr.handle, _ptr(self.inverseDiagonal.inverseDiagonal), _ptr(mask),
                 thr, self.iterations, self.relaxation, float(inScale), _ptr(in_), float(outScale), _ptr(out),
                 _ptr(self._work))
            sp.leave()
            return
        memory = sp.makeVector(self.size)
        previous = sp.makeVector(self.size)
        residual = sp.makeVector(self.size)
        sp.assign(memory, out)
        sp.fill(out, 0)
        for _ in range(self.iterations):
            sp.assign(previous, out)
            sp.assign(residual, in_)
            self.lhs.product(1, out, -1, residual)
            self.inverseDiagonal.product(1, residual, self.relaxation, out)
        sp.scale(out, outScale)
        sp.add(out, memory, inScale)


class MaskedIdentityOperator(LinearOperator):
    """MaskedIdentityOperator (MaskedIdentityOperator.cpp:14-74)."""

    def __init__(self, space, mask, threshold):
        self.space = space
        self.mask = _mask_tensor(mask, space.device)
        self.threshold = int(threshold)

    def product(self, inScale, in_, outScale, out):
        self.space._check(in_, out)
        self.space.enter()
        call("ciecu_masked_identity_f64", self.space.handle, out.numel(), _ptr(self.mask), self.threshold,
             float(inScale), _ptr(in_), float(outScale), _ptr(out))
        self.space.leave()


class NestedProductOperator(LinearOperator):
    """NestedProductOperator (NestedProductOperator_impl.hpp:24-32): lhs(rhs(in))."""

    def __init__(self, space, lhs, rhs, rowCount):
        self.space = space
        self.lhs = lhs
        self.rhs = rhs
        self._buffer = space.makeVector(rowCount)
        space.fill(self._buffer, 0)

    def product(self, inScale, in_, outScale, out):
        self.rhs.product(0, in_, 1, self._buffer)
        self.lhs.product(inScale, self._buffer, outScale, out)


class ChebyshevOperator(LinearOperator):
    """Chebyshev polynomial smoother of D^-1 A (no reference counterpart)."""

    def __init__(self, lhs, inverseDiagonal, degree=4, lambdaMin=None, lambdaMax=None, ratio=30.0,
                 powerIterations=20, seed=0):
        self.lhs = lhs
        self.space = lhs.space
        self.inverseDiagonal = inverseDiagonal
        n = lhs.lhs.rowCount()
        self._work = self.space.makeVector(4 * n)
        if lambdaMax is None:
            lam = ctypes.c_double()
            self.space.enter()
            call("ciecu_power_lambda_max_f64", lhs.csr.handle, _ptr(inverseDiagonal.inverseDiagonal),
                 int(powerIterations), int(seed), _ptr(self._work), ctypes.byref(lam))
            lambdaMax = 1.1 * lam.value
        self.lambdaMax = float(lambdaMax)
        self.lambdaMin = float(lambdaMin) if lambdaMin is not None else self.lambdaMax / ratio
        self.degree = int(degree)

    def product(self, inScale, in_, outScale, out):
        self.space.enter()
        call("ciecu_chebyshev_f64", self.lhs.csr.handle, _ptr(self.inverseDiagonal.inverseDiagonal), self.degree,
             self.lambdaMin, self.lambdaMax, float(inScale), _ptr(in_), float(outScale), _ptr(out),
             _ptr(self._work))
        self.space.leave()


def _float_less(a, b):
    """utils::Comparison<double>::less with default tolerances (Comparison_impl.hpp:32-63)."""
    norm = min(abs(a) + abs(b), np.finfo(np.float64).max)
    tol = max(np.finfo(np.float64).tiny, np.finfo(np.float64).eps * norm)
    return a < b and not abs(a - b) < tol


class ConjugateGradients(LinearOperator):
    """ConjugateGradients<CUDASpace> (ConjugateGradients_impl.hpp:49-201).

    A plain CSROperator with no preconditioner or a DiagonalOperator runs the fused
    device-resident solver (ciecu_pcg_*).  Any other operator combination (masked
    operators, multigrid preconditioners) runs the reference algorithm composed of
    operator products and space operations, all on the GPU."""

    def __init__(self, lhs, space, preconditioner=None, settings=None, verbosity=0):
        self.lhs = lhs
        self.space = space
        self.preconditioner = preconditioner
        self.settings = settings if settings is not None else Statistics(0, 0.0, 0.0)
        self.verbosity = verbosity
        self._stats = None
        self._solver = None
        if type(lhs) is CSROperator and space._sfx == "f64" and (
                preconditioner is None or type(preconditioner) is DiagonalOperator):
            h = ctypes.c_void_p()
            dinv = preconditioner.inverseDiagonal if preconditioner is not None else None
            self._dinv = dinv
            call("ciecu_pcg_create", lhs.csr.handle, _ptr(dinv), self.settings, int(verbosity), ctypes.byref(h))
            self._solver = h

    def __del__(self):
        try:
            if getattr(self, "_solver", None):
                _lib.load().ciecu_pcg_destroy(self._solver)
                self._solver = None
        except Exception:
            pass

    def configure(self, settings):
        self.settings = settings
        if self._solver is not None:
            _lib.load().ciecu_pcg_destroy(self._solver)
            h = ctypes.c_void_p()
            call("ciecu_pcg_create", self.lhs.csr.handle, _ptr(self._dinv), settings, int(self.verbosity),
                 ctypes.byref(h))
            self._solver = h

    def getConfiguration(self):
        return self.settings

    def getStats(self):
        return self._stats

    def set_graph_chunk(self, iterations):
        if self._solver is not None:
            call("ciecu_pcg_set_graph_chunk", self._solver, int(iterations))

    def set_schedule(self, schedule):
        """Pins the fused solver's SpMV schedule (0: autotune at the next solve)."""
        if self._solver is not None:
            call("ciecu_pcg_set_schedule", self._solver, int(schedule))

    def set_loop(self, mode):
        """How the fused solver runs its iterations: 0 auto (a single cooperative
        launch when every SM's rows of the matrix fit in its shared memory), 1 the
        graph of three kernels per iteration, 2 the single launch."""
        if self._solver is not None:
            call("ciecu_pcg_set_loop", self._solver, int(mode))

    def debug_exchange(self, waitNanoseconds=2_000_000_000, withholdExchange=0):
        """Test hook of the single-launch solve's bounded waits (ciecu_pcg_debug_exchange):
        the wait limit in nanoseconds and an exchange at which the last block
        withholds its partial sums (0: none), which makes the solve time out."""
        if self._solver is not None:
            call("ciecu_pcg_debug_exchange", self._solver, int(waitNanoseconds), int(withholdExchange))

    def info(self):
        """SpMV schedule chosen for the fused solver kernel and how the last solve
        ran (fused device solver only)."""
        if self._solver is None:
            return {"fused": False}
        k, d = ctypes.c_int(), ctypes.c_int()
        call("ciecu_pcg_info", self._solver, ctypes.byref(k), ctypes.byref(d))
        nd, sym = ctypes.c_int(), ctypes.c_int()
        call("ciecu_pcg_dia_info", self._solver, ctypes.byref(nd), ctypes.byref(sym))
        return {"fused": True, "spmv_schedule": k.value, "device_loop": d.value >= 1,
                "loop": ("graph chunks", "graph loop", "single launch")[d.value],
                "dia_stored_diagonals": nd.value, "dia_symmetric": bool(sym.value)}

    def product(self, inScale, in_, outScale, out):
        n = self.space.size(out)
        if self.space.size(in_) != n:
            raise CiecuError(1, "incompatible vector sizes %d != %d" % (self.space.size(in_), n))
        if self._solver is not None:
            stats = Statistics()
            self.space._check(in_, out)
            self.space.enter()
            try:
                call("ciecu_pcg_product", self._solver, float(inScale), _ptr(in_), float(outScale), _ptr(out),
                     ctypes.byref(stats))
            finally:
                self._stats = stats
                self.space.leave()
            return
        self._generic_product(inScale, in_, outScale, out)

    def _generic_product(self, inScale, in_, outScale, out):
        sp = self.space
        settings = self.settings
        n = sp.size(out)
        stats = Statistics(0, np.finfo(np.float64).max, np.finfo(np.float64).max)
        solution = sp.makeVector(n)
        sp.assign(solution, out)
        if settings.iterationCount:
            search = sp.makeVector(n)
            searchProduct = sp.makeVector(n)
            sp.fill(searchProduct, 0)
            z = None
            residual = sp.makeVector(n)
            sp.assign(residual, in_)
            self.lhs.product(1, solution, -1, residual)
            residualNorm = sp.innerProduct(residual, residual)
            initial = float(np.sqrt(residualNorm))
            stats.absoluteResidual = initial
            stats.relativeResidual = 1.0
            if _float_less(stats.absoluteResidual, settings.absoluteResidual) or _float_less(
                    stats.relativeResidual, settings.relativeResidual):
                self._finish(inScale, outScale, out, solution, stats)
                return
            if self.preconditioner is not None:
                z = sp.makeVector(n)
                self.preconditioner.product(0, residual, 1, z)
                rz = sp.innerProduct(residual, z)
                sp.assign(search, z)
                if not 0 < rz:
                    raise CiecuError(3, "preconditioned norm vanished in iteration 0 (r^T @ z = 0)")
            else:
                rz = residualNorm
                sp.assign(search, residual)
                if not 0 < rz:
                    raise CiecuError(3, "residual norm vanished in iteration 0 (r^T @ r = 0)")
            while stats.iterationCount < settings.iterationCount:
                self.lhs.product(0, search, 1, searchProduct)
                den = sp.innerProduct(search, searchProduct)
                if not 0 < den:
                    self._stats = stats
                    raise CiecuError(3, "p^T @ A @ p vanished in iteration %d" % stats.iterationCount)
                alpha = rz / den
                sp.add(solution, search, alpha)
                sp.add(residual, searchProduct, -alpha)
                residualNorm = sp.innerProduct(residual, residual)
                previous = rz
                if z is not None:
                    self.preconditioner.product(0, residual, 1, z)
                    rz = sp.innerProduct(residual, z)
                else:
                    rz = residualNorm
                sp.scale(search, rz / previous)
                sp.add(search, z if z is not None else residual, 1)
                stats.absoluteResidual = float(np.sqrt(residualNorm))
                stats.relativeResidual = stats.absoluteResidual / initial
                if _float_less(stats.absoluteResidual, settings.absoluteResidual) or _float_less(
                        stats.relativeResidual, settings.relativeResidual):
                    break
                stats.iterationCount += 1
        self._finish(inScale, outScale, out, solution, stats)

    def _finish(self, inScale, outScale, out, solution, stats):
        sp = self.space
        if inScale == 1:
            sp.add(out, solution, outScale)
        elif inScale == 0:
            sp.assign(out, solution)
            sp.scale(out, outScale)
        else:
            sp.scale(out, inScale)
            sp.add(out, solution, outScale)
        self._stats = stats


class MixedPrecisionCG(LinearOperator):
    """FP32-inner Jacobi-PCG with FP64 refinement (ciecu_mixed_*): the FP32 matrix
    copy (16-bit column offsets where the bandwidth allows), FP32 vectors with FP64
    dot accumulators, FP64 residual r = b - A x and FP64 solution.  mode 0 =
    reliable updates (delta = replacement trigger), mode 1 = restarted iterative
    refinement (delta = inner tolerance).  Stops on the true FP64 residual.
    fuseDirection: False/0 = three kernels per inner iteration; True/1 = the search
    direction and its product formed in the inner SpMV by recurrence (two
    kernels); 2 = one kernel per inner iteration over the diagonal-storage copy
    (pending step, direction and product in one row pass; form 1 with any other
    inner kernel).  `kernels_per_iteration` reports the form that runs."""

    def __init__(self, lhs, inverseDiagonal, settings=None, mode=0, delta=None, compressColumns=True,
                 innerKernel=0, scaleInner=False, fuseDirection=False):
        if type(lhs) is not CSROperator or lhs.space._sfx != "f64":
            raise CiecuError(1, "MixedPrecisionCG needs an FP64 CSROperator")
        self.lhs = lhs
        self.space = lhs.space
        self.inverseDiagonal = inverseDiagonal
        self.settings = settings if settings is not None else Statistics(5000, 0.0, 1e-10)
        delta = (0.1 if mode == 0 else 1e-4) if delta is None else float(delta)
        self.options = MixedOptions(int(mode), delta, int(bool(compressColumns)), int(innerKernel),
                                    int(bool(scaleInner)), int(fuseDirection))
        h = ctypes.c_void_p()
        self.space.enter()
        call("ciecu_mixed_create", lhs.csr.handle, _ptr(inverseDiagonal.inverseDiagonal), self.settings, self.options,
             ctypes.byref(h))
        self._solver = h
        self._stats = None

    def __del__(self):
        try:
            if getattr(self, "_solver", None):
                _lib.load().ciecu_mixed_destroy(self._solver)
                self._solver = None
        except Exception:
            pass

    def info(self):
        c, v = ctypes.c_int(), ctypes.c_int()
        call("ciecu_mixed_info", self._solver, ctypes.byref(c), ctypes.byref(v))
        e = ctypes.c_int64()
        call("ciecu_mixed_padded_entries", self._solver, ctypes.byref(e))
        if v.value == -2:
            # the SELL copy (compressed_columns, padded_entries) is kept beside the DIA one
            nd, tr = ctypes.c_int(), ctypes.c_int()
            call("ciecu_mixed_dia_info", self._solver, ctypes.byref(nd), ctypes.byref(tr))
            return {"format": "dia", "inner_kernel": "dia", "group_unroll": v.value,
                    "compressed_columns": bool(c.value), "padded_entries": e.value,
                    "dia_diagonals": nd.value, "dia_triples": bool(tr.value)}
        return {"compressed_columns": bool(c.value), "format": "sell-32x4", "padded_entries": e.value,
                "group_unroll": v.value, "inner_kernel": "tma-pipeline" if v.value == 0 else "registers"}

    @property
    def kernels_per_iteration(self):
        k = ctypes.c_int()
        call("ciecu_mixed_form", self._solver, ctypes.byref(k))
        return k.value

    def set_graph_chunk(self, iterations):
        call("ciecu_mixed_set_graph_chunk", self._solver, int(iterations))

    def apply_inner(self, in32, out32):
        """out32 = A32 in32 with the solver's FP32 inner operator."""
        self.space.enter()
        call("ciecu_mixed_apply_f32", self._solver, _ptr(in32), _ptr(out32))
        self.space.leave()

    def getStats(self):
        return self._stats

    def product(self, inScale, in_, outScale, out):
        self.space._check(in_, out)
        stats = MixedStatistics()
        self.space.enter()
        try:
            call("ciecu_mixed_product", self._solver, float(inScale), _ptr(in_), float(outScale), _ptr(out),
                 ctypes.byref(stats))
        finally:
            self._stats = stats
            self.space.leave()


def block_diagonal(matrices):
    """One block-diagonal CSRMatrix holding the given square device CSR matrices
    (system s in rows/columns offsets[s] .. offsets[s+1]-1), and the row offsets."""
    if not matrices:
        raise CiecuError(1, "block_diagonal: no matrices")
    rowptrs, cols, vals, offsets = [], [], [], [0]
    nnz = 0
    for m in matrices:
        if m.rowCount() != m.columnCount:
            raise CiecuError(1, "block_diagonal: square matrices expected")
        rowptrs.append(m.rowExtents[:-1].to(torch.int64) + nnz)
        cols.append(m.columnIndices.to(torch.int64) + offsets[-1])
        vals.append(m.entries)
        nnz += m.nnz()
        offsets.append(offsets[-1] + m.rowCount())
    if nnz >= 2 ** 31 or offsets[-1] >= 2 ** 31:
        raise CiecuError(1, "block_diagonal: more than 2^31 rows or entries")
    dev = matrices[0].rowExtents.device
    rowptr = torch.cat(rowptrs + [torch.tensor([nnz], dtype=torch.int64, device=dev)]).to(torch.int32)
    return (CSRMatrix(offsets[-1], rowptr, torch.cat(cols).to(torch.int32), torch.cat(vals)),
            np.asarray(offsets, dtype=np.int64))


class BatchedConjugateGradients(LinearOperator):
    """Independent Jacobi-PCG solves of all systems of a block-diagonal matrix in
    shared kernel launches (ciecu_batch_*); every system follows
    ConjugateGradients_impl.hpp:49-201 with its own scalars and stopping test.
    getStats() returns one Statistics per system."""

    def __init__(self, lhs, rowOffsets, space, inverseDiagonal, settings=None):
        self.lhs = lhs
        self.space = space
        self.rowOffsets = np.ascontiguousarray(rowOffsets, dtype=np.int64)
        self.systems = len(self.rowOffsets) - 1
        self.settings = settings if settings is not None else Statistics(0, 0.0, 0.0)
        self.csr = inverseDiagonal._csr if getattr(inverseDiagonal, "_csr", None) is not None else _CSRHandle(
            lhs, space)
        self.inverseDiagonal = inverseDiagonal
        h = ctypes.c_void_p()
        space.enter()
        call("ciecu_batch_create", self.csr.handle, self.systems, self.rowOffsets.ctypes.data_as(ctypes.c_void_p),
             _ptr(inverseDiagonal.inverseDiagonal), self.settings, ctypes.byref(h))
        space.leave()
        self._solver = h
        self._stats = None

    def __del__(self):
        try:
            if getattr(self, "_solver", None):
                _lib.load().ciecu_batch_destroy(self._solver)
                self._solver = None
        except Exception:
            pass

    def info(self):
        v, d, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        call("ciecu_batch_info", self._solver, ctypes.byref(v), ctypes.byref(d), ctypes.byref(t))
        return {"lanes_per_row": v.value, "device_loop": bool(d.value), "tiles": t.value}

    def set_refinement(self, innerTolerance):
        """innerTolerance > 0: FP32 inner solves with FP64 refinement (0: FP64)."""
        self.space.enter()
        try:
            call("ciecu_batch_set_refinement", self._solver, float(innerTolerance))
        finally:
            self.space.leave()

    def set_reliable_updates(self, delta):
        """delta in (0, 1): FP32 iterations per system with FP64 reliable updates
        (the Krylov space kept across replacements); 0: off."""
        self.space.enter()
        try:
            call("ciecu_batch_set_reliable_updates", self._solver, float(delta))
        finally:
            self.space.leave()

    def refinements(self):
        """FP64 residual replacements per system in the last reliable-update solve."""
        out = (ctypes.c_int64 * self.systems)()
        call("ciecu_batch_refinements", self._solver, out)
        return list(out)

    def getStats(self):
        return self._stats

    def product(self, inScale, in_, outScale, out):
        self.space._check(in_, out)
        if in_.numel() != out.numel() or out.numel() != self.lhs.rowCount():
            raise CiecuError(1, "incompatible vector sizes")
        stats = (Statistics * self.systems)()
        self.space.enter()
        try:
            call("ciecu_batch_product", self._solver, float(inScale), _ptr(in_), float(outScale), _ptr(out), stats)
        finally:
            self._stats = list(stats)
            self.space.leave()


class MultiRHSConjugateGradients(LinearOperator):
    """k <= 32 independent Jacobi-PCG solves against one CSR matrix in shared
    SpMM launches (ciecu_multi_*).  product() takes row-major n x k blocks (a
    (n, k) tensor); getStats() returns one Statistics per right-hand side."""

    def __init__(self, lhs, inverseDiagonal, rhsCount, settings=None):
        if type(lhs) is not CSROperator or lhs.space._sfx != "f64":
            raise CiecuError(1, "MultiRHSConjugateGradients needs an FP64 CSROperator")
        self.lhs = lhs
        self.space = lhs.space
        self.k = int(rhsCount)
        self.inverseDiagonal = inverseDiagonal
        self.settings = settings if settings is not None else Statistics(0, 0.0, 0.0)
        h = ctypes.c_void_p()
        call("ciecu_multi_create", lhs.csr.handle, self.k, _ptr(inverseDiagonal.inverseDiagonal), self.settings,
             ctypes.byref(h))
        self._solver = h
        self._stats = None

    def __del__(self):
        try:
            if getattr(self, "_solver", None):
                _lib.load().ciecu_multi_destroy(self._solver)
                self._solver = None
        except Exception:
            pass

    def set_refinement(self, delta):
        """delta in (0, 1): FP32 iterations per column with FP64 reliable updates
        (replacement when the FP32 residual norm fell below delta times its largest
        value since the last one); 0: FP64 iterations."""
        call("ciecu_multi_set_refinement", self._solver, float(delta))
        self.refinement = float(delta)

    def set_format(self, fmt):
        """Pins the SpMM format: 1 the DIA copy (when the matrix has one), 0 CSR,
        -1 timed at the first solve (default)."""
        call("ciecu_multi_set_format", self._solver, int(fmt))

    def refinements(self):
        """FP64 residual recomputations per column in the last refined solve."""
        out = (ctypes.c_int64 * self.k)()
        call("ciecu_multi_refinements", self._solver, out)
        return list(out)

    def info(self):
        v, d = ctypes.c_int(), ctypes.c_int()
        call("ciecu_multi_info", self._solver, ctypes.byref(v), ctypes.byref(d))
        f = ctypes.c_int()
        call("ciecu_multi_format", self._solver, ctypes.byref(f))
        return {"lanes_per_row": v.value, "device_loop": bool(d.value),
                "spmm_format": "dia-%d" % f.value if f.value else "csr",
                "refinement": getattr(self, "refinement", 0.0)}

    def getStats(self):
        return self._stats

    def product(self, inScale, in_, outScale, out):
        n = self.lhs.lhs.rowCount()
        for v in (in_, out):
            if not (v.is_cuda and v.dtype == torch.float64 and v.is_contiguous() and v.numel() == n * self.k):
                raise CiecuError(1, "expected contiguous float64 CUDA blocks of %d x %d" % (n, self.k))
        stats = (Statistics * self.k)()
        self.space.enter()
        try:
            call("ciecu_multi_product", self._solver, float(inScale), _ptr(in_), float(outScale), _ptr(out), stats)
        finally:
            self._stats = list(stats)
            self.space.leave()
