"""Linear-system output in MatrixMarket text (cie::io::MatrixMarket::Output,
cieutils/packages/io/src/MatrixMarket.cpp), as the reference's driver writes
lhs.mm / rhs.mm before solving (executables/fem_examples/src/poisson2D/solver.cpp:521-539)."""
import ctypes

import numpy as np

from ._lib import call
from .linalg import CSRMatrix, _CSRHandle, _ptr

__all__ = ["write_matrix_market", "write_matrix_market_vector"]


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def write_matrix_market(path, matrix, space=None):
    """Writes a CSR matrix: a device CSRMatrix (with its space) or host arrays
    (rowptr, col, val[, columns])."""
    if isinstance(matrix, CSRMatrix):
        if space is None:
            raise ValueError("write_matrix_market: a device matrix needs its space")
        handle = _CSRHandle(matrix, space)
        call("ciecu_write_matrix_market", handle.handle, str(path).encode())
        return
    rowptr, col, val = (np.ascontiguousarray(a, dtype=t) for a, t in zip(matrix[:3], (np.int32, np.int32, np.float64)))
    columns = matrix[3] if len(matrix) > 3 else len(rowptr) - 1
    call("ciecu_write_matrix_market_host", str(path).encode(), len(rowptr) - 1, int(columns), _np_ptr(rowptr),
         _np_ptr(col), _np_ptr(val))


def write_matrix_market_vector(path, values, space=None):
    """Writes a vector (device tensor with its space, or a host array) in the
    MatrixMarket array format."""
    if space is not None:
        call("ciecu_write_matrix_market_vector", space.handle, int(values.numel()), _ptr(values), str(path).encode())
        return
    v = np.ascontiguousarray(values, dtype=np.float64)
    call("ciecu_write_matrix_market_vector_host", str(path).encode(), len(v), _np_ptr(v))
