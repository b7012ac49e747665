"""Graph set-up on the device: Cuthill-McKee / reverse Cuthill-McKee reordering
(makeReordering, linalg/packages/utilities/src/reorder.cpp:23-173), the
permutation of CSR matrices and vectors (reorder, :215-425), and the sparsity
pattern of a DoF map (Assembler::makeCSRMatrix, fem/packages/graph/src/Assembler.cpp:55-175)."""
import ctypes

import torch

from ._lib import call
from .linalg import CSRMatrix, _ptr

__all__ = ["CUTHILL_MCKEE", "REVERSE_CUTHILL_MCKEE", "make_reordering", "reorder", "reorder_vector",
           "csr_pattern_device"]

CUTHILL_MCKEE = 1
REVERSE_CUTHILL_MCKEE = 2


def make_reordering(space, matrix, strategy=CUTHILL_MCKEE):
    """map[k] = the row of `matrix` placed at position k (int32 tensor on the device)."""
    n = matrix.rowCount()
    out = torch.empty(n, dtype=torch.int32, device=space.device)
    space.enter()
    call("ciecu_make_reordering", space.handle, n, _ptr(matrix.rowExtents), _ptr(matrix.columnIndices),
         int(strategy), _ptr(out))
    space.leave()
    return out


def reorder(space, mapping, matrix):
    """The matrix with new row i = old row mapping[i] and columns renumbered
    (reorder<int,double,false>), as a new device CSRMatrix."""
    n = matrix.rowCount()
    dev = space.device
    rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    col = torch.empty_like(matrix.columnIndices)
    val = torch.empty_like(matrix.entries)
    space.enter()
    call("ciecu_reorder_csr", space.handle, n, _ptr(mapping), _ptr(matrix.rowExtents), _ptr(matrix.columnIndices),
         _ptr(matrix.entries), _ptr(rp), _ptr(col), _ptr(val))
    space.leave()
    return CSRMatrix(matrix.columnCount, rp, col, val)


def reorder_vector(space, mapping, v, reverse=False):
    """out[i] = v[mapping[i]] (reverse: out[mapping[i]] = v[i])."""
    out = torch.empty_like(v)
    space.enter()
    call("ciecu_reorder_vector", space.handle, v.numel(), _ptr(mapping), int(bool(reverse)), _ptr(v), _ptr(out))
    space.leave()
    return out


def csr_pattern_device(space, ncells, nb, dofmap, ndofs):
    """(rowExtents, columnIndices) of a DoF map (device int32 tensor of ncells * nb)
    built on the device."""
    dev = space.device
    rp = torch.empty(int(ndofs) + 1, dtype=torch.int32, device=dev)
    nnz = ctypes.c_int64()
    space.enter()
    call("ciecu_csr_pattern_device", space.handle, int(ncells), int(nb), _ptr(dofmap), int(ndofs), _ptr(rp), None,
         ctypes.byref(nnz))
    col = torch.empty(nnz.value, dtype=torch.int32, device=dev)
    call("ciecu_csr_pattern_device", space.handle, int(ncells), int(nb), _ptr(dofmap), int(ndofs), _ptr(rp),
         _ptr(col), ctypes.byref(nnz))
    space.leave()
    return rp, col
