"""p-multigrid over the CUDA operators: the cycle of the reference's
solveMultigrid (executables/fem_examples/src/poisson2D/solver.cpp:111-232).

Grids are DoF subsets selected by a per-DoF polynomial level (the ansatz mask):
grid 0 (threshold 2: level-1 DoFs) is solved by Jacobi-preconditioned CG on the
masked operator to a relative residual of 0.5; grid k = 1 .. p-1 (threshold k+2)
applies 6 damped Jacobi sweeps (relaxation 2/3) of the masked operator to the
masked residual.  One cycle visits the grids from the finest down to the
coarsest and back up to the finest, each visit adding its correction to the
solution and updating the residual with the grid operator; cycles repeat until
||r|| <= tolerance ||r0|| (tolerance 1e-6 in the reference).  All vectors stay on
the GPU; masked SpMV and the Jacobi sweeps are single kernels.
"""
import numpy as np
import torch

from ._lib import Statistics
from .linalg import (ConjugateGradients, JacobiOperator, MaskedCSROperator, MaskedIdentityOperator,
                     NestedProductOperator, makeDiagonalOperator, _CSRHandle, _mask_tensor)

__all__ = ["lagrange_ansatz_mask", "PMultigrid", "solveMultigrid"]


def lagrange_ansatz_mask(mesh):
    """Per-DoF polynomial level of a structured Q_p Lagrange mesh, the rule of
    makeAnsatzMask (fem/packages/graph/src/connectivity.cpp:63-91: level =
    max(1, largest 1-D basis index) over the tensor-product index, first index
    fastest) applied to the hierarchical order of the 1-D nodes: the two end nodes
    are the vertex functions (indices 0, 1), interior node i (1 <= i < p) is the
    degree-(i+1) function (index i + 1)."""
    p, dim = mesh.order, mesh.dim
    local = np.arange((p + 1) ** dim)
    level = np.ones(local.size, dtype=np.uint16)
    for d in range(dim):
        i = (local // (p + 1) ** d) % (p + 1)
        hier = np.where((i == 0) | (i == p), 0, i + 1)
        level = np.maximum(level, hier.astype(np.uint16))
    mask = np.zeros(mesh.ndofs, dtype=np.uint16)
    dofs = mesh.dofmap.reshape(mesh.ncells, -1)
    mask[dofs] = level[None, :]
    return mask


class PMultigrid:
    """The grids of solveMultigrid for `polynomialOrder` levels over one matrix."""

    def __init__(self, space, matrix, mask, polynomialOrder, csr_handle=None, coarseSettings=None,
                 sweeps=6, relaxation=2.0 / 3.0):
        self.space = space
        self.matrix = matrix
        n = matrix.rowCount()
        self.n = n
        csr = csr_handle if csr_handle is not None else _CSRHandle(matrix, space)
        self.csr = csr
        self.mask = _mask_tensor(mask, space.device)
        inverseDiagonal = makeDiagonalOperator(matrix, space, csr_handle=csr)
        self.inverseDiagonal = inverseDiagonal
        self.grids = []  # (operator, restriction, lhs)
        # grid 0: CG on the level-1 DoFs (solver.cpp:141-168)
        threshold = 2
        lhs = MaskedCSROperator(matrix, self.mask, threshold, space, csr_handle=csr)
        settings = coarseSettings if coarseSettings is not None else Statistics(5000, 0.0, 0.5)
        cg = ConjugateGradients(lhs, space, inverseDiagonal, settings)
        self.grids.append((cg, MaskedIdentityOperator(space, self.mask, threshold), lhs))
        # grids 1..p-1: damped Jacobi on levels <= order (solver.cpp:171-201)
        for order in range(2, polynomialOrder + 1):
            threshold = order + 1
            lhs = MaskedCSROperator(matrix, self.mask, threshold, space, csr_handle=csr)
            restriction = MaskedIdentityOperator(space, self.mask, threshold)
            smoother = JacobiOperator(space, n, lhs, inverseDiagonal, sweeps, relaxation)
            self.grids.append((NestedProductOperator(space, smoother, restriction, n), restriction, lhs))
        self.coarseIterations = []

    def _visit(self, grid, residual, gridResidual, update, solution):
        operator, restriction, lhs = grid
        sp = self.space
        restriction.product(0, residual, 1, gridResidual)
        sp.fill(update, 0)
        operator.product(0, gridResidual, 1, update)
        if isinstance(operator, ConjugateGradients) and operator.getStats() is not None:
            self.coarseIterations.append(operator.getStats().iterationCount)
        sp.add(solution, update, 1)
        lhs.product(1, update, -1, residual)

    def solve(self, rhs, solution, tolerance=1e-6, maxCycles=1000):
        """solution += corrections until ||r|| <= tolerance ||b - A solution_0|| with
        solution_0 = 0 (the reference starts from the zero guess).  Returns
        (cycles, relative residual)."""
        sp = self.space
        residual = sp.makeVector(self.n)
        sp.assign(residual, rhs)
        initial = float(np.sqrt(sp.innerProduct(residual, residual)))
        norm = initial
        gridResidual = sp.makeVector(self.n)
        update = sp.makeVector(self.n)
        cycles = 0
        while tolerance * initial < norm and cycles < maxCycles:
            for grid in reversed(self.grids):
                self._visit(grid, residual, gridResidual, update, solution)
            for grid in self.grids[1:]:
                self._visit(grid, residual, gridResidual, update, solution)
            norm = float(np.sqrt(sp.innerProduct(residual, residual)))
            cycles += 1
        return cycles, (norm / initial if initial > 0 else 0.0)


def solveMultigrid(space, matrix, solution, rhs, mask, polynomialOrder, tolerance=1e-6, maxCycles=1000):
    """solveMultigrid (solver.cpp:111-232) on device vectors; returns (cycles, relative residual)."""
    return PMultigrid(space, matrix, mask, polynomialOrder).solve(rhs, solution, tolerance, maxCycles)
