"""Differentiable Poisson solve: u = A(kappa)^-1 P b on a structured Q_p mesh,
with A(kappa) = sum_e kappa_e K_e (GPU assembly) and the boundary DoFs eliminated
symmetrically (P zeroes them: homogeneous Dirichlet).  Gradients come from the
hand-written adjoint (ciecu_adjoint_gradient):

    lambda      = A^-1 P dJ/du        (transposed solve; A is symmetric -> same PCG)
    dJ/db       = lambda
    dJ/dkappa_e = -(P lambda)_e^T K_e(kappa = 1) (P u)_e

the method of the reference's 1-D adjoint model
(fem/python/modules/fem/optcontrol/adjointmodel.py:16-126, adjointelement.py:70-84)
applied to the Q_p stiffness of LinearIsotropicStiffnessIntegrand.  PoissonSolve
is the torch.autograd.Function over it; DifferentiablePoisson(kappa, b) applies it.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import CiecuError, Statistics, call
from .fem import Assembler, StructuredMesh, csr_pattern
from .linalg import CSRMatrix, CSROperator, _ptr

__all__ = ["DifferentiablePoisson", "PoissonSolve"]


class DifferentiablePoisson:
    """Owns the mesh, the CSR pattern, the assembly plan and an FP64 Jacobi-PCG
    solver of one structured Poisson problem; the matrix is re-assembled whenever
    it is asked for a different kappa."""

    def __init__(self, space, dim, order, cells, settings=None, convention=0):
        self.space = space
        self.mesh = StructuredMesh(dim, order, cells)
        m = self.mesh
        rowptr, col = csr_pattern(m.ncells, m.nb, m.dofmap, m.ndofs)
        dev = space.device
        self.n = m.ndofs
        self.matrix = CSRMatrix(m.ndofs, torch.as_tensor(rowptr).to(dev), torch.as_tensor(col).to(dev),
                                torch.zeros(col.size, dtype=torch.float64, device=dev))
        self.operator = CSROperator(self.matrix, space)
        self.assembler = Assembler(space, self.matrix, m, csr_handle=self.operator.csr)
        self.boundary = torch.as_tensor(m.boundary()).to(dev)
        self.convention = int(convention)
        self.settings = settings if settings is not None else Statistics(20000, 0.0, 1e-12)
        self.dinv = torch.empty(self.n, dtype=torch.float64, device=dev)
        self._h = np.ascontiguousarray(m.h, dtype=np.float64)
        self._work = torch.empty(2 * self.n + m.nb * m.nb, dtype=torch.float64, device=dev)
        self._solver = None
        self._kappa = None
        self.forward_stats = None
        self.adjoint_stats = None

    def __del__(self):
        try:
            if getattr(self, "_solver", None):
                _lib.load().ciecu_pcg_destroy(self._solver)
                self._solver = None
        except Exception:
            pass

    def __call__(self, kappa, b):
        return PoissonSolve.apply(kappa, b, self)

    def assemble(self, kappa):
        """A(kappa) into the matrix (skipped when it already holds this kappa)."""
        kappa = kappa.detach()
        if kappa.dtype != torch.float64 or kappa.numel() != self.mesh.ncells:
            raise CiecuError(1, "kappa must be %d float64 values" % self.mesh.ncells)
        if self._kappa is not None and torch.equal(kappa, self._kappa):
            return
        kappa = kappa.contiguous()
        self.assembler.assemble(kappa, convention=self.convention)
        self.assembler.dirichlet(self.boundary)
        sp = self.space
        sp.enter()
        call("ciecu_diagonal_inverse_f64", self.operator.csr.handle, _ptr(self.dinv))
        if self._solver is None:
            h = ctypes.c_void_p()
            call("ciecu_pcg_create", self.operator.csr.handle, _ptr(self.dinv), self.settings, 0, ctypes.byref(h))
            self._solver = h
        sp.leave()
        self._kappa = kappa.clone()

    def solve(self, b):
        """u = A^-1 P b for the kappa assembled last."""
        b = b.detach().to(torch.float64).contiguous()
        rhs = torch.where(self.boundary.bool(), torch.zeros_like(b), b)
        u = torch.zeros_like(rhs)
        stats = Statistics()
        self.space.enter()
        try:
            call("ciecu_pcg_product", self._solver, 0.0, _ptr(rhs), 1.0, _ptr(u), ctypes.byref(stats))
        finally:
            self.space.leave()
        self.forward_stats = stats
        return u

    def gradients(self, u, dJdu):
        """(dJ/dkappa, dJ/db) for the solution u and the sensitivity dJ/du."""
        dJdu = dJdu.detach().to(torch.float64).contiguous()
        lam = torch.empty_like(dJdu)
        grad = torch.empty(self.mesh.ncells, dtype=torch.float64, device=dJdu.device)
        stats = Statistics()
        self.space.enter()
        try:
            call("ciecu_adjoint_gradient", self._solver, self.assembler.handle, self._h.ctypes.data_as(ctypes.c_void_p),
                 self.convention, _ptr(self.boundary), _ptr(u.detach().contiguous()), _ptr(dJdu), _ptr(lam),
                 _ptr(grad), _ptr(self._work), ctypes.byref(stats))
        finally:
            self.space.leave()
        self.adjoint_stats = stats
        return grad, lam


class PoissonSolve(torch.autograd.Function):
    """u = A(kappa)^-1 P b; backward through the adjoint of DifferentiablePoisson."""

    @staticmethod
    def forward(ctx, kappa, b, problem):
        problem.assemble(kappa)
        u = problem.solve(b)
        ctx.problem = problem
        ctx.save_for_backward(kappa, u)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        kappa, u = ctx.saved_tensors
        problem = ctx.problem
        problem.assemble(kappa)  # the matrix may hold another kappa since this forward
        grad_kappa, grad_b = problem.gradients(u, grad_u)
        return (grad_kappa if ctx.needs_input_grad[0] else None,
                grad_b if ctx.needs_input_grad[1] else None, None)
