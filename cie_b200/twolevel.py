"""Two-level (Q_p -> Q1) multigrid preconditioner on a structured grid, for the
finite-cell problems (no reference counterpart as a class; it is built from the
reference's operator algebra: CSR operators, diagonal, Chebyshev smoothing, CG).

  P  (fine x coarse): the trilinear (bi-/linear) interpolation of Q1 vertex values
     at the Q_p nodes of the same cells; R = P^T.  Rows of fine boundary DoFs and
     columns of coarse boundary DoFs are dropped, so corrections keep the
     homogeneous Dirichlet values.
  A1 (coarse): the Q1 operator assembled on the same cells with the same
     quadrature (same base rule and cut-cell tree), i.e. P^T A P on the interior;
     boundary rows eliminated.
  V-cycle (symmetric): z = S r; z += P A1^-1 R (r - A z); z += S (r - A z), with S
  a Chebyshev polynomial smoother in D^-1 A and the coarse problem solved by the
  fused Jacobi-PCG to a tight tolerance.
"""
import numpy as np
import torch

from ._lib import CiecuError, Statistics
from .fem import Assembler, StructuredMesh, csr_pattern
from .linalg import (ChebyshevOperator, ConjugateGradients, CSRMatrix, CSROperator, LinearOperator,
                     makeDiagonalOperator)

__all__ = ["prolongation", "TwoLevelMultigrid", "make_two_level"]


def _csr_from_triplets(nrows, ncols, rows, cols, vals):
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(nrows + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def prolongation(dim, order, cells, fineBoundary=None, coarseBoundary=None):
    """P (fine Q_order nodes x coarse Q1 vertices) as host CSR arrays (rowptr,
    col, val) and the transpose R in the same form."""
    cells = np.asarray(cells, dtype=np.int64)
    nf = cells * order + 1
    nc = cells + 1
    g = np.stack(np.meshgrid(*[np.arange(n) for n in nf[::-1]], indexing="ij")[::-1], axis=-1).reshape(-1, dim)
    fine = np.arange(g.shape[0])
    c = np.minimum(g // order, cells - 1)
    local = (g - order * c) / order  # in [0, 1]
    rows, cols, vals = [], [], []
    for corner in range(1 << dim):
        bits = np.array([(corner >> d) & 1 for d in range(dim)])
        w = np.prod(np.where(bits == 1, local, 1.0 - local), axis=1)
        vertex = c + bits
        idx = vertex[:, 0].copy()
        stride = 1
        for d in range(1, dim):
            stride *= nc[d - 1]
            idx += stride * vertex[:, d]
        keep = w != 0.0
        rows.append(fine[keep])
        cols.append(idx[keep])
        vals.append(w[keep])
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    keep = np.ones(rows.size, dtype=bool)
    if fineBoundary is not None:
        keep &= ~np.asarray(fineBoundary, dtype=bool)[rows]
    if coarseBoundary is not None:
        keep &= ~np.asarray(coarseBoundary, dtype=bool)[cols]
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    nfine, ncoarse = int(np.prod(nf)), int(np.prod(nc))
    return (_csr_from_triplets(nfine, ncoarse, rows, cols, vals),
            _csr_from_triplets(ncoarse, nfine, cols, rows, vals))


class TwoLevelMultigrid(LinearOperator):
    """The symmetric two-level V-cycle as a LinearOperator (out = inScale*out +
    outScale*M^-1 in), for use as the preconditioner of ConjugateGradients."""

    def __init__(self, space, fine, fineDiagonal, P, R, coarse, coarseDiagonal, degree=4,
                 coarseSettings=None):
        self.space = space
        self.fine, self.P, self.R = fine, P, R
        self.smoother = ChebyshevOperator(fine, fineDiagonal, degree=degree)
        self.coarseSolver = ConjugateGradients(coarse, space, coarseDiagonal,
                                               coarseSettings or Statistics(5000, 0.0, 1e-10))
        n, m = fine.lhs.rowCount(), coarse.lhs.rowCount()
        self._z = space.makeVector(n)
        self._r = space.makeVector(n)
        self._rc = space.makeVector(m)
        self._ec = space.makeVector(m)
        self.coarseIterations = []

    def product(self, inScale, in_, outScale, out):
        sp = self.space
        z, r, rc, ec = self._z, self._r, self._rc, self._ec
        self.smoother.product(0.0, in_, 1.0, z)       # z = S r
        sp.assign(r, in_)
        self.fine.product(1.0, z, -1.0, r)            # r - A z
        self.R.product(0.0, r, 1.0, rc)
        sp.fill(ec, 0.0)
        self.coarseSolver.product(0.0, rc, 1.0, ec)
        self.coarseIterations.append(self.coarseSolver.getStats().iterationCount)
        self.P.product(1.0, ec, 1.0, z)               # z += P A1^-1 R (r - A z)
        sp.assign(r, in_)
        self.fine.product(1.0, z, -1.0, r)
        self.smoother.product(1.0, r, 1.0, z)         # z += S (r - A z)
        if inScale == 0.0:
            sp.assign(out, z)
            if outScale != 1.0:
                sp.scale(out, outScale)
        else:
            sp.scale(out, inScale)
            sp.add(out, z, outScale)


def make_two_level(space, problem, center=None, radius=0.4, alpha=1e-6, depth=2, degree=4, coarseSettings=None):
    """The two-level preconditioner of a finite-cell problem made by
    make_embedded_poisson (same sphere, factor and tree)."""
    mesh = problem.mesh
    if mesh.order < 2:
        raise CiecuError(1, "make_two_level: the fine problem must be of order >= 2")
    dev = space.device
    cmesh = StructuredMesh(mesh.dim, 1, mesh.cells)
    rp, col = csr_pattern(cmesh.ncells, cmesh.nb, cmesh.dofmap, cmesh.ndofs)
    cmat = CSRMatrix(cmesh.ndofs, torch.as_tensor(rp).to(dev), torch.as_tensor(col).to(dev),
                     torch.zeros(col.size, dtype=torch.float64, device=dev))
    casm = Assembler(space, cmat, cmesh, quadratureOrder=mesh.order + 1)
    casm.assemble_embedded([0.5] * mesh.dim if center is None else center, radius, alpha, depth)
    cbnd = cmesh.boundary()
    casm.dirichlet(torch.as_tensor(cbnd).to(dev))
    (prp, pcol, pval), (rrp, rcol, rval) = prolongation(mesh.dim, mesh.order, mesh.cells,
                                                        problem.boundary.cpu().numpy(), cbnd)
    Pm = CSRMatrix(cmesh.ndofs, torch.as_tensor(prp).to(dev), torch.as_tensor(pcol).to(dev),
                   torch.as_tensor(pval).to(dev))
    Rm = CSRMatrix(mesh.ndofs, torch.as_tensor(rrp).to(dev), torch.as_tensor(rcol).to(dev),
                   torch.as_tensor(rval).to(dev))
    fine = CSROperator(problem.matrix, space)
    fineD = makeDiagonalOperator(problem.matrix, space, csr_handle=fine.csr)
    coarse = CSROperator(cmat, space)
    coarseD = makeDiagonalOperator(cmat, space, csr_handle=coarse.csr)
    mg = TwoLevelMultigrid(space, fine, fineD, CSROperator(Pm, space), CSROperator(Rm, space), coarse, coarseD,
                           degree=degree, coarseSettings=coarseSettings)
    mg._keep = (cmat, casm, Pm, Rm)
    return fine, fineD, mg
