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
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import CiecuError, MgOptions, Statistics, call
from .fem import Assembler, StructuredMesh, csr_pattern
from .linalg import (ChebyshevOperator, ConjugateGradients, CSRMatrix, CSROperator, LinearOperator,
                     _CSRHandle, _ptr, makeDiagonalOperator)

__all__ = ["prolongation", "TwoLevelMultigrid", "make_two_level", "TwoLevelCG", "make_two_level_cg"]


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


class TwoLevelCG(LinearOperator):
    """Conjugate gradients preconditioned by the symmetric two-level cycle, run on
    the device as one CUDA graph (ciecu_mgcg_*): Chebyshev smoothing of `degree`
    in D^-1 A before and after a coarse correction made of `coarseIterations`
    Jacobi-PCG iterations.  With `smoother32` (an FP32 CSRMatrix in the fine
    pattern) the cycle smooths and forms its residuals in FP32; the outer
    iteration stays FP64.  flexible=True uses the flexible CG beta, which keeps
    the outer iteration convergent when the cycle is not a fixed linear operator."""

    def __init__(self, fine, fineDiagonal, P, R, coarse, coarseDiagonal, settings, degree=2, coarseIterations=8,
                 ratio=30.0, lambdaMax=0.0, flexible=True, smoother32=None):
        self.lhs = fine
        self.space = fine.space
        self.settings = settings
        self._stats = Statistics()
        self._s32 = _CSRHandle(smoother32, self.space) if smoother32 is not None else None
        opts = MgOptions(int(degree), float(lambdaMax), float(ratio), int(coarseIterations), int(bool(flexible)))
        h = ctypes.c_void_p()
        self.space.enter()
        call("ciecu_mgcg_create", fine.csr.handle, _ptr(fineDiagonal.inverseDiagonal),
             self._s32.handle if self._s32 is not None else None, P.csr.handle, R.csr.handle, coarse.csr.handle,
             _ptr(coarseDiagonal.inverseDiagonal), opts, settings, ctypes.byref(h))
        self.handle = h
        self._keep = (fine, fineDiagonal, P, R, coarse, coarseDiagonal, smoother32)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                _lib.load().ciecu_mgcg_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def product(self, inScale, in_, outScale, out):
        stats = Statistics()
        self.space.enter()
        try:
            call("ciecu_mgcg_product", self.handle, float(inScale), _ptr(in_), float(outScale), _ptr(out),
                 ctypes.byref(stats))
        finally:
            self._stats = stats
            self.space.leave()

    def getStats(self):
        return self._stats

    def set_coarse_cluster(self, enable):
        """False: the pipelined coarse kernels (one launch per coarse iteration) even
        where the one-launch cluster form applies; True (the default): the cluster
        form where the coarse matrix allows it.  Takes effect at the next product."""
        call("ciecu_mgcg_set_coarse_cluster", self.handle, int(bool(enable)))

    def coarse_apply(self, in_, out):
        """out = C in: the cycle's coarse solve alone (coarse-sized FP64 vectors)."""
        self.space.enter()
        try:
            call("ciecu_mgcg_coarse_apply", self.handle, _ptr(in_), _ptr(out))
        finally:
            self.space.leave()

    def info(self):
        lam, cycles = ctypes.c_double(), ctypes.c_int64()
        call("ciecu_mgcg_info", self.handle, ctypes.byref(lam), ctypes.byref(cycles))
        o16, lanes = ctypes.c_int(), ctypes.c_int()
        call("ciecu_mgcg_smoother_info", self.handle, ctypes.byref(o16), ctypes.byref(lanes))
        ctas, active = ctypes.c_int(), ctypes.c_int()
        call("ciecu_mgcg_coarse_info", self.handle, ctypes.byref(ctas), ctypes.byref(active))
        return {"lambda_max": lam.value, "cycles": cycles.value, "smoother_offsets16": bool(o16.value),
                "smoother_lanes_per_row": lanes.value, "coarse_cluster_ctas": ctas.value,
                "coarse_cluster_active": bool(active.value)}


def make_two_level_cg(space, problem, settings, center=None, radius=0.4, alpha=1e-6, depth=2, degree=2,
                      coarseIterations=8, ratio=30.0, flexible=True, precision="f64"):
    """The device two-level CG of a finite-cell problem made by
    make_embedded_poisson (same sphere, factor and tree).  precision "f32"
    smooths on the FP32 matrix assembled with the tensor-core contraction
    (ciecu_assemble_embedded_f32) and eliminated like the FP64 one."""
    fine, fineD, mg = make_two_level(space, problem, center=center, radius=radius, alpha=alpha, depth=depth,
                                     degree=degree)
    cmat, casm, Pm, Rm = mg._keep
    coarse = mg.coarseSolver.lhs
    coarseD = mg.coarseSolver.preconditioner
    s32 = None
    if precision == "f32":
        m = problem.matrix
        v32 = torch.zeros(m.entries.numel(), dtype=torch.float32, device=space.device)
        problem.assembler.assemble_embedded_f32(v32, [0.5] * problem.mesh.dim if center is None else center, radius,
                                                alpha, depth)
        problem.assembler.dirichlet_f32(problem.boundary, v32)
        s32 = CSRMatrix(m.columnCount, m.rowExtents, m.columnIndices, v32)
    solver = TwoLevelCG(fine, fineD, mg.P, mg.R, coarse, coarseD, settings, degree=degree,
                        coarseIterations=coarseIterations, ratio=ratio, lambdaMax=mg.smoother.lambdaMax,
                        flexible=flexible, smoother32=s32)
    solver._mg = mg
    return solver
