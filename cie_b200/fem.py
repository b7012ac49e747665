"""Assembly path over the CUDA backend: structured Q_p meshes, the CSR pattern
(Assembler::makeCSRMatrix), GPU element stiffness integration + atomic-free
coloured scatter (IntegrandProcessor + Assembler::addContribution), symmetric
Dirichlet elimination, and the seeded synthetic Poisson problems.

Seeded inputs (identical host arrays feed the GPU and the oracle):
  RHS      uniform [-1, 1] from std::mt19937_64(seed)        ((x >> 11) 2^-53) 2 - 1
  kappa    exp(g), g ~ N(0,1) per cell (Box-Muller, seed+1), convolved with a
           separable Gaussian kernel (sigma = 1 cell, truncated at +-3 cells,
           clamped at the boundary) and standardised to unit variance.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call, CiecuError
from .linalg import CSRMatrix, CUDASpace, _ptr, _CSRHandle

__all__ = ["StructuredMesh", "csr_pattern", "Assembler", "random_uniform", "random_normal", "kappa_field",
           "PoissonProblem", "make_poisson", "make_embedded_poisson"]


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def random_uniform(seed, n):
    out = np.empty(int(n), dtype=np.float64)
    call("ciecu_random_uniform", int(seed), int(n), _np_ptr(out))
    return out


def random_normal(seed, n):
    out = np.empty(int(n), dtype=np.float64)
    call("ciecu_random_normal", int(seed), int(n), _np_ptr(out))
    return out


def kappa_field(seed, cells, sigma=1.0, truncation=3):
    cells = np.asarray(cells, dtype=np.int32)
    out = np.empty(int(np.prod(cells)), dtype=np.float64)
    call("ciecu_kappa_field", int(seed), len(cells), _np_ptr(cells), float(sigma), int(truncation), _np_ptr(out))
    return out


class StructuredMesh:
    """Uniform grid of Q_order Lagrange cells on the unit box."""

    def __init__(self, dim, order, cells):
        self.dim = int(dim)
        self.order = int(order)
        self.cells = np.asarray(cells, dtype=np.int32)
        assert self.cells.size == self.dim
        self.ncells = int(np.prod(self.cells))
        self.nb = (self.order + 1) ** self.dim
        self.dofmap = np.empty(self.ncells * self.nb, dtype=np.int32)
        nd = ctypes.c_int32()
        call("ciecu_structured_dofmap", self.dim, self.order, _np_ptr(self.cells), _np_ptr(self.dofmap),
             ctypes.byref(nd))
        self.ndofs = nd.value
        self.h = 1.0 / self.cells.astype(np.float64)

    def boundary(self):
        b = np.empty(self.ndofs, dtype=np.uint8)
        call("ciecu_structured_boundary", self.dim, self.order, _np_ptr(self.cells), _np_ptr(b))
        return b

    def colors(self):
        c = np.empty(self.ncells, dtype=np.int32)
        call("ciecu_structured_colors", self.dim, _np_ptr(self.cells), _np_ptr(c))
        return c


def csr_pattern(ncells, nb, dofmap, ndofs):
    """Assembler::makeCSRMatrix (fem/packages/graph/src/Assembler.cpp:55-175)."""
    dofmap = np.ascontiguousarray(dofmap, dtype=np.int32)
    rowptr = np.empty(int(ndofs) + 1, dtype=np.int32)
    nnz = ctypes.c_int64()
    call("ciecu_csr_pattern", int(ncells), int(nb), _np_ptr(dofmap), int(ndofs), _np_ptr(rowptr), None,
         ctypes.byref(nnz))
    col = np.empty(nnz.value, dtype=np.int32)
    call("ciecu_csr_pattern", int(ncells), int(nb), _np_ptr(dofmap), int(ndofs), _np_ptr(rowptr), _np_ptr(col),
         ctypes.byref(nnz))
    return rowptr, col


class Assembler:
    """GPU stiffness assembly into a device CSR pattern (ciecu_assembly_*)."""

    def __init__(self, space, matrix, mesh, quadratureOrder=None, colors=None, csr_handle=None,
                 d_dofmap=None):
        self.space = space
        self.matrix = matrix
        self.mesh = mesh
        self.csr = csr_handle if csr_handle is not None else _CSRHandle(matrix, space)
        self.d_dofmap = d_dofmap if d_dofmap is not None else torch.as_tensor(mesh.dofmap).to(space.device)
        colors = mesh.colors() if colors is None else np.ascontiguousarray(colors, dtype=np.int32)
        q = mesh.order + 1 if quadratureOrder is None else int(quadratureOrder)
        h = ctypes.c_void_p()
        space.enter()
        call("ciecu_assembly_create", self.csr.handle, mesh.dim, mesh.order, q, mesh.ncells, _ptr(self.d_dofmap),
             _np_ptr(colors), ctypes.byref(h))
        self.handle = h
        self._work = torch.empty(mesh.nb * mesh.nb, dtype=torch.float64, device=space.device)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                _lib.load().ciecu_assembly_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def assemble(self, kappa, convention=0, accumulate=False, entries=None):
        entries = self.matrix.entries if entries is None else entries
        h = np.ascontiguousarray(self.mesh.h, dtype=np.float64)
        self.space.enter()
        call("ciecu_assemble_stiffness", self.handle, _ptr(kappa), _np_ptr(h), int(convention), int(bool(accumulate)),
             _ptr(entries))
        self.space.leave()

    def assemble_embedded(self, center, radius, alpha, maxDepth, kappa=None, convention=0, accumulate=False,
                          entries=None, origin=None):
        """Finite-cell stiffness of the sphere |x - center| < radius inside the grid
        (fictitious part scaled by alpha, cut cells on a depth-maxDepth quadrature
        tree; ciecu_assemble_embedded).  Returns the number of cut cells."""
        entries = self.matrix.entries if entries is None else entries
        m = self.mesh
        h = np.ascontiguousarray(m.h, dtype=np.float64)
        cells = np.ascontiguousarray(m.cells, dtype=np.int32)
        org = np.zeros(m.dim) if origin is None else np.asarray(origin, dtype=np.float64)
        cen = np.ascontiguousarray(center, dtype=np.float64)
        cut = ctypes.c_int64()
        self.space.enter()
        call("ciecu_assemble_embedded", self.handle, _ptr(kappa), _np_ptr(h), _np_ptr(cells), _np_ptr(org),
             _np_ptr(cen), float(radius), float(alpha), int(maxDepth), int(convention), int(bool(accumulate)),
             _ptr(entries), _ptr(self._work), ctypes.byref(cut))
        self.space.leave()
        return cut.value

    def assemble_embedded_f32(self, entries32, center, radius, alpha, maxDepth, kappa=None, convention=0,
                              accumulate=False, origin=None):
        """The finite-cell matrix in FP32 (values in the same pattern): the cut
        cells' contractions on the tensor cores in split BF16 with FP32
        accumulation (ciecu_assemble_embedded_f32).  Returns the number of cut cells."""
        m = self.mesh
        h = np.ascontiguousarray(m.h, dtype=np.float64)
        cells = np.ascontiguousarray(m.cells, dtype=np.int32)
        org = np.zeros(m.dim) if origin is None else np.asarray(origin, dtype=np.float64)
        cen = np.ascontiguousarray(center, dtype=np.float64)
        cut = ctypes.c_int64()
        self.space.enter()
        call("ciecu_assemble_embedded_f32", self.handle, _ptr(kappa), _np_ptr(h), _np_ptr(cells), _np_ptr(org),
             _np_ptr(cen), float(radius), float(alpha), int(maxDepth), int(convention), int(bool(accumulate)),
             _ptr(entries32), ctypes.byref(cut))
        self.space.leave()
        return cut.value

    def dirichlet_f32(self, isBoundary, entries32):
        """Symmetric elimination on an FP32 copy of the values."""
        self.space.enter()
        call("ciecu_dirichlet_eliminate_f32", self.csr.handle, _ptr(isBoundary), _ptr(entries32))
        self.space.leave()

    def dirichlet_penalty(self, penalty, faceMask=0, quadratureOrder=0, boundaryValues=None, rhs=None,
                          entries=None):
        """Weak Dirichlet condition by penalty on the box faces selected by faceMask
        (bit 2d: x_d = 0, bit 2d + 1: x_d = max; 0 = all): the face terms of
        DirichletPenaltyIntegrand added to the matrix and, for nodal boundary values
        (a device vector over the DoFs), to rhs (ciecu_assemble_dirichlet_penalty)."""
        entries = self.matrix.entries if entries is None else entries
        m = self.mesh
        h = np.ascontiguousarray(m.h, dtype=np.float64)
        cells = np.ascontiguousarray(m.cells, dtype=np.int32)
        self.space.enter()
        call("ciecu_assemble_dirichlet_penalty", self.handle, _np_ptr(cells), _np_ptr(h), float(penalty),
             int(faceMask), int(quadratureOrder), _ptr(boundaryValues), _ptr(entries), _ptr(rhs))
        self.space.leave()

    def dirichlet(self, isBoundary, rhs=None, entries=None):
        entries = self.matrix.entries if entries is None else entries
        self.space.enter()
        call("ciecu_dirichlet_eliminate", self.csr.handle, _ptr(isBoundary), _ptr(entries), _ptr(rhs))
        self.space.leave()

    def element_gradient(self, lam, u, grad, convention=0):
        h = np.ascontiguousarray(self.mesh.h, dtype=np.float64)
        self.space.enter()
        call("ciecu_element_gradient", self.handle, _np_ptr(h), int(convention), _ptr(lam), _ptr(u), _ptr(grad),
             _ptr(self._work))
        self.space.leave()


class PoissonProblem:
    """A seeded Poisson system assembled on the GPU: matrix (device CSR, FP64),
    rhs (device), kappa (device), boundary flags, plus host copies on request."""

    def __init__(self, space, mesh, matrix, rhs, kappa, boundary, assembler, seed):
        self.space = space
        self.mesh = mesh
        self.matrix = matrix
        self.rhs = rhs
        self.kappa = kappa
        self.boundary = boundary
        self.assembler = assembler
        self.seed = seed

    def host_csr(self):
        m = self.matrix
        return (m.rowExtents.cpu().numpy(), m.columnIndices.cpu().numpy(), m.entries.cpu().numpy())


def make_embedded_poisson(space, dim, order, cells, center=None, radius=0.4, alpha=1e-6, depth=2, seed=0):
    """Finite-cell Poisson problem: Q_order cells on the unit box, the physical
    domain the sphere |x - center| < radius (center: the box centre), the rest
    scaled by alpha, cut cells integrated on a depth-`depth` quadrature tree with
    the (order+1)^dim Gauss rule per node; kappa = 1, homogeneous Dirichlet on the
    box boundary, RHS uniform [-1, 1] (seed)."""
    mesh = StructuredMesh(dim, order, cells)
    rowptr, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    dev = space.device
    matrix = CSRMatrix(mesh.ndofs, torch.as_tensor(rowptr).to(dev), torch.as_tensor(col).to(dev),
                       torch.zeros(col.size, dtype=torch.float64, device=dev))
    rhs = torch.as_tensor(random_uniform(seed, mesh.ndofs)).to(dev)
    bnd = torch.as_tensor(mesh.boundary()).to(dev)
    asm = Assembler(space, matrix, mesh)
    center = [0.5] * dim if center is None else center
    cut = asm.assemble_embedded(center, radius, alpha, depth)
    asm.dirichlet(bnd, rhs)
    torch.cuda.synchronize()
    prob = PoissonProblem(space, mesh, matrix, rhs, None, bnd, asm, seed)
    prob.cut_cells = cut
    return prob


def make_poisson(space, dim, order, cells, seed=0, kappa="lognormal", convention=0, kappa_seed=None):
    """Q_order Poisson problem on a cells^dim grid of the unit box, homogeneous
    Dirichlet boundary by symmetric elimination, RHS uniform [-1, 1] (seed),
    kappa = 1 or the smoothed log-normal field (seed + 1 unless kappa_seed)."""
    mesh = StructuredMesh(dim, order, cells)
    rowptr, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    dev = space.device
    matrix = CSRMatrix(mesh.ndofs, torch.as_tensor(rowptr).to(dev), torch.as_tensor(col).to(dev),
                       torch.zeros(col.size, dtype=torch.float64, device=dev))
    if isinstance(kappa, str) and kappa == "lognormal":
        k = kappa_field(seed + 1 if kappa_seed is None else kappa_seed, mesh.cells)
    elif isinstance(kappa, str) and kappa == "one":
        k = np.ones(mesh.ncells)
    else:
        k = np.asarray(kappa, dtype=np.float64)
    kappa_d = torch.as_tensor(k).to(dev)
    rhs = torch.as_tensor(random_uniform(seed, mesh.ndofs)).to(dev)
    bnd = torch.as_tensor(mesh.boundary()).to(dev)
    asm = Assembler(space, matrix, mesh)
    asm.assemble(kappa_d, convention=convention)
    asm.dirichlet(bnd, rhs)
    torch.cuda.synchronize()
    return PoissonProblem(space, mesh, matrix, rhs, kappa_d, bnd, asm, seed)
