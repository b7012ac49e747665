"""Weak Dirichlet conditions by penalty (DirichletPenaltyIntegrand_impl.hpp:38-88,
applied on boundary faces as constraints.cpp:306-380 does).  The reference's
integrand needs Eigen and cannot be built here, so the restatement is pinned by
what the face terms must satisfy: the penalty matrix sums to penalty x the
boundary measure (the basis is a partition of unity), it is symmetric positive
semi-definite and vanishes off the boundary DoFs, the RHS of g = 1 sums to the
same measure, and the penalised solution of a harmonic (linear) problem tends to
the prescribed values as 1/penalty.  The GPU assembly is then compared with the
restatement (-m gpu)."""
import numpy as np
import pytest


def penalty_only(restatement, dim, order, cells, penalty, faceMask=0, g=None):
    rp, col, val, b, bnd, _ = restatement.poisson_system(dim, order, cells, seed=0)
    zero = np.zeros_like(val)
    pv, prhs = restatement.dirichlet_penalty(dim, order, cells, penalty, rp, col, zero, faceMask=faceMask, g=g,
                                             rhs=None if g is None else np.zeros(len(rp) - 1))
    return rp, col, pv, prhs, bnd


@pytest.mark.parametrize("dim,order,cells", [(2, 1, [5, 4]), (2, 2, [3, 4]), (3, 1, [3, 2, 4]), (3, 3, [2, 2, 1])])
def test_penalty_terms_sum_to_the_boundary_measure(restatement, dim, order, cells):
    penalty = 7.5
    n = int(np.prod(order * np.array(cells) + 1))
    rp, col, pv, prhs, bnd = penalty_only(restatement, dim, order, cells, penalty, g=np.ones(n))
    measure = 2.0 * dim  # the faces of the unit box
    assert abs(pv.sum() - penalty * measure) <= 1e-12 * penalty * measure
    assert abs(prhs.sum() - penalty * measure) <= 1e-12 * penalty * measure
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    A[rows, col] = pv
    assert np.allclose(A, A.T, atol=1e-14 * penalty)
    assert np.linalg.eigvalsh(A).min() >= -1e-12 * penalty
    interior = ~bnd.astype(bool)
    assert np.all(A[interior] == 0.0) and np.all(A[:, interior] == 0.0)
    # one face only: the measure of that face
    _, _, pv1, _, _ = penalty_only(restatement, dim, order, cells, penalty, faceMask=1 << (2 * dim - 1))
    assert abs(pv1.sum() - penalty) <= 1e-12 * penalty


def test_penalised_harmonic_solution_converges(restatement):
    """-div grad u = 0 on the unit square with u = g = 1 + x + 2y weakly imposed:
    the nodal error of the penalised Q2 solution falls like 1/penalty (the
    stiffness of the reference convention carries (2/h)^2, so the penalty has to
    dominate that scale first)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    dim, order, cells = 2, 2, [6, 6]
    rp, col, _, _, _, _ = restatement.poisson_system(dim, order, cells, seed=0, kappa="one")
    # the stiffness without the symmetric elimination: assembled again from the element matrix
    nodes = order * np.array(cells) + 1
    xs = np.linspace(0.0, 1.0, nodes[0])
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    g = (1.0 + X + 2.0 * Y).ravel()
    dofmap = restatement.structured_dofmap(dim, order, cells)
    Ke = restatement.element_stiffness(dim, order, 1.0, 1.0 / np.array(cells))
    ncells = int(np.prod(cells))
    K, st = restatement.assemble(ncells, (order + 1) ** dim, dofmap, np.tile(Ke, ncells), rp, col)
    assert st == 0
    errs = []
    for penalty in (1e4, 1e6, 1e8):
        pv, prhs = restatement.dirichlet_penalty(dim, order, cells, penalty, rp, col, K, g=g,
                                                 rhs=np.zeros(len(rp) - 1))
        A = sp.csr_matrix((pv, col, rp), shape=(len(rp) - 1,) * 2)
        u = spl.spsolve(A.tocsc(), prhs)
        errs.append(np.abs(u - g).max())
    assert errs[1] < errs[0] / 50 and errs[2] < errs[1] / 50 and errs[2] < 1e-5, errs


@pytest.mark.gpu
@pytest.mark.parametrize("dim,order,cells,faceMask", [(2, 1, [9, 7], 0), (2, 2, [5, 6], 0b0110), (3, 1, [6, 5, 4], 0),
                                                      (3, 3, [3, 2, 3], 0b100001)])
def test_penalty_gpu_vs_restatement(restatement, dim, order, cells, faceMask):
    import torch
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CUDASpace
    space = CUDASpace()
    prob = make_poisson(space, dim, order, cells, seed=3)
    rp, col, val = prob.host_csr()
    b = prob.rhs.cpu().numpy()
    n = len(b)
    g = np.random.default_rng(1).uniform(-1, 1, n)
    prob.assembler.dirichlet_penalty(1e3, faceMask=faceMask, boundaryValues=torch.as_tensor(g).cuda(),
                                     rhs=prob.rhs)
    torch.cuda.synchronize()
    gv, gr = prob.host_csr()[2], prob.rhs.cpu().numpy()
    ov, orhs = restatement.dirichlet_penalty(dim, order, cells, 1e3, rp, col, val, faceMask=faceMask, g=g, rhs=b)
    assert np.abs(gv - ov).max() <= 1e-13 * np.abs(ov).max()
    assert np.abs(gr - orhs).max() <= 1e-13 * np.abs(orhs).max()


@pytest.mark.gpu
def test_penalised_solve_vs_reference(reference):
    """Homogeneous elimination replaced by the penalty: the GPU PCG solve of the
    penalised 3D Q1 system matches the reference CG on the same arrays."""
    import torch
    from cie_b200.fem import Assembler, StructuredMesh, csr_pattern, kappa_field, random_uniform
    from cie_b200.linalg import (CSRMatrix, CSROperator, ConjugateGradients, CUDASpace, Statistics,
                                 makeDiagonalOperator)
    space = CUDASpace()
    mesh = StructuredMesh(3, 1, [20, 20, 20])
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    m = CSRMatrix(mesh.ndofs, torch.as_tensor(rp).cuda(), torch.as_tensor(col).cuda(),
                  torch.zeros(len(col), dtype=torch.float64, device="cuda"))
    asm = Assembler(space, m, mesh)
    asm.assemble(torch.as_tensor(kappa_field(1, mesh.cells)).cuda())
    rhs = torch.as_tensor(random_uniform(0, mesh.ndofs)).cuda()
    g = torch.as_tensor(random_uniform(5, mesh.ndofs)).cuda()
    asm.dirichlet_penalty(1e4, boundaryValues=g, rhs=rhs)
    A = CSROperator(m, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(m, space, csr_handle=A.csr), Statistics(20000, 0.0, 1e-10))
    x = torch.zeros_like(rhs)
    cg.product(0.0, rhs, 1.0, x)
    hrp, hcol, hval = m.rowExtents.cpu().numpy(), m.columnIndices.cpu().numpy(), m.entries.cpu().numpy()
    xr, sr, err, _ = reference.pcg(hrp, hcol, hval, rhs.cpu().numpy(), maxit=20000, reltol=1e-10)
    assert err is None
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-9 * np.linalg.norm(xr)
