"""Graph set-up on the device against the reference's compiled reorder.cpp and the
restated pattern builder:
  * Cuthill-McKee / reverse maps identical to the reference's makeReordering
    wherever its std::sort keeps the column order of equal degrees (every batch
    of queued rows at most 16 long), and to the sequential restatement always;
  * the permuted CSR matrix identical to the reference's reorder, and a solve of
    the permuted system equal to the permuted solution;
  * the sparsity pattern of structured and scattered DoF maps identical to
    Assembler::makeCSRMatrix's (restatement, pinned by Assembler_test.cpp)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = [(2, 1, [17, 13]), (3, 1, [9, 7, 6]), (2, 2, [9, 8]), (2, 3, [6, 5]), (3, 2, [4, 5, 3]),
         (3, 1, [40, 40, 40])]


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


def device_matrix(space, rp, col, val):
    from cie_b200.linalg import CSRMatrix
    return CSRMatrix(len(rp) - 1, torch.as_tensor(rp).cuda(), torch.as_tensor(col).cuda(),
                     torch.as_tensor(val).cuda())


@pytest.mark.parametrize("dim,order,cells", CASES)
@pytest.mark.parametrize("strategy", [1, 2])
def test_reordering_vs_reference(space, restatement, reference, dim, order, cells, strategy):
    from cie_b200.graph import make_reordering
    rp, col, val, _, _, _ = restatement.poisson_system(dim, order, cells, seed=1)
    m = make_reordering(space, device_matrix(space, rp, col, val), strategy).cpu().numpy()
    seq, largest = restatement.cuthill_mckee(rp, col, strategy)
    assert np.array_equal(m, seq)
    assert np.array_equal(np.sort(m), np.arange(len(rp) - 1))
    if largest <= 16:
        assert np.array_equal(m, reference.make_reordering(rp, col, val, strategy))


def test_reordering_of_disconnected_rows(space, restatement, reference):
    """Two blocks and isolated rows: each component starts at the least-degree
    unqueued row, as the reference's restart does."""
    from cie_b200.graph import make_reordering
    from cie_b200.linalg import block_diagonal
    a = restatement.poisson_system(2, 1, [5, 4], seed=2)
    b = restatement.poisson_system(2, 1, [3, 6], seed=3)
    single = (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.0]))
    mats = [device_matrix(space, *a[:3]), device_matrix(space, *single), device_matrix(space, *b[:3]),
            device_matrix(space, *single)]
    bd, _ = block_diagonal(mats)
    rp, col, val = (t.cpu().numpy() for t in (bd.rowExtents, bd.columnIndices, bd.entries))
    for strategy in (1, 2):
        m = make_reordering(space, bd, strategy).cpu().numpy()
        assert np.array_equal(m, reference.make_reordering(rp, col, val, strategy))


@pytest.mark.parametrize("dim,order,cells", CASES[:4])
def test_reorder_csr_vs_reference(space, restatement, reference, dim, order, cells):
    from cie_b200.graph import make_reordering, reorder
    rp, col, val, _, _, _ = restatement.poisson_system(dim, order, cells, seed=4)
    A = device_matrix(space, rp, col, val)
    mapping = make_reordering(space, A, 2)
    B = reorder(space, mapping, A)
    rrp, rcol, rval = reference.reorder(mapping.cpu().numpy(), rp, col, val)
    assert np.array_equal(B.rowExtents.cpu().numpy(), rrp)
    assert np.array_equal(B.columnIndices.cpu().numpy(), rcol)
    assert np.array_equal(B.entries.cpu().numpy().view(np.uint64), rval.view(np.uint64))


def test_reordered_solve_is_the_permuted_solution(space, restatement):
    """PCG on the RCM-permuted 3D Q1 system (solver.cpp:490-519 reorders before
    solving) gives the permuted solution of the original system."""
    from cie_b200.graph import make_reordering, reorder, reorder_vector
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    rp, col, val, b, _, _ = restatement.poisson_system(3, 1, [24, 24, 24], seed=6)
    A = device_matrix(space, rp, col, val)
    bd = torch.as_tensor(b).cuda()
    mapping = make_reordering(space, A, 2)
    B = reorder(space, mapping, A)
    bp = reorder_vector(space, mapping, bd)
    sols = []
    for M, rhs in ((A, bd), (B, bp)):
        op = CSROperator(M, space)
        cg = ConjugateGradients(op, space, makeDiagonalOperator(M, space, csr_handle=op.csr),
                                Statistics(5000, 0.0, 1e-10))
        x = torch.zeros_like(rhs)
        cg.product(0.0, rhs, 1.0, x)
        sols.append(x)
    back = reorder_vector(space, mapping, sols[1], reverse=True)
    x0 = sols[0].cpu().numpy()
    assert np.linalg.norm(back.cpu().numpy() - x0) <= 1e-9 * np.linalg.norm(x0)


@pytest.mark.parametrize("dim,order,cells", [(2, 1, [7, 5]), (3, 1, [6, 5, 4]), (2, 3, [5, 6]), (3, 3, [3, 2, 4]),
                                             (3, 1, [64, 64, 64])])
def test_device_pattern_vs_restatement(space, restatement, dim, order, cells):
    from cie_b200.graph import csr_pattern_device
    dofmap = restatement.structured_dofmap(dim, order, cells)
    nb = (order + 1) ** dim
    ncells = int(np.prod(cells))
    ndofs = int(dofmap.max()) + 1
    rp, col = csr_pattern_device(space, ncells, nb, torch.as_tensor(dofmap).cuda(), ndofs)
    orp, ocol = restatement.csr_pattern(ncells, nb, dofmap, ndofs)
    assert np.array_equal(rp.cpu().numpy(), orp) and np.array_equal(col.cpu().numpy(), ocol)


def test_device_pattern_of_a_scattered_dofmap(space, restatement):
    """A DoF map with cells in random order, shared and unused DoFs (the
    Assembler_test.cpp shapes are structured; this one is not)."""
    from cie_b200.graph import csr_pattern_device
    rng = np.random.default_rng(12)
    ncells, nb, ndofs = 500, 6, 900
    dofmap = np.stack([rng.choice(ndofs - 50, nb, replace=False) for _ in range(ncells)]).astype(np.int32).ravel()
    rp, col = csr_pattern_device(space, ncells, nb, torch.as_tensor(dofmap).cuda(), ndofs)
    orp, ocol = restatement.csr_pattern(ncells, nb, dofmap, ndofs)
    assert np.array_equal(rp.cpu().numpy(), orp) and np.array_equal(col.cpu().numpy(), ocol)
