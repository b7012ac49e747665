"""GPU parity of the assembly path through the C-ABI: element stiffness
integration + coloured scatter against the C restatement of
TransformedIntegrand<LinearIsotropicStiffnessIntegrand> + Assembler::addContribution,
Dirichlet elimination, and the adjoint's per-element gradient."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from tests.test_gpu_linalg import dev, host  # noqa: E402


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


CASES = [(2, 1, [7, 5]), (3, 1, [4, 3, 5]), (2, 2, [5, 4]), (3, 2, [3, 2, 2]), (3, 3, [2, 3, 2]), (2, 3, [4, 4])]


def oracle_matrix(restatement, mesh, kappa, convention):
    rp, col = restatement.csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    Ke = np.concatenate([restatement.element_stiffness(mesh.dim, mesh.order, kappa[e], mesh.h, convention)
                         for e in range(mesh.ncells)])
    val, st = restatement.assemble(mesh.ncells, mesh.nb, mesh.dofmap, Ke, rp, col)
    assert st == 0
    return rp, col, val


@pytest.mark.parametrize("dim,order,cells", CASES)
@pytest.mark.parametrize("convention", [0, 1])
def test_assembly_vs_oracle(space, restatement, dim, order, cells, convention):
    from cie_b200.fem import Assembler, StructuredMesh, csr_pattern, kappa_field
    from cie_b200.linalg import CSRMatrix
    mesh = StructuredMesh(dim, order, cells)
    kappa = kappa_field(5, cells)
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    m = CSRMatrix(mesh.ndofs, dev(rp, torch.int32), dev(col, torch.int32), dev(np.zeros(len(col))))
    asm = Assembler(space, m, mesh)
    asm.assemble(dev(kappa), convention=convention)
    rp2, col2, ref = oracle_matrix(restatement, mesh, kappa, convention)
    assert np.array_equal(rp, rp2) and np.array_equal(col, col2)
    got = host(m.entries)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-13, err
    # accumulate mode adds a second copy
    asm.assemble(dev(kappa), convention=convention, accumulate=True)
    assert np.allclose(host(m.entries), 2 * ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def test_dirichlet_vs_oracle(space, restatement):
    from cie_b200.fem import make_poisson
    prob = make_poisson(space, 3, 1, [6, 5, 4], seed=7)
    mesh = prob.mesh
    kappa = host(prob.kappa)
    rp, col, val = oracle_matrix(restatement, mesh, kappa, 0)
    from cie_b200.fem import random_uniform
    rhs = random_uniform(7, mesh.ndofs)
    val, rhs = restatement.dirichlet(rp, col, val, mesh.boundary(), rhs)
    rp2, col2, val2 = prob.host_csr()
    assert np.array_equal(rp, rp2) and np.array_equal(col, col2)
    assert np.max(np.abs(val2 - val)) <= 1e-13 * np.abs(val).max()
    assert np.array_equal(host(prob.rhs), rhs)


def test_missing_pattern_entry_is_reported(space):
    from cie_b200.fem import Assembler, StructuredMesh
    from cie_b200.linalg import CSRMatrix
    from cie_b200._lib import CiecuError
    mesh = StructuredMesh(2, 1, [2, 2])
    # diagonal-only pattern: element couplings are missing
    n = mesh.ndofs
    m = CSRMatrix(n, dev(np.arange(n + 1), torch.int32), dev(np.arange(n), torch.int32), dev(np.zeros(n)))
    with pytest.raises(CiecuError, match="not part of the CSR pattern"):
        Assembler(space, m, mesh)


@pytest.mark.parametrize("dim,order,cells", [(3, 1, [5, 4, 3]), (2, 2, [6, 5])])
def test_element_gradient_vs_oracle(space, restatement, dim, order, cells):
    from cie_b200.fem import Assembler, StructuredMesh, csr_pattern
    from cie_b200.linalg import CSRMatrix
    mesh = StructuredMesh(dim, order, cells)
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    m = CSRMatrix(mesh.ndofs, dev(rp, torch.int32), dev(col, torch.int32), dev(np.zeros(len(col))))
    asm = Assembler(space, m, mesh)
    rng = np.random.default_rng(50)
    lam, u = rng.uniform(-1, 1, mesh.ndofs), rng.uniform(-1, 1, mesh.ndofs)
    grad = dev(np.zeros(mesh.ncells))
    asm.element_gradient(dev(lam), dev(u), grad)
    K1 = restatement.element_stiffness(dim, order, 1.0, mesh.h, 0)
    ref = restatement.element_gradient(mesh.ncells, mesh.nb, mesh.dofmap, K1, lam, u)
    assert np.allclose(host(grad), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
