"""Finite-cell (embedded sphere) stiffness assembly on the GPU against the
oracle: per cell, the restated cut-cell quadrature tree
(KDTreeQuadraturePointFactory.hpp:67-173, material factor alpha outside) and the
restated element stiffness at those points, scattered into the same pattern."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


@pytest.mark.parametrize("dim,order,cells,depth", [(3, 3, [5, 6, 5], 2), (2, 2, [12, 10], 3), (3, 1, [9, 9, 9], 2),
                                                   (2, 3, [7, 7], 0)])
def test_embedded_assembly_vs_oracle(space, restatement, dim, order, cells, depth):
    from cie_b200.fem import Assembler, StructuredMesh, csr_pattern
    from cie_b200.linalg import CSRMatrix
    mesh = StructuredMesh(dim, order, cells)
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    m = CSRMatrix(mesh.ndofs, torch.as_tensor(rp).cuda(), torch.as_tensor(col).cuda(),
                  torch.zeros(col.size, dtype=torch.float64, device="cuda"))
    asm = Assembler(space, m, mesh)
    center, radius, alpha = [0.5] * dim, 0.4, 1e-6
    cut = asm.assemble_embedded(center, radius, alpha, depth)
    got = m.entries.cpu().numpy()
    h = mesh.h
    Ke = []
    for e in range(mesh.ncells):
        idx, rest = [], e
        for d in range(dim):
            idx.append(rest % cells[d])
            rest //= cells[d]
        origin = np.array(idx) * h
        pts, w, s = restatement.cut_cell_points(dim, depth, order + 1, center, radius, origin, h, alpha)
        Ke.append(restatement.element_stiffness(dim, order, 1.0, h, 0, points=pts.ravel(), weights=w * s))
    ref, st = restatement.assemble(mesh.ncells, mesh.nb, mesh.dofmap, np.concatenate(Ke), rp, col)
    assert st == 0
    print("%dD Q%d %s depth %d: %d cut cells of %d" % (dim, order, cells, depth, cut, mesh.ncells))
    assert 0 < cut < mesh.ncells
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    # the FP32 copy from the split-BF16 tensor-core contraction, against the FP64 matrix
    v32 = torch.zeros(col.size, dtype=torch.float32, device="cuda")
    assert asm.assemble_embedded_f32(v32, center, radius, alpha, depth) == cut
    err = np.abs(v32.cpu().numpy().astype(np.float64) - got).max() / np.abs(got).max()
    print("FP32 (split BF16 tensor cores) max entry error relative to the largest entry: %.3e" % err)
    assert err <= 1e-4


def test_embedded_assembly_is_deterministic(space):
    """Eight CTAs per cut cell, partial matrices summed in tree-node order and
    scattered by colour: repeated assemblies are bit-identical."""
    from cie_b200.fem import make_embedded_poisson
    outs = [make_embedded_poisson(space, 3, 3, [8, 8, 8], radius=0.4, alpha=1e-6, depth=2).matrix.entries.cpu().numpy()
            for _ in range(2)]
    assert np.array_equal(outs[0].view(np.uint64), outs[1].view(np.uint64))
