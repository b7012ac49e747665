"""Host-side level mask of the p-multigrid (no GPU): the Lagrange analogue of
makeAnsatzMask (fem/packages/graph/src/connectivity.cpp:63-91)."""
import numpy as np

from cie_b200.fem import StructuredMesh
from cie_b200.multigrid import lagrange_ansatz_mask


def test_vertices_are_level_one_and_levels_nest():
    for dim, order, cells in [(2, 3, [4, 3]), (3, 2, [3, 2, 2]), (2, 1, [5, 5])]:
        mesh = StructuredMesh(dim, order, cells)
        mask = lagrange_ansatz_mask(mesh)
        assert mask.min() >= 1 and mask.max() == max(1, order)
        # level-1 DoFs are exactly the mesh vertices: (cells + 1)^dim of them
        assert int(np.sum(mask == 1)) == int(np.prod(np.asarray(cells) + 1))
        # every DoF of a cell gets the same level from every cell sharing it
        dofs = mesh.dofmap.reshape(mesh.ncells, -1)
        p = order
        local = np.arange((p + 1) ** dim)
        level = np.ones(local.size, dtype=np.uint16)
        for d in range(dim):
            i = (local // (p + 1) ** d) % (p + 1)
            level = np.maximum(level, np.where((i == 0) | (i == p), 0, i + 1).astype(np.uint16))
        assert np.all(mask[dofs] == level[None, :])
