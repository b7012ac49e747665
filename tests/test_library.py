"""CPU checks of the product library: libciecu.so loads, exports every symbol the
public headers declare, and its host-side set-up (DoF maps, sparsity pattern,
colouring, seeded generators) agrees with the oracle.  No GPU calls."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        for m in re.finditer(r"^\s*(?:int|void\*|void|int64_t)\s+(ciecu_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from cie_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them
    unbound = [n for n in names if n not in _lib.SIGNATURES]
    assert not unbound, unbound


def test_structured_dofmap_matches_oracle(restatement):
    from cie_b200.fem import StructuredMesh
    for dim, order, cells in ((2, 1, [3, 4]), (3, 1, [2, 3, 2]), (2, 2, [3, 2]), (3, 3, [2, 2, 1])):
        mesh = StructuredMesh(dim, order, cells)
        assert np.array_equal(mesh.dofmap, restatement.structured_dofmap(dim, order, cells))
        assert mesh.ndofs == int(np.prod([order * c + 1 for c in cells]))


def test_csr_pattern_matches_oracle(restatement):
    from cie_b200.fem import StructuredMesh, csr_pattern
    for dim, order, cells in ((2, 1, [5, 4]), (3, 1, [3, 3, 2]), (2, 2, [4, 3]), (3, 3, [2, 1, 2])):
        mesh = StructuredMesh(dim, order, cells)
        rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
        rp2, col2 = restatement.csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
        assert np.array_equal(rp, rp2) and np.array_equal(col, col2)


def test_pattern_sizes_of_the_configurations():
    # full Q1 patterns: 9-point stencil (3N-2)^2 and 27-point (3N-2)^3 entries
    from cie_b200.fem import StructuredMesh, csr_pattern
    mesh = StructuredMesh(2, 1, [256, 256])
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    assert mesh.ndofs == 66049 and rp[-1] == 591361
    mesh = StructuredMesh(3, 1, [16, 16, 16])
    rp, col = csr_pattern(mesh.ncells, mesh.nb, mesh.dofmap, mesh.ndofs)
    assert rp[-1] == (3 * 17 - 2) ** 3


def test_colours_separate_shared_dofs():
    from cie_b200.fem import StructuredMesh
    mesh = StructuredMesh(3, 1, [4, 3, 5])
    colors = mesh.colors()
    dm = mesh.dofmap.reshape(mesh.ncells, mesh.nb)
    for c in range(8):
        cells = np.flatnonzero(colors == c)
        dofs = dm[cells].ravel()
        assert len(np.unique(dofs)) == len(dofs)


def test_random_uniform_is_mt19937_64():
    # std::mt19937_64 default-seed (5489) 10000th output is 9981545732273789042 (C++ standard [rand.predef])
    from cie_b200 import fem
    u = fem.random_uniform(5489, 10000)
    x = 9981545732273789042
    assert u[-1] == (x >> 11) * 2.0 ** -53 * 2.0 - 1.0
    assert np.all((u >= -1) & (u < 1))


def test_kappa_field_statistics():
    from cie_b200 import fem
    k = fem.kappa_field(1, [32, 32, 32])
    g = np.log(k)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12
    # smoothing correlates neighbours
    g3 = g.reshape(32, 32, 32)
    corr = np.corrcoef(g3[:, :, :-1].ravel(), g3[:, :, 1:].ravel())[0, 1]
    assert 0.5 < corr < 0.95


def test_errors_are_reported_without_gpu():
    from cie_b200 import _lib
    with pytest.raises(_lib.CiecuError) as e:
        _lib.call("ciecu_structured_dofmap", 4, 1, None, None, None)
    assert e.value.status == 1 and "structured_dofmap" in str(e.value)


@pytest.mark.parametrize("name,args", [("ciecu_mixed_form", (None, None)), ("ciecu_mixed_dia_info", (None, None, None)),
                                       ("ciecu_mixed_set_graph_chunk", (None, 16))])
def test_mixed_solver_queries_refuse_null_handles(name, args):
    """Argument checks of the mixed solver's C-ABI run on the host: a null handle is
    CIECU_ERR_ARGUMENT with a message naming the call, and no CUDA call is made."""
    from cie_b200 import _lib
    with pytest.raises(_lib.CiecuError) as e:
        _lib.call(name, *args)
    assert e.value.status == 1 and name.replace("ciecu_", "") in str(e.value)
