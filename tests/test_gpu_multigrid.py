"""GPU p-multigrid (solveMultigrid, executables/fem_examples/src/poisson2D/
solver.cpp:111-232) against the reference's own cycle compiled from its sources,
on the same matrix, level mask and right-hand side: same number of cycles and
solutions within 1e-9."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,order,cells", [(2, 3, [24, 24]), (3, 2, [10, 10, 10]), (3, 3, [6, 6, 6])])
def test_pmultigrid_vs_reference(reference, dim, order, cells):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CUDASpace
    from cie_b200.multigrid import PMultigrid, lagrange_ansatz_mask
    space = CUDASpace()
    prob = make_poisson(space, dim, order, cells, seed=3)
    mask = lagrange_ansatz_mask(prob.mesh)
    mg = PMultigrid(space, prob.matrix, mask, order)
    x = torch.zeros_like(prob.rhs)
    cycles, rel = mg.solve(prob.rhs, x, tolerance=1e-6, maxCycles=200)
    rp, col, val = prob.host_csr()
    b = prob.rhs.cpu().numpy()
    xr, cycles_r, rel_r = reference.pmg(rp, col, val, mask, order, b, tol=1e-6, maxCycles=200)
    err = np.linalg.norm(x.cpu().numpy() - xr) / np.linalg.norm(xr)
    print("p=%d %s: GPU %d cycles (rel %.3e), reference %d cycles (rel %.3e), |x - x_ref|/|x_ref| = %.3e, "
          "coarse CG iterations %s" % (order, cells, cycles, rel, cycles_r, rel_r, err, mg.coarseIterations[:6]))
    assert cycles == cycles_r
    assert rel <= 1e-6 and abs(rel - rel_r) <= 1e-9 * max(1.0, rel_r) + 1e-12
    assert err <= 1e-9


def test_pmultigrid_breakdown_matches_reference(reference):
    """Damped Jacobi does not smooth degree-5 equispaced Lagrange levels: the cycle
    diverges and the coarse CG breaks down -- in the reference and here alike, at
    the same iteration and with the same message."""
    from cie_b200._lib import CiecuError
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CUDASpace
    from cie_b200.multigrid import PMultigrid, lagrange_ansatz_mask
    space = CUDASpace()
    prob = make_poisson(space, 2, 5, [8, 8], seed=3)
    mask = lagrange_ansatz_mask(prob.mesh)
    rp, col, val = prob.host_csr()
    with pytest.raises(RuntimeError, match=r"p\^T @ A @ p vanished in iteration 1"):
        reference.pmg(rp, col, val, mask, 5, prob.rhs.cpu().numpy(), tol=1e-6, maxCycles=200)
    mg = PMultigrid(space, prob.matrix, mask, 5)
    with pytest.raises(CiecuError, match=r"p\^T @ A @ p vanished in iteration 1") as info:
        mg.solve(prob.rhs, torch.zeros_like(prob.rhs), tolerance=1e-6, maxCycles=200)
    assert info.value.status == 3
