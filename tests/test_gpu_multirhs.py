"""Multi-right-hand-side Jacobi-PCG (SpMM-CG): every right-hand side against the
reference's compiled CG solving it alone -- same iteration count, solution within
1e-9 -- for k = 32 (full warp groups) and k = 5 (partial groups), plus initial
guesses, output scales and per-column iteration limits."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


@pytest.mark.parametrize("k,dim,cells", [(32, 3, [14, 14, 14]), (5, 2, [40, 40]), (1, 2, [30, 30])])
def test_multirhs_pcg_vs_reference_per_column(space, reference, k, dim, cells):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, MultiRHSConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, dim, 1, cells, seed=7)
    n = prob.rhs.numel()
    rng = np.random.default_rng(11)
    B = rng.uniform(-1, 1, (n, k))
    bnd = prob.boundary.cpu().numpy().astype(bool)
    B[bnd, :] = 0.0
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    solver = MultiRHSConjugateGradients(A, D, k, Statistics(5000, 0.0, 1e-10))
    X = torch.zeros(n, k, dtype=torch.float64, device="cuda")
    solver.product(0.0, torch.as_tensor(B).cuda().contiguous(), 1.0, X)
    stats = solver.getStats()
    Xh = X.cpu().numpy()
    rp, col, val = prob.host_csr()
    print(solver.info(), [s.iterationCount for s in stats[:4]])
    for c in range(k):
        xr, sr, err, _ = reference.pcg(rp, col, val, B[:, c].copy(), maxit=5000, abstol=0.0, reltol=1e-10)
        assert err is None
        assert stats[c].iterationCount == int(sr[0]), (c, stats[c].iterationCount, sr[0])
        rel = np.linalg.norm(Xh[:, c] - xr) / np.linalg.norm(xr)
        assert rel <= 1e-9, (c, rel)


def test_multirhs_pcg_scales_guesses_limits(space):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import (CSROperator, ConjugateGradients, MultiRHSConjugateGradients, Statistics,
                                 makeDiagonalOperator)
    prob = make_poisson(space, 2, 1, [32, 32], seed=8)
    n, k = prob.rhs.numel(), 7
    rng = np.random.default_rng(12)
    B = torch.as_tensor(rng.uniform(-1, 1, (n, k))).cuda().contiguous()
    Y0 = torch.as_tensor(rng.uniform(-1, 1, (n, k))).cuda().contiguous()
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    for settings in (Statistics(5000, 0.0, 1e-10), Statistics(9, 0.0, 1e-10)):
        solver = MultiRHSConjugateGradients(A, D, k, settings)
        out = Y0.clone()
        solver.product(2.0, B, -0.5, out)
        cg = ConjugateGradients(A, space, D, settings)
        for c in range(k):
            o = Y0[:, c].contiguous().clone()
            cg.product(2.0, B[:, c].contiguous(), -0.5, o)
            assert solver.getStats()[c].iterationCount == cg.getStats().iterationCount
            got = out[:, c]
            assert float(torch.linalg.norm(got - o) / torch.linalg.norm(o)) <= 1e-9
