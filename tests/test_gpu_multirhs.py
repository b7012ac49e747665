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


@pytest.mark.parametrize("k,dim,order,cells,offset,fmt", [(32, 3, 1, [14, 14, 14], 0, 1), (32, 3, 1, [14, 14, 14], 0, 0),
                                                          (32, 2, 1, [40, 40], 0, 1), (32, 3, 2, [6, 6, 6], 0, -1),
                                                          (32, 3, 1, [10, 10, 10], 1, 1), (5, 2, 1, [40, 40], 0, -1),
                                                          (1, 2, 1, [30, 30], 0, -1)])
def test_multirhs_pcg_vs_reference_per_column(space, reference, k, dim, order, cells, offset, fmt):
    """k = 32 runs the four-columns-per-lane SpMM: Q1 over the DIA copy (fmt 1:
    the triple pass, four rows per lane) or CSR (fmt 0), Q2 over CSR (no DIA
    copy); right-hand sides at an 8-byte offset (not 16-byte aligned) take the
    row-per-warp kernels.  Same iteration counts as the reference either way."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, MultiRHSConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, dim, order, cells, seed=7)
    n = prob.rhs.numel()
    rng = np.random.default_rng(11)
    B = rng.uniform(-1, 1, (n, k))
    bnd = prob.boundary.cpu().numpy().astype(bool)
    B[bnd, :] = 0.0
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    solver = MultiRHSConjugateGradients(A, D, k, Statistics(5000, 0.0, 1e-10))
    solver.set_format(fmt)
    X = torch.zeros(n, k, dtype=torch.float64, device="cuda")
    buf = torch.zeros(n * k + offset, dtype=torch.float64, device="cuda")
    Bd = buf[offset:].view(n, k)
    Bd.copy_(torch.as_tensor(B))
    solver.product(0.0, Bd, 1.0, X)
    stats = solver.getStats()
    Xh = X.cpu().numpy()
    rp, col, val = prob.host_csr()
    print(solver.info(), [s.iterationCount for s in stats[:4]])
    if fmt == 1:
        assert solver.info()["spmm_format"] == "dia-%d" % 3 ** dim
    elif fmt == 0:
        assert solver.info()["spmm_format"] == "csr"
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


@pytest.mark.parametrize("k,dim,order,cells,fmt", [(32, 3, 1, [14, 14, 14], 1), (32, 3, 1, [14, 14, 14], 0),
                                                   (5, 3, 2, [6, 6, 6], -1), (1, 2, 1, [30, 30], -1)])
def test_multirhs_fp32_refined_vs_reference_per_column(space, reference, k, dim, order, cells, fmt):
    """The FP32-refined form (FP32 SpMM iterations per column, FP64 reliable
    updates): every column's solution within 1e-9 of the reference's FP64 CG and
    its true FP64 residual at the 1e-10 stop; Q2 (125 diagonals) runs the FP32 CSR
    copy, Q1 the FP32 copy of whichever format the FP64 solve chose."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, MultiRHSConjugateGradients, Statistics, makeDiagonalOperator
    from oracle.oracle import Restatement
    prob = make_poisson(space, dim, order, cells, seed=7)
    n = prob.rhs.numel()
    rng = np.random.default_rng(13)
    B = rng.uniform(-1, 1, (n, k))
    bnd = prob.boundary.cpu().numpy().astype(bool)
    B[bnd, :] = 0.0
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    solver = MultiRHSConjugateGradients(A, D, k, Statistics(5000, 0.0, 1e-10))
    solver.set_refinement(0.1)
    solver.set_format(fmt)
    X = torch.zeros(n, k, dtype=torch.float64, device="cuda")
    solver.product(0.0, torch.as_tensor(B).cuda().contiguous(), 1.0, X)
    stats = solver.getStats()
    refinements = solver.refinements()
    Xh = X.cpu().numpy()
    rp, col, val = prob.host_csr()
    print(solver.info(), [s.iterationCount for s in stats[:4]], refinements[:4])
    ora = Restatement()
    for c in range(k):
        xr, sr, err, _ = reference.pcg(rp, col, val, B[:, c].copy(), maxit=5000, abstol=0.0, reltol=1e-10)
        assert err is None
        rel = np.linalg.norm(Xh[:, c] - xr) / np.linalg.norm(xr)
        r = ora.spmv(rp, col, val, 1.0, Xh[:, c].copy(), -1.0, B[:, c].copy())
        assert rel <= 1e-9, (c, rel)
        assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(B[:, c]), c
        assert stats[c].relativeResidual < 1e-10
        assert refinements[c] >= 1
        assert stats[c].iterationCount <= 1.3 * int(sr[0]) + 10, (c, stats[c].iterationCount, sr[0])


def test_multirhs_fp32_refined_limits_and_reuse(space):
    """Iteration limit per column in the refined form (done at the limit, the
    residual reported is the FP64 one), and switching one solver between the FP64
    and refined forms on the same blocks."""
    from cie_b200._lib import CiecuError
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, MultiRHSConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 2, 1, [32, 32], seed=8)
    n, k = prob.rhs.numel(), 4
    rng = np.random.default_rng(14)
    B = torch.as_tensor(rng.uniform(-1, 1, (n, k))).cuda().contiguous()
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    limited = MultiRHSConjugateGradients(A, D, k, Statistics(9, 0.0, 1e-10))
    limited.set_refinement(0.1)
    X = torch.zeros(n, k, dtype=torch.float64, device="cuda")
    limited.product(0.0, B, 1.0, X)
    for s in limited.getStats():
        assert s.iterationCount == 9 and 1e-10 < s.relativeResidual < 1.0
    solver = MultiRHSConjugateGradients(A, D, k, Statistics(5000, 0.0, 1e-10))
    X64 = torch.zeros_like(X)
    solver.product(0.0, B, 1.0, X64)
    solver.set_refinement(0.1)
    X32 = torch.zeros_like(X)
    solver.product(0.0, B, 1.0, X32)
    solver.set_refinement(0.0)
    X64b = torch.zeros_like(X)
    solver.product(0.0, B, 1.0, X64b)
    assert torch.equal(X64, X64b)
    assert float(torch.linalg.norm(X32 - X64) / torch.linalg.norm(X64)) <= 1e-9
    with pytest.raises(CiecuError):
        solver.set_refinement(1.5)
