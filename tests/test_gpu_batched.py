"""Batched Jacobi-PCG over systems of different sizes (block-diagonal CSR, one
tile list, per-system scalars): every system against the reference's compiled CG
solving it alone -- same iteration count, solution within 1e-9 -- plus initial
guesses and output scales, the block check and a breakdown in one system."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


def systems(space, count, seed, lo=4, hi=40):
    from cie_b200.fem import make_poisson
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, count)
    return [make_poisson(space, 2, 2, [int(n), int(n)], seed=seed + 10 * i) for i, n in enumerate(sizes)]


def test_batched_pcg_vs_reference_per_system(space, reference):
    from cie_b200.linalg import BatchedConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator
    probs = systems(space, 12, seed=5)
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    solver = BatchedConjugateGradients(bd, offsets, space, D, Statistics(5000, 0.0, 1e-10))
    x = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x)
    stats = solver.getStats()
    xh = x.cpu().numpy()
    print(solver.info())
    for s, p in enumerate(probs):
        rp, col, val = p.host_csr()
        b = p.rhs.cpu().numpy()
        xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=5000, abstol=0.0, reltol=1e-10)
        xs = xh[offsets[s]:offsets[s + 1]]
        rel = np.linalg.norm(xs - xr) / np.linalg.norm(xr)
        assert err is None
        assert stats[s].iterationCount == int(sr[0]), (s, stats[s].iterationCount, sr[0])
        assert abs(stats[s].relativeResidual - sr[2]) <= 1e-6 * sr[2]
        assert rel <= 1e-9, (s, rel)


def test_batched_pcg_initial_guess_scales_and_limits(space):
    from cie_b200.linalg import (BatchedConjugateGradients, CSROperator, ConjugateGradients, Statistics,
                                 block_diagonal, makeDiagonalOperator)
    probs = systems(space, 5, seed=9)
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    rng = np.random.default_rng(2)
    y0 = torch.as_tensor(rng.uniform(-1, 1, rhs.numel())).cuda()
    for settings in (Statistics(5000, 0.0, 1e-10), Statistics(7, 0.0, 1e-10), Statistics(5000, 1e-3, 0.0)):
        solver = BatchedConjugateGradients(bd, offsets, space, D, settings)
        out = y0.clone()
        solver.product(2.0, rhs, -0.5, out)
        for s, p in enumerate(probs):
            A = CSROperator(p.matrix, space)
            cg = ConjugateGradients(A, space, makeDiagonalOperator(p.matrix, space, csr_handle=A.csr), settings)
            o = y0[offsets[s]:offsets[s + 1]].clone()
            cg.product(2.0, p.rhs, -0.5, o)
            st = solver.getStats()[s]
            assert st.iterationCount == cg.getStats().iterationCount
            # the batched dots reduce per tile, the single solver per grid: rounding differs
            got = out[offsets[s]:offsets[s + 1]]
            assert float(torch.linalg.norm(got - o) / torch.linalg.norm(o)) <= 1e-9


def test_batched_pcg_rejects_coupled_blocks(space):
    from cie_b200._lib import CiecuError
    from cie_b200.linalg import BatchedConjugateGradients, CSRMatrix, Statistics, makeDiagonalOperator
    # 4 rows, two 2x2 blocks, plus an entry coupling row 1 to column 2
    rp = torch.tensor([0, 2, 5, 7, 9], dtype=torch.int32).cuda()
    col = torch.tensor([0, 1, 0, 1, 2, 2, 3, 2, 3], dtype=torch.int32).cuda()
    val = torch.tensor([4, -1, -1, 4, -1, 4, -1, -1, 4], dtype=torch.float64).cuda()
    m = CSRMatrix(4, rp, col, val)
    D = makeDiagonalOperator(m, space)
    with pytest.raises(CiecuError, match="row 1 has an entry outside its system"):
        BatchedConjugateGradients(m, np.array([0, 2, 4]), space, D, Statistics(100, 0.0, 1e-10))


def test_batched_pcg_breakdown_names_the_system(space):
    from cie_b200._lib import CiecuError
    from cie_b200.linalg import BatchedConjugateGradients, CSRMatrix, Statistics, block_diagonal, makeDiagonalOperator
    probs = systems(space, 3, seed=13)
    mats = [p.matrix for p in probs]
    bad = mats[1]
    # an indefinite block: the first half of its diagonal entries negated
    entries = bad.entries.clone()
    rp = bad.rowExtents.cpu().numpy()
    cols = bad.columnIndices.cpu().numpy()
    diag = np.array([rp[i] + np.flatnonzero(cols[rp[i]:rp[i + 1]] == i)[0] for i in range(bad.rowCount())])
    half = diag[: len(diag) // 2]
    entries[torch.as_tensor(half).cuda()] *= -1.0
    mats[1] = CSRMatrix(bad.columnCount, bad.rowExtents, bad.columnIndices, entries)
    bd, offsets = block_diagonal(mats)
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    solver = BatchedConjugateGradients(bd, offsets, space, D, Statistics(5000, 0.0, 1e-10))
    x = torch.zeros_like(rhs)
    with pytest.raises(CiecuError, match=r"system 1: "):
        solver.product(0.0, rhs, 1.0, x)
    stats = solver.getStats()
    assert stats[0].relativeResidual <= 1e-10 and stats[2].relativeResidual <= 1e-10


def test_batched_fp32_refined_vs_reference(space, reference):
    """FP32 inner solves with FP64 refinement (set_refinement): every system reaches
    its true FP64 relative residual 1e-10 and lands within 1e-9 of the reference
    CG's solution."""
    from cie_b200.linalg import BatchedConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator
    probs = systems(space, 10, seed=17)
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    solver = BatchedConjugateGradients(bd, offsets, space, D, Statistics(20000, 0.0, 1e-10))
    solver.set_refinement(1e-3)
    x = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x)
    stats = solver.getStats()
    xh = x.cpu().numpy()
    for s, p in enumerate(probs):
        rp, col, val = p.host_csr()
        b = p.rhs.cpu().numpy()
        xs = xh[offsets[s]:offsets[s + 1]]
        xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=20000, abstol=0.0, reltol=1e-10)
        r = b - np.array([val[rp[i]:rp[i + 1]] @ xs[col[rp[i]:rp[i + 1]]] for i in range(len(b))])
        assert stats[s].relativeResidual <= 1e-10, (s, stats[s].relativeResidual)
        assert np.linalg.norm(r) <= 1.05e-10 * np.linalg.norm(b)
        assert np.linalg.norm(xs - xr) <= 1e-9 * np.linalg.norm(xr)
    print("refined: inner iterations %s (FP64 reference %s)" % ([st.iterationCount for st in stats[:4]], int(sr[0])))


@pytest.mark.parametrize("delta", [0.1, 0.01])
def test_batched_reliable_updates_vs_reference(space, reference, delta):
    """FP32 iterations per system with FP64 reliable updates
    (set_reliable_updates): every system's true FP64 residual at the 1e-10 stop,
    its solution within 1e-9 of the reference CG's, at least one replacement, and
    an iteration count near the FP64 one (the Krylov space is kept)."""
    from cie_b200.linalg import BatchedConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator
    from oracle.oracle import Restatement
    probs = systems(space, 10, seed=19)
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    solver = BatchedConjugateGradients(bd, offsets, space, D, Statistics(20000, 0.0, 1e-10))
    solver.set_reliable_updates(delta)
    x = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x)
    stats = solver.getStats()
    reps = solver.refinements()
    xh = x.cpu().numpy()
    ora = Restatement()
    for s, p in enumerate(probs):
        rp, col, val = p.host_csr()
        b = p.rhs.cpu().numpy()
        xs = xh[offsets[s]:offsets[s + 1]].copy()
        xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=20000, abstol=0.0, reltol=1e-10)
        r = ora.spmv(rp, col, val, 1.0, xs, -1.0, b)
        assert stats[s].relativeResidual < 1e-10, (s, stats[s].relativeResidual)
        assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b), s
        assert np.linalg.norm(xs - xr) <= 1e-9 * np.linalg.norm(xr), s
        assert reps[s] >= 1
        assert stats[s].iterationCount <= 1.3 * int(sr[0]) + 10, (s, stats[s].iterationCount, sr[0])
    print("reliable updates delta %g: iterations %s, replacements %s" % (delta, [st.iterationCount for st in stats[:4]],
                                                                       reps[:4]))


def test_batched_reliable_updates_limits_and_switch(space):
    """The iteration limit in the reliable-update form (FP64 residual reported),
    and one solver switched between the FP64 and reliable-update forms."""
    from cie_b200.linalg import BatchedConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator
    probs = systems(space, 5, seed=23)
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    D = makeDiagonalOperator(bd, space)
    limited = BatchedConjugateGradients(bd, offsets, space, D, Statistics(7, 0.0, 1e-10))
    limited.set_reliable_updates(0.1)
    x = torch.zeros_like(rhs)
    limited.product(0.0, rhs, 1.0, x)
    for st in limited.getStats():
        assert st.iterationCount == 7 and 1e-10 < st.relativeResidual < 1.0
    solver = BatchedConjugateGradients(bd, offsets, space, D, Statistics(20000, 0.0, 1e-10))
    x64 = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x64)
    solver.set_reliable_updates(0.1)
    x32 = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x32)
    solver.set_reliable_updates(0.0)
    x64b = torch.zeros_like(rhs)
    solver.product(0.0, rhs, 1.0, x64b)
    assert torch.equal(x64, x64b)
    assert float(torch.linalg.norm(x32 - x64) / torch.linalg.norm(x64)) <= 1e-9
