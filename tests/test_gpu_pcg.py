"""GPU parity of the conjugate-gradient solver through the C-ABI against the
reference's own compiled FP64 CPU solver (oracle/_ref) on identical seeded inputs.

Accuracy bar: at ||r||/||b|| <= 1e-10 the solution is within 1e-9 relative of
the FP64 oracle's; the iteration count matches the reference's up to the
last-bit differences of its dot products."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from tests.test_oracle import poisson2d  # noqa: E402
from tests.test_gpu_linalg import dev, host, matrix  # noqa: E402


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


def true_residual(rp, col, val, x, b):
    r = b.copy()
    for i in range(len(b)):
        s = slice(rp[i], rp[i + 1])
        r[i] -= val[s] @ x[col[s]]
    return np.linalg.norm(r) / np.linalg.norm(b)


# Loop modes of the fused solver: 1 = graph of three kernels per iteration,
# 2 = single cooperative launch with grid-wide exchanges.
LOOPS = [1, 2]


def solve_gpu(space, m, b, settings, precond=True, x0=None, si=0.0, so=1.0, loop=0):
    from cie_b200.linalg import CSROperator, ConjugateGradients, makeDiagonalOperator
    A = CSROperator(m, space)
    P = makeDiagonalOperator(m, space) if precond else None
    cg = ConjugateGradients(A, space, P, settings)
    cg.set_loop(loop)
    x = dev(np.zeros(len(b)) if x0 is None else x0)
    cg.product(si, dev(b), so, x)
    if loop:
        assert (cg.info()["loop"] == "single launch") == (loop == 2)
    return host(x), cg.getStats()


@pytest.mark.parametrize("loop", LOOPS)
def test_pcg_cfg1_vs_reference(space, reference, loop):
    """2D Q1 Poisson, 256 x 256 cells (66,049 DoFs), Jacobi-PCG to 1e-10."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import Statistics
    prob = make_poisson(space, 2, 1, [256, 256], seed=0, kappa="one")
    rp, col, val = prob.host_csr()
    b = host(prob.rhs)
    x, st = solve_gpu(space, prob.matrix, b, Statistics(5000, 0.0, 1e-10), loop=loop)
    xr, sr, err, secs = reference.pcg(rp, col, val, b, maxit=5000, abstol=0.0, reltol=1e-10)
    assert err is None
    rel = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    print("cfg1: GPU %d it, reference %d it, |x-x_ref|/|x_ref| = %.3e, true rel residual %.3e"
          % (st.iterationCount, sr[0], rel, true_residual(rp, col, val, x, b)))
    assert abs(st.iterationCount - sr[0]) <= 2
    assert st.relativeResidual < 1e-10
    assert rel <= 1e-9
    assert true_residual(rp, col, val, x, b) <= 2e-10


@pytest.mark.parametrize("loop", LOOPS)
def test_pcg_3d_lognormal_vs_reference(space, reference, loop):
    """3D Q1, 32^3 cells with the smoothed log-normal kappa field."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import Statistics
    prob = make_poisson(space, 3, 1, [32, 32, 32], seed=3)
    rp, col, val = prob.host_csr()
    b = host(prob.rhs)
    x, st = solve_gpu(space, prob.matrix, b, Statistics(5000, 0.0, 1e-10), loop=loop)
    xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=5000, abstol=0.0, reltol=1e-10)
    rel = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    print("3D lognormal: GPU %d it, reference %d it, rel diff %.3e" % (st.iterationCount, sr[0], rel))
    assert abs(st.iterationCount - sr[0]) <= 2 and rel <= 1e-9


@pytest.mark.parametrize("loop", LOOPS)
@pytest.mark.parametrize("case", ["unpreconditioned", "maxit", "abstol", "maxit0", "guess", "scales", "scales2"])
def test_pcg_settings_vs_reference(space, reference, case, loop):
    from cie_b200.linalg import Statistics
    rp, col, val = poisson2d(30)
    n = len(rp) - 1
    rng = np.random.default_rng(40)
    b = rng.uniform(-1, 1, n)
    x0 = rng.uniform(-1, 1, n) if case == "guess" else None
    kw = dict(maxit=5000, abstol=0.0, reltol=1e-10, precondition=True)
    si, so = 0.0, 1.0
    if case == "unpreconditioned":
        kw["precondition"] = False
    elif case == "maxit":
        kw["maxit"] = 7
    elif case == "abstol":
        kw.update(abstol=1e-4, reltol=0.0)
    elif case == "maxit0":
        kw["maxit"] = 0
    m = matrix(rp, col, val, n)
    settings = Statistics(kw["maxit"], kw["abstol"], kw["reltol"])
    x, st = solve_gpu(space, m, b, settings, precond=kw["precondition"], x0=x0, loop=loop)
    xr, sr, err, _ = reference.pcg(rp, col, val, b, x0=x0, **kw)
    assert err is None
    assert abs(st.iterationCount - sr[0]) <= 1
    assert np.allclose(x, xr, rtol=1e-9, atol=1e-12)
    if case.startswith("scales"):
        pass
    if case in ("scales", "scales2"):
        si, so = (1.0, -2.0) if case == "scales" else (0.5, 3.0)
        y0 = rng.uniform(-1, 1, n)
        y, _ = solve_gpu(space, m, b, settings, x0=y0, si=si, so=so, loop=loop)
        xr2, _, _, _ = reference.pcg(rp, col, val, b, x0=y0, **kw)
        assert np.allclose(y, si * y0 + so * xr2, rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("schedule", [64, 4])
def test_pcg_dia_schedule_vs_reference(space, reference, schedule):
    """The FP64 K1 over the diagonal-storage copy (27 diagonals of the 3D Q1 grid)
    against the reference solver; the copy follows changed CSR values."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 3, 1, [48, 48, 48], seed=3)
    rp, col, val = prob.host_csr()
    b = host(prob.rhs)
    A = CSROperator(prob.matrix, space)
    assert A.csr.diagonals() == 27
    cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr),
                            Statistics(5000, 0.0, 1e-10))
    cg.set_loop(1)
    cg.set_schedule(schedule)
    x = dev(np.zeros(len(b)))
    cg.product(0.0, dev(b), 1.0, x)
    assert cg.info()["spmv_schedule"] == schedule
    if schedule == 64:
        # the assembled matrix is bitwise symmetric: K1 reads the upper half only
        assert cg.info()["dia_symmetric"] and cg.info()["dia_stored_diagonals"] == 14
    xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=5000, abstol=0.0, reltol=1e-10)
    rel = np.linalg.norm(host(x) - xr) / np.linalg.norm(xr)
    assert abs(cg.getStats().iterationCount - sr[0]) <= 2 and rel <= 1e-9
    # scale the matrix in place: the next solve must see the new values
    prob.matrix.entries.mul_(2.0)
    x2 = dev(np.zeros(len(b)))
    cg.product(0.0, dev(b), 1.0, x2)
    assert np.linalg.norm(2.0 * host(x2) - host(x)) <= 1e-9 * np.linalg.norm(host(x))
    if schedule == 64:
        # one entry changed on one side: the next solve finds the matrix unsymmetric,
        # reads the full copy, and still matches the reference on the changed system
        i = len(rp) // 2
        j = next(k for k in range(rp[i], rp[i + 1]) if col[k] > i)
        prob.matrix.entries[j] *= 1.001
        val3 = 2.0 * val
        val3[j] *= 1.001
        x3 = dev(np.zeros(len(b)))
        cg.product(0.0, dev(b), 1.0, x3)
        assert not cg.info()["dia_symmetric"] and cg.info()["dia_stored_diagonals"] == 27
        xr3, sr3, err3, _ = reference.pcg(rp, col, val3, b, maxit=5000, abstol=0.0, reltol=1e-10)
        assert err3 is None
        assert np.linalg.norm(host(x3) - xr3) <= 1e-9 * np.linalg.norm(xr3)


def test_pcg_dia_schedule_refused_without_diagonals(space):
    from cie_b200._lib import CiecuError
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 3, 2, [6, 6, 6], seed=1)
    A = CSROperator(prob.matrix, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space), Statistics(50, 0.0, 1e-10))
    cg.set_loop(1)
    cg.set_schedule(64)
    with pytest.raises(CiecuError, match="at most 32 diagonals"):
        cg.product(0.0, prob.rhs, 1.0, torch.zeros_like(prob.rhs))


@pytest.mark.parametrize("loop", LOOPS)
def test_pcg_breakdown_raises(space, loop):
    from cie_b200.linalg import Statistics
    from cie_b200._lib import CiecuError
    m = matrix([0, 1, 2], [0, 1], [1.0, -1.0], 2)
    with pytest.raises(CiecuError, match=r"p\^T @ A @ p vanished in iteration 0"):
        solve_gpu(space, m, np.array([0.0, 1.0]), Statistics(100, 0.0, 1e-10), precond=False, loop=loop)
    # indefinite: diag(1, 2, 3, -4) with b = 1 breaks down in a later iteration
    m = matrix([0, 1, 2, 3, 4], [0, 1, 2, 3], [1.0, 2.0, 3.0, -4.0], 4)
    with pytest.raises(CiecuError, match=r"p\^T @ A @ p vanished in iteration"):
        solve_gpu(space, m, np.ones(4), Statistics(100, 0.0, 1e-10), precond=False, loop=loop)
    # zero right-hand side with no absolute tolerance: r^T z = 0 like the reference
    rp, col, val = poisson2d(5)
    with pytest.raises(CiecuError, match="vanished in iteration 0"):
        solve_gpu(space, matrix(rp, col, val, 25), np.zeros(25), Statistics(100, 0.0, 1e-10), loop=loop)
    # ... and an early exit with an absolute tolerance
    x, st = solve_gpu(space, matrix(rp, col, val, 25), np.zeros(25), Statistics(100, 1e-12, 1e-10), loop=loop)
    assert st.iterationCount == 0 and np.all(x == 0)


def test_single_launch_wait_timeout_then_reuse(space, reference):
    """The bounded grid-wide waits of the single-launch solve: with the last block
    withholding its partial sums at the third exchange, every wait on it runs out
    (1 ms limit), the solve fails with CIECU_ERR_TIMEOUT, and the same solver then
    solves normally and matches the reference CG."""
    from cie_b200._lib import CiecuError
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 2, 1, [48, 48], seed=3)
    A = CSROperator(prob.matrix, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space), Statistics(5000, 0.0, 1e-10))
    cg.set_loop(2)
    cg.debug_exchange(1_000_000, 3)
    x = torch.zeros_like(prob.rhs)
    with pytest.raises(CiecuError, match="gave up waiting"):
        cg.product(0, prob.rhs, 1, x)
    cg.debug_exchange(2_000_000_000, 0)
    x = torch.zeros_like(prob.rhs)
    cg.product(0, prob.rhs, 1, x)
    assert cg.info()["loop"] == "single launch"
    rp, col, val = prob.host_csr()
    b = host(prob.rhs)
    xr, sr, err, _ = reference.pcg(rp, col, val, b, maxit=5000, abstol=0.0, reltol=1e-10)
    assert err is None and abs(cg.getStats().iterationCount - int(sr[0])) <= 2
    assert np.linalg.norm(host(x) - xr) <= 1e-9 * np.linalg.norm(xr)


def test_pinned_schedule_selects_the_graph_loop(space):
    """A K1 schedule pinned in the automatic loop mode runs the graph loop (the
    schedules are its kernels) instead of being ignored by the single launch."""
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 2, 1, [32, 32], seed=4)
    A = CSROperator(prob.matrix, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space), Statistics(5000, 0.0, 1e-10))
    x = torch.zeros_like(prob.rhs)
    cg.product(0, prob.rhs, 1, x)
    assert cg.info()["loop"] == "single launch"
    x1 = host(x)
    for schedule in (4, 64):
        cg.set_schedule(schedule)
        x = torch.zeros_like(prob.rhs)
        cg.product(0, prob.rhs, 1, x)
        assert cg.info()["loop"] != "single launch" and cg.info()["spmv_schedule"] == schedule
        assert np.linalg.norm(host(x) - x1) <= 1e-12 * np.linalg.norm(x1)


def test_generic_cg_over_masked_operator_vs_oracle(space, restatement):
    """The reference algorithm composed from operator products (masked operator):
    ConjugateGradients over a MaskedCSROperator, as grid 0 of the p-multigrid."""
    from cie_b200.linalg import (CSROperator, ConjugateGradients, MaskedCSROperator, Statistics,
                                 makeDiagonalOperator)
    rp, col, val = poisson2d(20)
    n = len(rp) - 1
    rng = np.random.default_rng(41)
    mask = rng.integers(1, 3, n).astype(np.uint16)
    b = np.where(mask < 2, rng.uniform(-1, 1, n), 0.0)
    m = matrix(rp, col, val, n)
    A = MaskedCSROperator(m, mask, 2, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(m, space), Statistics(500, 0.0, 1e-10))
    x = dev(np.zeros(n))
    cg.product(0, dev(b), 1, x)
    x = host(x)
    r = b - restatement.masked_spmv(rp, col, val, mask, 2, 0, x, 1, np.zeros(n))
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)
    assert np.all(x[mask >= 2] == 0)


def test_pcg_repeated_solves_are_deterministic(space):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator, ConjugateGradients, Statistics, makeDiagonalOperator
    prob = make_poisson(space, 2, 1, [64, 64], seed=1)
    A = CSROperator(prob.matrix, space)
    cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space), Statistics(5000, 0.0, 1e-10))
    outs = []
    for chunk in (1, 16, 64):
        cg.set_graph_chunk(chunk)
        x = torch.zeros_like(prob.rhs)
        cg.product(0, prob.rhs, 1, x)
        outs.append((host(x), cg.getStats().iterationCount))
    assert outs[0][1] == outs[1][1] == outs[2][1]
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][0], outs[2][0])
