"""GPU parity of the linalg operators through the C-ABI (ciecu_*), against the
reference's known answers and the oracle on identical seeded inputs.

Tolerances: SpMV per row |y_gpu - y_ref| <= 1e-13 * sum_j |a_ij x_j| (+ the
|inScale * out| term), i.e. 1e-13 relative per row; elementwise
operations exact or 1 ulp."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from tests.test_oracle import poisson2d, random_csr  # noqa: E402


@pytest.fixture(scope="module")
def space():
    from cie_b200.linalg import CUDASpace
    return CUDASpace()


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def matrix(rowptr, col, val, ncols, dtype=torch.float64):
    from cie_b200.linalg import CSRMatrix
    return CSRMatrix(ncols, dev(rowptr, torch.int32), dev(col, torch.int32), dev(val, dtype))


def row_scale(rowptr, col, val, x, inScale, y0):
    absrow = np.zeros(len(rowptr) - 1)
    for i in range(len(rowptr) - 1):
        s = slice(rowptr[i], rowptr[i + 1])
        absrow[i] = np.sum(np.abs(val[s] * x[col[s]]))
    return absrow + np.abs(inScale * y0) + 1e-300


# ---- space (SYCLSpace_test.cpp:19-138) ----------------------------------------

def test_inner_product_known_answers(space, golden):
    for case in golden["linalg_space"]["inner_product"]:
        n = case["size"]
        a = torch.arange(n, dtype=torch.float64, device="cuda")
        b = -torch.ones(n, dtype=torch.float64, device="cuda")
        assert space.innerProduct(a, b) == pytest.approx(case["expected"], rel=1e-14)


def test_add_and_scale_known_answers(space, golden):
    g = golden["linalg_space"]
    for n in g["elementwise_sizes"]:
        src = np.arange(n, dtype=np.float64)
        s, t = dev(src), dev(g["add"]["target_factor"] * src)
        space.add(t, s, g["add"]["first_scale"])
        assert np.allclose(host(t), (1e1 + 1e2) * src, rtol=1e-15)
        space.add(t, s, g["add"]["second_scale"])
        assert np.allclose(host(t), (1e1 + 1e2 + 1) * src, rtol=1e-15)
        t = dev(src)
        space.scale(t, g["scale_uniform"]["factor"])
        assert np.array_equal(host(t), 2 * src)
        s, t = dev(src), dev(1e1 * src)
        space.scale(t, s, g["scale_componentwise"]["scale"])
        assert np.allclose(host(t), 1e1 * 1e2 * src * src, rtol=1e-15)
        # assign host -> device -> device -> host
        d1, d2 = space.makeVector(n), space.makeVector(n)
        space.assign(d1, src)
        space.assign(d2, d1)
        back = np.zeros(n)
        space.assign(back, d2)
        assert np.array_equal(back, src)


def test_space_ops_match_reference(space, reference):
    rng = np.random.default_rng(11)
    a, b = rng.uniform(-1, 1, 100003), rng.uniform(-1, 1, 100003)
    ta, tb = dev(a), dev(b)
    assert space.innerProduct(ta, tb) == pytest.approx(reference.dot(a, b), rel=1e-12)
    for op, alpha in ((0, 1.0), (0, -1.0), (0, 3.5), (2, 1.0), (2, -1.0), (2, -0.25)):
        t = dev(a)
        if op == 0:
            space.scale(t, tb, alpha)
        else:
            space.add(t, tb, alpha)
        assert np.array_equal(host(t), reference.space_op(op, a, b, alpha))
    t = dev(a)
    space.fill(t, 2.5)
    assert np.all(host(t) == 2.5)


# ---- SpMV ---------------------------------------------------------------------

def test_spmv_known_answer(space, golden):
    from cie_b200.linalg import CSROperator
    c = golden["linalg_space"]["spmv"]
    op = CSROperator(matrix(c["row_extents"], c["column_indices"], c["entries"], c["column_count"]), space)
    out = dev(c["out_initial"])
    op.product(c["in_scale"], dev(c["in"]), c["out_scale"], out)
    assert np.allclose(host(out), c["expected"], rtol=1e-15)


def test_masked_spmv_known_answer(space, golden):
    from cie_b200.linalg import MaskedCSROperator
    c = golden["linalg_space"]["masked_spmv"]
    op = MaskedCSROperator(matrix(c["row_extents"], c["column_indices"], c["entries"], c["column_count"]),
                           c["mask"], c["threshold"], space)
    out = dev(c["out_initial"])
    op.product(c["in_scale"], dev(c["in"]), c["out_scale"], out)
    assert np.allclose(host(out), c["expected"], rtol=1e-15)


SCALES = [(0, 1), (1, -1), (1, 1), (-1, 1), (-1, -1), (0, -1), (2.5, -0.75), (1, 3.0), (0, 0.5)]


@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32])
def test_spmv_all_schedules_vs_oracle(space, restatement, kernel):
    from cie_b200.linalg import CSROperator
    rowptr, col, val = random_csr(3000, 2500, 0.01, 21)
    rng = np.random.default_rng(22)
    x, y0 = rng.uniform(-1, 1, 2500), rng.uniform(-1, 1, 3000)
    op = CSROperator(matrix(rowptr, col, val, 2500), space)
    op.csr.set_kernel(kernel)
    for si, so in SCALES:
        out = dev(y0)
        op.product(si, dev(x), so, out)
        ref = restatement.spmv(rowptr, col, val, si, x, so, y0)
        err = np.abs(host(out) - ref) / row_scale(rowptr, col, val, x, si, y0)
        assert err.max() <= 1e-13, (kernel, si, so, err.max())


def test_spmv_stream_kernel_is_bitwise_on_row_sums(space, reference):
    # The row-block kernel accumulates each row in CSR order with FMA, like the
    # reference's contracted loop: for (inScale, outScale) = (0, 1) the outputs match.
    from cie_b200.linalg import CSROperator
    rowptr, col, val = random_csr(4000, 4000, 0.005, 23)
    x = np.random.default_rng(24).uniform(-1, 1, 4000)
    op = CSROperator(matrix(rowptr, col, val, 4000), space)
    op.csr.set_kernel(1)
    out = dev(np.zeros(4000))
    op.product(0, dev(x), 1, out)
    ref = reference.spmv(rowptr, col, val, 0.0, x, 1.0, np.zeros(4000))
    mismatches = int(np.sum(host(out) != ref))
    err = np.abs(host(out) - ref) / row_scale(rowptr, col, val, x, 0, np.zeros(4000))
    print("stream kernel: %d / 4000 rows differ from the reference bitwise, max normalised error %.2e"
          % (mismatches, err.max()))
    assert err.max() <= 1e-13


def test_spmv_edge_cases(space, restatement):
    from cie_b200.linalg import CSROperator
    rng = np.random.default_rng(25)
    # empty rows, a row longer than the 2048-entry tile, single-entry rows
    lens = [0, 1, 0, 5000, 3, 0, 2049, 2048, 1, 0]
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(6000, size=k, replace=False)) for k in lens]).astype(np.int32)
    val = rng.uniform(-1, 1, len(col))
    x, y0 = rng.uniform(-1, 1, 6000), rng.uniform(-1, 1, 10)
    for kernel in (0, 1, 2, 32):
        op = CSROperator(matrix(rowptr, col, val, 6000), space)
        if kernel:
            op.csr.set_kernel(kernel)
        for si, so in ((0, 1), (2.0, -1.0)):
            out = dev(y0)
            op.product(si, dev(x), so, out)
            ref = restatement.spmv(rowptr, col, val, si, x, so, y0)
            err = np.abs(host(out) - ref) / row_scale(rowptr, col, val, x, si, y0)
            assert err.max() <= 1e-13
    # zero-row matrix
    op = CSROperator(matrix(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0), space)
    op.product(0, dev(np.zeros(0)), 1, dev(np.zeros(0)))


def test_spmv_unaligned_views(space, restatement):
    # column indices / entries that start off a 16-byte boundary use the scalar staging path
    from cie_b200.linalg import CSRMatrix, CSROperator
    rowptr, col, val = random_csr(500, 500, 0.05, 26)
    x = np.random.default_rng(27).uniform(-1, 1, 500)
    col_buf = dev(np.concatenate([[0], col]), torch.int32)
    val_buf = dev(np.concatenate([[0.0], val]))
    m = CSRMatrix(500, dev(rowptr, torch.int32), col_buf[1:], val_buf[1:])
    op = CSROperator(m, space)
    out = dev(np.zeros(500))
    op.product(0, dev(x), 1, out)
    ref = restatement.spmv(rowptr, col, val, 0, x, 1, np.zeros(500))
    assert np.max(np.abs(host(out) - ref) / row_scale(rowptr, col, val, x, 0, np.zeros(500))) <= 1e-13


def test_spmv_f32(restatement):
    from cie_b200.linalg import CUDASpace, CSROperator
    sp32 = CUDASpace(dtype=torch.float32)
    rowptr, col, val = random_csr(2000, 2000, 0.01, 28)
    val32 = val.astype(np.float32)
    x = np.random.default_rng(29).uniform(-1, 1, 2000).astype(np.float32)
    for kernel in (1, 4, 32):
        op = CSROperator(matrix(rowptr, col, val32, 2000, torch.float32), sp32)
        op.csr.set_kernel(kernel)
        out = dev(np.zeros(2000), torch.float32)
        op.product(0, dev(x, torch.float32), 1, out)
        ref = restatement.spmv(rowptr, col, val32.astype(np.float64), 0, x.astype(np.float64), 1, np.zeros(2000))
        err = np.abs(host(out) - ref) / row_scale(rowptr, col, val32.astype(np.float64), x.astype(np.float64), 0,
                                                   np.zeros(2000))
        assert err.max() <= 1e-5


def test_spmv_poisson_vs_reference(space, reference):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CSROperator
    prob = make_poisson(space, 2, 1, [256, 256], seed=0, kappa="one")
    rp, col, val = prob.host_csr()
    x = np.random.default_rng(30).uniform(-1, 1, len(rp) - 1)
    op = CSROperator(prob.matrix, space)
    for si, so in ((0, 1), (1, -1)):
        y0 = np.random.default_rng(31).uniform(-1, 1, len(rp) - 1)
        out = dev(y0)
        op.product(si, dev(x), so, out)
        ref = reference.spmv(rp, col, val, si, x, so, y0)
        err = np.abs(host(out) - ref) / row_scale(rp, col, val, x, si, y0)
        assert err.max() <= 1e-13


def test_csr_create_rejects_inconsistent_extents(space):
    from cie_b200.linalg import CSROperator
    from cie_b200._lib import CiecuError
    with pytest.raises(CiecuError):
        CSROperator(matrix([0, 2, 1], [0, 1], [1.0, 2.0], 2), space)
    with pytest.raises(CiecuError):
        CSROperator(matrix([0, 1, 3], [0, 1], [1.0, 2.0], 2), space)


# ---- diagonal, Jacobi, masked identity, Chebyshev --------------------------------

def test_diagonal_inverse_and_errors(space, reference):
    from cie_b200.linalg import makeDiagonalOperator
    from cie_b200._lib import CiecuError
    rp, col, val = poisson2d(20)
    d = makeDiagonalOperator(matrix(rp, col, val, 400), space)
    ref, err = reference.diag_inverse(rp, col, val)
    assert err is None and np.array_equal(host(d.inverseDiagonal), ref)
    val2 = val.copy()
    k = rp[37] + int(np.flatnonzero(col[rp[37]:rp[38]] == 37)[0])
    val2[k] = 0.0
    with pytest.raises(CiecuError, match="row 37 has an explicit zero on its diagonal"):
        makeDiagonalOperator(matrix(rp, col, val2, 400), space)
    keep = np.ones(len(col), bool)
    keep[rp[5] + int(np.flatnonzero(col[rp[5]:rp[6]] == 5)[0])] = False
    rp3 = np.concatenate([[0], np.cumsum([np.sum(keep[rp[i]:rp[i + 1]]) for i in range(400)])]).astype(np.int32)
    with pytest.raises(CiecuError, match="row 5 has no diagonal entry"):
        makeDiagonalOperator(matrix(rp3, col[keep], val[keep], 400), space)


def test_diagonal_apply(space):
    from cie_b200.linalg import DiagonalOperator
    rng = np.random.default_rng(32)
    dinv, x, y0 = rng.uniform(0.5, 2, 1000), rng.uniform(-1, 1, 1000), rng.uniform(-1, 1, 1000)
    op = DiagonalOperator(dev(dinv), space)
    for si, so in ((0, 1), (1, 1), (2.0, -3.0)):
        out = dev(y0)
        op.product(si, dev(x), so, out)
        b = x * dinv if so == 1 else so * x * dinv
        expect = b if si == 0 else (y0 if si == 1 else y0 * si) + b
        assert np.allclose(host(out), expect, rtol=1e-15, atol=1e-16)


@pytest.mark.parametrize("iterations,relaxation,si,so", [(1, 1.0, 0, 1), (6, 2.0 / 3.0, 0, 1), (3, 0.5, 1, -1),
                                                         (2, 0.8, 2.0, 0.5)])
def test_jacobi_vs_reference(space, reference, iterations, relaxation, si, so):
    from cie_b200.linalg import CSROperator, JacobiOperator, makeDiagonalOperator
    rp, col, val = poisson2d(30)
    n = len(rp) - 1
    rng = np.random.default_rng(33)
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    m = matrix(rp, col, val, n)
    A = CSROperator(m, space)
    J = JacobiOperator(space, n, A, makeDiagonalOperator(m, space), iterations, relaxation)
    out = dev(y0)
    J.product(si, dev(x), so, out)
    ref = reference.jacobi(rp, col, val, iterations, relaxation, si, x, so, y0)
    assert np.allclose(host(out), ref, rtol=1e-13, atol=1e-13)


def test_masked_jacobi_and_identity_vs_oracle(space, restatement):
    from cie_b200.linalg import MaskedCSROperator, JacobiOperator, MaskedIdentityOperator, makeDiagonalOperator
    rp, col, val = poisson2d(25)
    n = len(rp) - 1
    rng = np.random.default_rng(34)
    mask = rng.integers(1, 5, n).astype(np.uint16)
    x = rng.uniform(-1, 1, n)
    m = matrix(rp, col, val, n)
    dinv = makeDiagonalOperator(m, space)
    for thr in (2, 4):
        I = MaskedIdentityOperator(space, mask, thr)
        g = dev(np.zeros(n))
        I.product(0, dev(x), 1, g)
        gx = np.where(mask < thr, x, 0.0)
        assert np.array_equal(host(g), gx)
        A = MaskedCSROperator(m, mask, thr, space)
        J = JacobiOperator(space, n, A, dinv, 6, 2.0 / 3.0)
        out = dev(np.zeros(n))
        J.product(0, g, 1, out)
        # oracle: Jacobi sweeps over the masked operator
        xk = np.zeros(n)
        d = host(dinv.inverseDiagonal)
        for _ in range(6):
            res = gx - restatement.masked_spmv(rp, col, val, mask, thr, 0, xk, 1, np.zeros(n))
            xk = xk + (2.0 / 3.0) * res * d
        assert np.allclose(host(out), xk, rtol=1e-13, atol=1e-14)


def test_chebyshev_and_power_vs_oracle(space, restatement):
    from cie_b200.linalg import CSROperator, ChebyshevOperator, makeDiagonalOperator
    rp, col, val = poisson2d(40)
    n = len(rp) - 1
    m = matrix(rp, col, val, n)
    A = CSROperator(m, space)
    D = makeDiagonalOperator(m, space)
    dinv = host(D.inverseDiagonal)
    lam = restatement.power_lambda_max(rp, col, val, dinv, 20, 0)
    C = ChebyshevOperator(A, D, degree=5, powerIterations=20, seed=0)
    assert C.lambdaMax == pytest.approx(1.1 * lam, rel=1e-12)
    x = np.random.default_rng(35).uniform(-1, 1, n)
    out = dev(np.zeros(n))
    C.product(0, dev(x), 1, out)
    ref = restatement.chebyshev(rp, col, val, dinv, 5, C.lambdaMin, C.lambdaMax, x)
    assert np.allclose(host(out), ref, rtol=1e-12, atol=1e-13)
    # a smoother: reduces the high-frequency error of A e = 0
    r0 = x - restatement.spmv(rp, col, val, 0, host(out), 1, np.zeros(n))
    assert np.linalg.norm(r0) < np.linalg.norm(x)
