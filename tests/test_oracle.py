"""Pins the oracle before it is trusted: the C restatement against the reference's
own known-answer tests (tests/golden) and against the reference's compiled CPU
solver on identical seeded inputs.  CPU only."""
import numpy as np
import pytest


def poisson2d(n):
    """5-point Dirichlet Laplacian on an n x n interior grid (small SPD test matrix)."""
    N = n * n
    rows, cols, vals = [], [], []
    for j in range(n):
        for i in range(n):
            r = j * n + i
            for dj, di, v in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
                jj, ii = j + dj, i + di
                if 0 <= jj < n and 0 <= ii < n:
                    rows.append(r)
                    cols.append(jj * n + ii)
                    vals.append(v)
    rowptr = np.zeros(N + 1, dtype=np.int32)
    np.add.at(rowptr, np.array(rows) + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, np.array(cols, dtype=np.int32), np.array(vals)


def random_csr(n, m, density, seed):
    rng = np.random.default_rng(seed)
    rowptr = [0]
    cols = []
    for _ in range(n):
        k = rng.binomial(m, density)
        c = np.sort(rng.choice(m, size=k, replace=False))
        cols.extend(c)
        rowptr.append(len(cols))
    return (np.array(rowptr, dtype=np.int32), np.array(cols, dtype=np.int32), rng.uniform(-1, 1, len(cols)))


# ---- goldens ------------------------------------------------------------------

def test_spmv_known_answer(restatement, golden):
    c = golden["linalg_space"]["spmv"]
    y = restatement.spmv(np.array(c["row_extents"], np.int32), np.array(c["column_indices"], np.int32),
                         np.array(c["entries"]), c["in_scale"], np.array(c["in"]), c["out_scale"],
                         np.array(c["out_initial"]))
    assert np.allclose(y, c["expected"], rtol=1e-15)


def test_masked_spmv_known_answer(restatement, golden):
    c = golden["linalg_space"]["masked_spmv"]
    y = restatement.masked_spmv(np.array(c["row_extents"], np.int32), np.array(c["column_indices"], np.int32),
                                np.array(c["entries"]), np.array(c["mask"]), c["threshold"], c["in_scale"],
                                np.array(c["in"]), c["out_scale"], np.array(c["out_initial"]))
    # The SYCL test expects the masked row to keep inScale*out (9 * 1000); the CPU
    # MaskedCSROperator writes combine(inScale, out, outScale, 0) = inScale*out too
    # for inScale not in {0, 1, -1}.
    assert np.allclose(y, c["expected"], rtol=1e-15)


def test_inner_product_known_answer(restatement, golden):
    for case in golden["linalg_space"]["inner_product"][:5]:
        n = case["size"]
        a = np.arange(n, dtype=np.float64)
        b = -np.ones(n)
        assert restatement.L.ora_dot(n, a.ctypes.data, b.ctypes.data) == pytest.approx(case["expected"], rel=1e-12)


def catch_approx(actual, expected, margin):
    """Catch2's Approx(expected).margin(m): |a-b| <= margin or within the default
    relative epsilon 100 * FLT_EPSILON (the reference test's comparison)."""
    actual, expected = np.asarray(actual), np.asarray(expected)
    diff = np.abs(actual - expected)
    return bool(np.all((diff <= margin) | (diff <= 100 * np.finfo(np.float32).eps * np.abs(expected))))


def test_gauss_legendre_tables(restatement, golden):
    tol = golden["gauss_legendre"]["max_absolute_error"]
    for case in golden["gauss_legendre"]["cases"]:
        n, w = restatement.gauss_legendre(case["order"])
        assert catch_approx(n, case["nodes"], tol) and catch_approx(w, case["weights"], tol)
        # the tables themselves carry 16 digits; the Newton nodes match them to 1e-14
        assert np.max(np.abs(n - case["nodes"])) < 1e-14
        assert np.max(np.abs(w - case["weights"])) < 1e-14


def test_gauss_legendre_restatement_vs_reference(restatement, reference):
    for order in range(1, 21):
        n, w = restatement.gauss_legendre(order)
        nr, wr = reference.gauss_legendre(order)
        assert np.max(np.abs(n - nr)) <= 1e-15 and np.max(np.abs(w - wr)) <= 1e-15


def test_stiffness_integrand_known_answer(restatement, golden):
    g = golden["stiffness_integrand"]
    for case in g["cases"]:
        out = restatement.stiffness_point(g["dimension"], g["basis_coefficients"], case["point"], g["modulus"])
        assert np.max(np.abs(out - g["modulus"] * np.array(case["reference"]))) <= g["margin"]


def test_transformed_integral_identities(restatement):
    # Sum of the element matrix rows vanishes (constants are in the kernel) and the
    # quadrature integrates the Q_p gradient products exactly: compare order+1 with
    # a higher-order rule.
    for dim, order in ((2, 1), (3, 1), (2, 2), (3, 3)):
        K = restatement.element_stiffness(dim, order, 1.0, [0.5] * dim).reshape((order + 1) ** dim, -1)
        assert np.max(np.abs(K.sum(axis=1))) < 1e-12 * np.abs(K).max()
        pts, wts = restatement.tensor_gauss(dim, order + 3)
        K2 = restatement.element_stiffness(dim, order, 1.0, [0.5] * dim, points=pts, weights=wts).reshape(K.shape)
        assert np.allclose(K, K2, rtol=1e-12, atol=1e-12)
        assert np.allclose(K, K.T, atol=1e-14)


def test_q1_2d_element_matches_closed_form(restatement):
    # Bilinear square, parametric gradients: sum_q w G^T G = [[4,-1,-1,-2],...]/6,
    # times |det J^-1| = (2/h)^2 for the reference convention.
    K = restatement.element_stiffness(2, 1, 1.0, [2.0, 2.0]).reshape(4, 4)
    expected = np.array([[4, -1, -1, -2], [-1, 4, -2, -1], [-1, -2, 4, -1], [-2, -1, -1, 4]]) / 6.0
    assert np.allclose(K, expected, atol=1e-15)
    Kp = restatement.element_stiffness(2, 1, 1.0, [0.25, 0.25], convention=1).reshape(4, 4)
    assert np.allclose(Kp, expected, atol=1e-14)  # physical 2-D stiffness is h-independent


# ---- oracle vs the compiled reference -------------------------------------------


def lagrange_nodes(order, kind):
    """Equispaced nodes -1 + 2i/p (the build's Q_p basis) or Chebyshev-Lobatto
    nodes -cos(i pi / p) (the reference's Lagrange example), ascending."""
    i = np.arange(order + 1)
    return -1.0 + 2.0 * i / order if kind == "equispaced" else -np.cos(i * np.pi / order)


@pytest.mark.parametrize("kind", ["equispaced", "chebyshev-lobatto"])
def test_lagrange_basis_restatement_vs_reference(restatement, reference, kind):
    """The restated product-form Lagrange values and derivatives against the
    reference's LagrangePolynomial (coefficients from LagrangePolynomial.cpp:18-72,
    Horner evaluation and makeDerivative of Polynomial_impl.hpp), Q1..Q5, at the
    Gauss points of the rules the assembly uses and at random points of [-1, 1]."""
    import ctypes
    rng = np.random.default_rng(9)
    for order in range(1, 6):
        nodes = lagrange_nodes(order, kind)
        points = np.concatenate([reference.gauss_legendre(q)[0] for q in range(2, 7)] + [rng.uniform(-1, 1, 16)])
        for base in range(order + 1):
            c, v_ref, d_ref = reference.lagrange(nodes, base, points)
            assert abs(np.polyval(c[::-1], nodes[base]) - 1.0) <= 1e-13
            for k, x in enumerate(points):
                vals, ders = np.zeros(order + 1), np.zeros(order + 1)
                restatement.L.ora_lagrange_1d(order + 1, nodes.ctypes.data_as(ctypes.c_void_p), float(x),
                                              vals.ctypes.data_as(ctypes.c_void_p),
                                              ders.ctypes.data_as(ctypes.c_void_p))
                assert abs(vals[base] - v_ref[k]) <= 1e-13, (order, base, x)
                assert abs(ders[base] - d_ref[k]) <= 1e-12 * max(1.0, abs(d_ref[k])), (order, base, x)


@pytest.mark.parametrize("dim,order", [(2, 2), (2, 3), (3, 2), (3, 3)])
def test_element_stiffness_with_reference_basis(restatement, reference, dim, order):
    """Q2/Q3 element matrices of the restatement (the checker of the GPU assembly)
    against the same integral built from the reference's own basis: the
    LagrangePolynomial coefficient vectors evaluated by the restated integrand at
    the reference's Gauss points, K = prod(2/h) sum_q w_q kappa G_q^T G_q."""
    nodes = lagrange_nodes(order, "equispaced")
    coefficients = np.array([reference.lagrange(nodes, i, [0.0])[0] for i in range(order + 1)])
    n1, w1 = reference.gauss_legendre(order + 1)
    q = np.arange((order + 1) ** dim)
    idx = (q[:, None] // (order + 1) ** np.arange(dim)[None, :]) % (order + 1)
    h = [0.25, 0.5, 0.125][:dim]
    kappa = 1.7
    K = 0.0
    for pt, w in zip(n1[idx], np.prod(w1[idx], axis=1)):
        K = K + w * restatement.stiffness_point(dim, coefficients, pt, kappa)
    K *= np.prod(2.0 / np.array(h))
    Kr = restatement.element_stiffness(dim, order, kappa, h)
    assert np.max(np.abs(K - Kr)) <= 1e-13 * np.abs(Kr).max()


def test_reference_matches_goldens(reference, golden):
    c = golden["linalg_space"]["spmv"]
    y = reference.spmv(np.array(c["row_extents"], np.int32), np.array(c["column_indices"], np.int32),
                       np.array(c["entries"]), c["in_scale"], np.array(c["in"]), c["out_scale"],
                       np.array(c["out_initial"]))
    assert np.allclose(y, c["expected"])
    c = golden["linalg_space"]["masked_spmv"]
    y = reference.masked_spmv(np.array(c["row_extents"], np.int32), np.array(c["column_indices"], np.int32),
                              np.array(c["entries"]), np.array(c["mask"]), c["threshold"], c["in_scale"],
                              np.array(c["in"]), c["out_scale"], np.array(c["out_initial"]))
    assert np.allclose(y, c["expected"])
    tol = golden["gauss_legendre"]["max_absolute_error"]
    for case in golden["gauss_legendre"]["cases"]:
        n, w = reference.gauss_legendre(case["order"])
        assert catch_approx(n, case["nodes"], tol) and catch_approx(w, case["weights"], tol)


@pytest.mark.parametrize("scales", [(0, 1), (1, -1), (1, 1), (-1, 1), (-1, -1), (0, -1), (2.5, -0.75), (1, 3.0)])
def test_spmv_restatement_vs_reference(restatement, reference, scales):
    rowptr, col, val = random_csr(300, 250, 0.04, 1)
    rng = np.random.default_rng(2)
    x, y0 = rng.uniform(-1, 1, 250), rng.uniform(-1, 1, 300)
    a = restatement.spmv(rowptr, col, val, scales[0], x, scales[1], y0)
    b = reference.spmv(rowptr, col, val, scales[0], x, scales[1], y0)
    scale = np.abs(val[None, :]).max() * 250
    assert np.max(np.abs(a - b)) <= 1e-14 * scale


def test_masked_spmv_restatement_vs_reference(restatement, reference):
    rowptr, col, val = poisson2d(12)
    rng = np.random.default_rng(3)
    mask = rng.integers(1, 4, len(rowptr) - 1)
    x, y0 = rng.uniform(-1, 1, len(rowptr) - 1), rng.uniform(-1, 1, len(rowptr) - 1)
    for thr in (2, 3):
        a = restatement.masked_spmv(rowptr, col, val, mask, thr, 0.5, x, 2.0, y0)
        b = reference.masked_spmv(rowptr, col, val, mask, thr, 0.5, x, 2.0, y0)
        assert np.allclose(a, b, rtol=1e-14, atol=1e-14)


def test_pcg_restatement_vs_reference(restatement, reference):
    rowptr, col, val = poisson2d(40)
    b = np.random.default_rng(4).uniform(-1, 1, len(rowptr) - 1)
    xa, sa, st = restatement.pcg(rowptr, col, val, b, reltol=1e-10)
    xb, sb, err, _ = reference.pcg(rowptr, col, val, b, reltol=1e-10)
    assert st == 0 and err is None
    assert sa[0] == sb[0]  # same iteration count
    assert np.linalg.norm(xa - xb) <= 1e-9 * np.linalg.norm(xb)
    r = b - np.array([val[rowptr[i]:rowptr[i + 1]] @ xa[col[rowptr[i]:rowptr[i + 1]]] for i in range(len(b))])
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)


def test_pcg_unpreconditioned_and_limits(restatement, reference):
    rowptr, col, val = poisson2d(10)
    b = np.random.default_rng(5).uniform(-1, 1, 100)
    for kw in (dict(precondition=False), dict(maxit=7), dict(abstol=1e-3, reltol=0.0), dict(maxit=0)):
        xa, sa, _ = restatement.pcg(rowptr, col, val, b, **kw)
        xb, sb, err, _ = reference.pcg(rowptr, col, val, b, **kw)
        assert err is None
        assert sa[0] == sb[0]
        assert np.allclose(xa, xb, rtol=1e-10, atol=1e-12)


def test_pcg_breakdown_matches_reference(restatement, reference):
    # indefinite matrix: p^T A p <= 0 must be reported by both
    rowptr = np.array([0, 1, 2], np.int32)
    col = np.array([0, 1], np.int32)
    val = np.array([1.0, -1.0])
    b = np.array([0.0, 1.0])
    _, _, st = restatement.pcg(rowptr, col, val, b, precondition=False)
    _, _, err, _ = reference.pcg(rowptr, col, val, b, precondition=False)
    assert st == 2 and err is not None and "vanished" in err


def test_diag_inverse_vs_reference(restatement, reference):
    rowptr, col, val = poisson2d(6)
    a, bad = restatement.diag_inverse(rowptr, col, val)
    b, err = reference.diag_inverse(rowptr, col, val)
    assert bad == -1 and err is None and np.array_equal(a, b)
    val2 = val.copy()
    val2[rowptr[7]:rowptr[8]][col[rowptr[7]:rowptr[8]] == 7] = 0.0
    _, bad = restatement.diag_inverse(rowptr, col, val2)
    _, err = reference.diag_inverse(rowptr, col, val2)
    assert bad == 7 and "row 7" in err


def test_jacobi_vs_reference(restatement, reference):
    rowptr, col, val = poisson2d(9)
    n = len(rowptr) - 1
    rng = np.random.default_rng(6)
    x, y0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    dinv, _ = restatement.diag_inverse(rowptr, col, val)
    for its, w, si, so in ((1, 1.0, 0, 1), (6, 2.0 / 3.0, 0, 1), (3, 0.5, 1, -1), (2, 0.8, 2.0, 0.5)):
        a = restatement.jacobi(rowptr, col, val, dinv, its, w, si, x, so, y0)
        b = reference.jacobi(rowptr, col, val, its, w, si, x, so, y0)
        assert np.allclose(a, b, rtol=1e-13, atol=1e-13)


def test_space_ops_vs_reference(restatement, reference):
    rng = np.random.default_rng(7)
    a, b = rng.uniform(-1, 1, 1000), rng.uniform(-1, 1, 1000)
    assert reference.dot(a, b) == pytest.approx(restatement.L.ora_dot(1000, a.ctypes.data, b.ctypes.data), rel=1e-13)
    assert np.allclose(reference.space_op(0, a, b, 3.0), 3.0 * a * b)
    assert np.allclose(reference.space_op(2, a, b, -2.0), a - 2.0 * b)


def test_pattern_and_assembly_restatement(restatement):
    # 2 x 3 bilinear grid: 12 DoFs, pattern = union of element DoF sets
    dofmap = restatement.structured_dofmap(2, 1, [2, 3])
    rowptr, col = restatement.csr_pattern(6, 4, dofmap, 12)
    assert rowptr[-1] == sum(len({c for e in range(6) if r in dofmap[4 * e:4 * e + 4]
                                  for c in dofmap[4 * e:4 * e + 4]}) for r in range(12))
    for r in range(12):
        seg = col[rowptr[r]:rowptr[r + 1]]
        assert np.all(np.diff(seg) > 0)
    Ke = np.tile(restatement.element_stiffness(2, 1, 1.0, [0.5, 1.0 / 3.0]), 6)
    val, st = restatement.assemble(6, 4, dofmap, Ke, rowptr, col)
    assert st == 0
    # constant vector in the kernel, symmetric
    y = restatement.spmv(rowptr, col, val, 0.0, np.ones(12), 1.0, np.zeros(12))
    assert np.max(np.abs(y)) < 1e-13
