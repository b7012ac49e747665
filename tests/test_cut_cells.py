"""The restated cut-cell quadrature (KDTreeQuadraturePointFactory.hpp:67-173).
The reference's factory cannot be built here: it includes
fem/packages/utilities/inc/kernel.hpp, which needs Eigen/Dense, and geo's
ContiguousSpaceTree, and Eigen is absent.  So the restatement is pinned by what
the tree rule must satisfy: a cell fully inside or outside keeps the plain tensor
Gauss rule (scale 1 / alpha); on a cut cell the kept points follow the keep rule;
on half-cells cut by a plane on a tree boundary the rule integrates polynomials
exactly; leaves that a plane cuts bound the volume error; and the quadrature of
the indicator function converges to the sphere's volume with the depth."""
import numpy as np


def test_regular_cells_keep_the_tensor_rule(restatement):
    gn, gw = restatement.gauss_legendre(4)
    for origin, scale in (([0.45, 0.45, 0.45], 1.0), ([0.0, 0.0, 0.0], 1e-6)):
        pts, w, s = restatement.cut_cell_points(3, 2, 4, [0.5] * 3, 0.4, origin, [0.05] * 3, 1e-6)
        assert len(w) == 64 and np.all(s == scale)
        assert abs(w.sum() - 8.0) <= 1e-13
        # first index fastest
        assert np.allclose(pts[:4, 0], gn) and np.allclose(pts[::4, 1][:4], gn)


def test_cut_cell_keep_rule(restatement):
    # a cell straddling the sphere surface
    pts, w, s = restatement.cut_cell_points(2, 2, 3, [0.5, 0.5], 0.4, [0.85, 0.45], [0.1, 0.1], 1e-6)
    assert len(w) % 9 == 0 and len(w) > 9
    # depth-1 nodes that are homogeneous outside are dropped; all kept weights are
    # node weights (1/2)^2 or (1/4)^2 times the tensor weights
    total = w.sum()
    assert 0 < total < 4.0
    assert set(np.round(s, 12).tolist()) <= {1.0, 1e-6}


def test_indicator_quadrature_converges_to_the_sphere_volume(restatement):
    n, r = 16, 0.4
    h = 1.0 / n
    exact = 4.0 / 3.0 * np.pi * r ** 3
    errors = []
    for depth in (0, 1, 2, 3):
        vol = 0.0
        for i in range(n):
            for j in range(n):
                for k in range(n):
                    _, w, s = restatement.cut_cell_points(3, depth, 2, [0.5] * 3, r, [i * h, j * h, k * h],
                                                          [h] * 3, 0.0)
                    vol += (w * s).sum() * (h / 2) ** 3
        errors.append(abs(vol - exact) / exact)
    assert errors[-1] < 2e-3 and errors[-1] < errors[0]


def _monomial_integral(lo, hi, exps):
    """Integral of prod_d x_d^e_d over the box [lo, hi]."""
    out = 1.0
    for a, b, e in zip(lo, hi, exps):
        out *= (b ** (e + 1) - a ** (e + 1)) / (e + 1)
    return out


def test_tree_rule_is_exact_on_tree_aligned_half_cells(restatement):
    """A plane on a tree boundary (x = 1/2, a depth-1 boundary; x = 1/4, 3/4, depth
    2) makes every node homogeneous at some depth.  The keep rule then gives a
    piecewise tensor rule: homogeneous inside nodes kept with scale 1, homogeneous
    outside nodes dropped above the maximum depth and kept with scale alpha at it.
    That rule integrates every monomial the base rule integrates (degree <= 7 per
    axis for 4 points) exactly over those pieces."""
    rng = np.random.default_rng(4)
    alpha = 1e-3
    # (offset, depth) -> x-intervals of the kept pieces with their scales
    cases = {(0.5, 1): [(0.0, 0.5, 1.0), (0.5, 1.0, alpha)],
             (0.5, 2): [(0.0, 0.5, 1.0)],
             (0.25, 2): [(0.0, 0.25, 1.0), (0.25, 0.5, alpha)],
             (0.75, 2): [(0.0, 0.75, 1.0), (0.75, 1.0, alpha)]}
    for (offset, depth), pieces in cases.items():
        pts, w, s = restatement.cut_cell_points_halfspace(3, depth, 4, [1.0, 0.0, 0.0], offset, [0.0] * 3,
                                                          [1.0] * 3, alpha)
        x = 0.5 * (pts + 1.0)                      # physical coordinates of the unit cell
        wx = w * s / 8.0                           # parametric -> physical volume, material scale
        assert np.all((s == 1.0) == (x[:, 0] < offset))
        for _ in range(12):
            e = rng.integers(0, 8, 3)
            got = np.sum(wx * np.prod(x ** e, axis=1))
            exact = sum(sc * _monomial_integral([lo, 0.0, 0.0], [hi, 1.0, 1.0], e) for lo, hi, sc in pieces)
            assert abs(got - exact) <= 1e-14 * max(1.0, abs(exact)), (offset, depth, e)


def test_tree_rule_keeps_mixed_leaves_with_material_scales(restatement):
    """A plane that cuts through leaves: the mixed nodes at the maximum depth keep
    all their points (scale alpha outside), so the inside volume is off by at most
    the volume of those leaves, and the error shrinks with the depth."""
    normal, offset = np.array([1.0, 1.0, 1.0]) / np.sqrt(3.0), 0.8
    errors = []
    for depth in (1, 2, 3, 4):
        pts, w, s = restatement.cut_cell_points_halfspace(3, depth, 2, normal, offset, [0.0] * 3, [1.0] * 3, 0.0)
        x = 0.5 * (pts + 1.0)
        inside = x @ normal < offset
        assert np.all(s[inside] == 1.0) and np.all(s[~inside] == 0.0)
        vol = np.sum(w * s) / 8.0
        # exact volume of {x in [0,1]^3 : x1 + x2 + x3 < t}, t = offset * sqrt(3) in [1, 2]
        t = offset * np.sqrt(3.0)
        exact = (t ** 3 - 3 * (t - 1) ** 3) / 6.0
        errors.append(abs(vol - exact))
    leaf = [8.0 ** -d for d in (1, 2, 3, 4)]
    assert all(err <= 3 * (2 ** d) ** 2 * lv for err, d, lv in zip(errors, (1, 2, 3, 4), leaf))
    assert errors[-1] < errors[0]
