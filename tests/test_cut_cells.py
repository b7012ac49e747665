"""The restated cut-cell quadrature (KDTreeQuadraturePointFactory.hpp:67-173 for
a sphere; no buildable reference for it here), pinned by properties: a cell
fully inside or outside keeps the plain tensor Gauss rule (scale 1 / alpha); on a
cut cell the kept points and weights follow the keep rule; and the quadrature
of the indicator function converges to the sphere's volume with the depth."""
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
