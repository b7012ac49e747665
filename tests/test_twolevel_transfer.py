"""Grid transfer of the two-level multigrid (host set-up, no GPU): P interpolates
Q1 vertex values at the Q_p nodes -- exact for (multi)linear functions -- and R
is its transpose; boundary rows/columns are dropped on request."""
import numpy as np

from cie_b200.twolevel import prolongation


def dense(rp, col, val, ncols):
    A = np.zeros((len(rp) - 1, ncols))
    for i in range(len(rp) - 1):
        A[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    return A


def test_prolongation_is_exact_for_linear_functions():
    for dim, order, cells in [(2, 3, [3, 4]), (3, 2, [2, 3, 2]), (3, 3, [2, 2, 2])]:
        (prp, pcol, pval), (rrp, rcol, rval) = prolongation(dim, order, cells)
        nf = np.asarray(cells) * order + 1
        nc = np.asarray(cells) + 1
        P = dense(prp, pcol, pval, int(np.prod(nc)))
        R = dense(rrp, rcol, rval, int(np.prod(nf)))
        assert np.array_equal(R, P.T)
        coef = np.array([0.7, -1.3, 2.1])[:dim]
        xc = np.stack(np.meshgrid(*[np.arange(n) / (n - 1) for n in nc[::-1]], indexing="ij")[::-1], -1)
        xf = np.stack(np.meshgrid(*[np.arange(n) / (n - 1) for n in nf[::-1]], indexing="ij")[::-1], -1)
        fc = 0.5 + xc.reshape(-1, dim) @ coef
        ff = 0.5 + xf.reshape(-1, dim) @ coef
        assert np.allclose(P @ fc, ff, atol=1e-14)
        assert np.allclose(P.sum(axis=1), 1.0)


def test_prolongation_drops_boundary_rows_and_columns():
    dim, order, cells = 2, 3, [3, 3]
    nf, nc = np.asarray(cells) * order + 1, np.asarray(cells) + 1
    fb = np.zeros(int(np.prod(nf)), bool)
    fb[:nf[0]] = True
    cb = np.zeros(int(np.prod(nc)), bool)
    cb[:nc[0]] = True
    (prp, pcol, pval), _ = prolongation(dim, order, cells, fb, cb)
    P = dense(prp, pcol, pval, int(np.prod(nc)))
    assert np.all(P[fb] == 0) and np.all(P[:, cb] == 0)
