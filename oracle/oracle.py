"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes front end of the two CPU checkers built by oracle/Makefile:
  Restatement  liboracle.so          plain-C restatement of the reference algorithms
  Reference    _ref/libcieref.so     the reference's own FP64 CPU solver (compiled in place)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libcieref.so")

_P = ctypes.c_void_p
_i, _l, _d, _u16, _u64 = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_uint16, ctypes.c_uint64


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def build(reference=True):
    """Build the restatement (and the reference library when its sources exist)."""
    target = "all" if reference else "restatement"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


class Restatement:
    def __init__(self):
        if not os.path.exists(RESTATE_PATH):
            build(reference=False)
        L = ctypes.CDLL(RESTATE_PATH)
        sig = {
            "ora_spmv": (None, [_i, _P, _P, _P, _d, _P, _d, _P]),
            "ora_masked_spmv": (None, [_i, _P, _P, _P, _P, _u16, _d, _P, _d, _P]),
            "ora_diag_inverse": (_i, [_i, _P, _P, _P, _P]),
            "ora_dot": (_d, [_l, _P, _P]),
            "ora_pcg": (_i, [_i, _P, _P, _P, _P, _P, _l, _d, _d, _i, _P]),
            "ora_jacobi": (None, [_i, _P, _P, _P, _P, _l, _d, _d, _P, _d, _P]),
            "ora_chebyshev": (None, [_i, _P, _P, _P, _P, _i, _d, _d, _P, _P]),
            "ora_power_lambda_max": (_d, [_i, _P, _P, _P, _P, _i, _u64]),
            "ora_gauss_legendre": (_i, [_i, _P, _P]),
            "ora_lagrange_1d": (None, [_i, _P, _d, _P, _P]),
            "ora_stiffness_point": (None, [_i, _i, _P, _i, _P, _d, _P]),
            "ora_element_stiffness": (None, [_i, _i, _i, _P, _P, _d, _P, _i, _P]),
            "ora_structured_dofmap": (None, [_i, _i, _P, _P]),
            "ora_csr_pattern": (_l, [_l, _i, _P, _i, _P, _P]),
            "ora_assemble": (_i, [_l, _i, _P, _P, _P, _P, _P]),
            "ora_element_gradient": (None, [_l, _i, _P, _P, _P, _P, _P]),
            "ora_dirichlet_eliminate": (None, [_i, _P, _P, _P, _P, _P]),
            "ora_cut_cell_points": (_i, [_i, _i, _i, _P, _d, _P, _P, _i, _P, _P, _P, _d]),
            "ora_cut_cell_points_halfspace": (_i, [_i, _i, _i, _P, _d, _P, _P, _i, _P, _P, _P, _d]),
            "ora_cuthill_mckee": (_i, [_i, _P, _P, _i, _P]),
            "ora_dirichlet_penalty": (_i, [_i, _i, _i, _P, _P, _d, _i, _P, _P, _P, _P, _P, _P]),
            "ora_random_uniform": (None, [_u64, _l, _P]),
            "ora_random_normal": (None, [_u64, _l, _P]),
            "ora_kappa_field": (None, [_u64, _i, _P, _d, _i, _P]),
            "ora_structured_boundary": (None, [_i, _i, _P, _P]),
            "ora_assemble_structured": (_i, [_i, _i, _i, _P, _P, _P, _P, _P, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L

    # -- linalg --
    def spmv(self, rowptr, col, val, inScale, x, outScale, y):
        y = np.array(y, dtype=np.float64, copy=True)
        self.L.ora_spmv(len(rowptr) - 1, p(rowptr), p(col), p(val), inScale, p(x), outScale, p(y))
        return y

    def masked_spmv(self, rowptr, col, val, mask, threshold, inScale, x, outScale, y):
        y = np.array(y, dtype=np.float64, copy=True)
        mask = np.ascontiguousarray(mask, dtype=np.uint16)
        self.L.ora_masked_spmv(len(rowptr) - 1, p(rowptr), p(col), p(val), p(mask), threshold, inScale, p(x),
                               outScale, p(y))
        return y

    def diag_inverse(self, rowptr, col, val):
        out = np.zeros(len(rowptr) - 1)
        bad = self.L.ora_diag_inverse(len(rowptr) - 1, p(rowptr), p(col), p(val), p(out))
        return out, bad

    def pcg(self, rowptr, col, val, b, x0=None, maxit=5000, abstol=0.0, reltol=1e-10, precondition=True):
        n = len(rowptr) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        stats = np.zeros(3)
        st = self.L.ora_pcg(n, p(rowptr), p(col), p(val), p(b), p(x), maxit, abstol, reltol, int(precondition),
                            p(stats))
        return x, stats, st

    def jacobi(self, rowptr, col, val, dinv, iterations, relaxation, inScale, x, outScale, y):
        y = np.array(y, dtype=np.float64, copy=True)
        self.L.ora_jacobi(len(rowptr) - 1, p(rowptr), p(col), p(val), p(dinv), iterations, relaxation, inScale, p(x),
                          outScale, p(y))
        return y

    def chebyshev(self, rowptr, col, val, dinv, degree, lmin, lmax, x):
        y = np.zeros(len(rowptr) - 1)
        self.L.ora_chebyshev(len(rowptr) - 1, p(rowptr), p(col), p(val), p(dinv), degree, lmin, lmax, p(x), p(y))
        return y

    def power_lambda_max(self, rowptr, col, val, dinv, iterations, seed):
        return self.L.ora_power_lambda_max(len(rowptr) - 1, p(rowptr), p(col), p(val), p(dinv), iterations, seed)

    # -- fem --
    def gauss_legendre(self, order):
        n, w = np.zeros(order), np.zeros(order)
        st = self.L.ora_gauss_legendre(order, p(n), p(w))
        assert st == 0
        return n, w

    def stiffness_point(self, dim, coefficients, point, modulus):
        coefficients = np.ascontiguousarray(coefficients, dtype=np.float64)
        setSize, deg1 = coefficients.shape
        out = np.zeros((setSize ** dim) ** 2)
        self.L.ora_stiffness_point(dim, setSize, p(coefficients), deg1 - 1, p(np.asarray(point, dtype=np.float64)),
                                   modulus, p(out))
        return out

    def tensor_gauss(self, dim, order):
        """Tensor Gauss points, first 1-D index fastest (OuterProduct_impl.hpp:27-45)."""
        n, w = self.gauss_legendre(order)
        q = np.arange(order ** dim)
        idx = (q[:, None] // order ** np.arange(dim)[None, :]) % order
        return np.ascontiguousarray(n[idx]), np.ascontiguousarray(np.prod(w[idx], axis=1))

    def element_stiffness(self, dim, order, kappa, h, convention=0, points=None, weights=None):
        if points is None:
            points, weights = self.tensor_gauss(dim, order + 1)
        nb = (order + 1) ** dim
        K = np.zeros(nb * nb)
        self.L.ora_element_stiffness(dim, order, len(weights), p(points), p(weights), kappa,
                                     p(np.asarray(h, dtype=np.float64)), convention, p(K))
        return K

    def structured_dofmap(self, dim, order, cells):
        cells = np.asarray(cells, dtype=np.int32)
        nb = (order + 1) ** dim
        out = np.zeros(int(np.prod(cells)) * nb, dtype=np.int32)
        self.L.ora_structured_dofmap(dim, order, p(cells), p(out))
        return out

    def csr_pattern(self, ncells, nb, dofmap, ndofs):
        rowptr = np.zeros(ndofs + 1, dtype=np.int32)
        nnz = self.L.ora_csr_pattern(ncells, nb, p(dofmap), ndofs, p(rowptr), None)
        col = np.zeros(nnz, dtype=np.int32)
        self.L.ora_csr_pattern(ncells, nb, p(dofmap), ndofs, p(rowptr), p(col))
        return rowptr, col

    def assemble(self, ncells, nb, dofmap, Ke, rowptr, col, val=None):
        val = np.zeros(len(col)) if val is None else np.array(val, dtype=np.float64, copy=True)
        st = self.L.ora_assemble(ncells, nb, p(dofmap), p(np.ascontiguousarray(Ke, dtype=np.float64)), p(rowptr),
                                 p(col), p(val))
        return val, st

    def element_gradient(self, ncells, nb, dofmap, Kunit, lam, u):
        g = np.zeros(ncells)
        self.L.ora_element_gradient(ncells, nb, p(dofmap), p(np.ascontiguousarray(Kunit)), p(lam), p(u), p(g))
        return g

    def dirichlet(self, rowptr, col, val, isBoundary, rhs=None):
        val = np.array(val, dtype=np.float64, copy=True)
        rhs = None if rhs is None else np.array(rhs, dtype=np.float64, copy=True)
        self.L.ora_dirichlet_eliminate(len(rowptr) - 1, p(rowptr), p(col), p(val),
                                       p(np.ascontiguousarray(isBoundary, dtype=np.uint8)), p(rhs))
        return val, rhs

    def cut_cell_points(self, dim, depth, order, center, radius, origin, size, alpha, maxPoints=1 << 16):
        pts = np.zeros(maxPoints * dim)
        w = np.zeros(maxPoints)
        s = np.zeros(maxPoints)
        n = self.L.ora_cut_cell_points(dim, depth, order, p(np.asarray(center, dtype=np.float64)), radius,
                                       p(np.asarray(origin, dtype=np.float64)), p(np.asarray(size, dtype=np.float64)),
                                       maxPoints, p(pts), p(w), p(s), alpha)
        assert n >= 0
        return pts[: n * dim].reshape(n, dim), w[:n], s[:n]

    def cut_cell_points_halfspace(self, dim, depth, order, normal, offset, origin, size, alpha,
                                  maxPoints=1 << 16):
        pts = np.zeros(maxPoints * dim)
        w = np.zeros(maxPoints)
        s = np.zeros(maxPoints)
        n = self.L.ora_cut_cell_points_halfspace(dim, depth, order, p(np.asarray(normal, dtype=np.float64)),
                                                 float(offset), p(np.asarray(origin, dtype=np.float64)),
                                                 p(np.asarray(size, dtype=np.float64)), maxPoints, p(pts), p(w),
                                                 p(s), alpha)
        assert n >= 0
        return pts[: n * dim].reshape(n, dim), w[:n], s[:n]

    def dirichlet_penalty(self, dim, order, cells, penalty, rowptr, col, val, faceMask=0, g=None, rhs=None,
                          quadratureOrder=None):
        """Penalty Dirichlet terms added to copies of val (and rhs when g is given)."""
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        h = 1.0 / cells.astype(np.float64)
        dofmap = self.structured_dofmap(dim, order, cells)
        val = np.array(val, dtype=np.float64, copy=True)
        rhs = None if rhs is None else np.array(rhs, dtype=np.float64, copy=True)
        g = None if g is None else np.ascontiguousarray(g, dtype=np.float64)
        st = self.L.ora_dirichlet_penalty(dim, order, order + 1 if quadratureOrder is None else quadratureOrder,
                                          p(cells), p(h), float(penalty), int(faceMask), p(g), p(dofmap), p(rowptr),
                                          p(col), p(val), p(rhs))
        assert st == 0
        return val, rhs

    # -- graph --
    def cuthill_mckee(self, rowptr, col, strategy=1):
        """(map, largest batch queued at once)."""
        n = len(rowptr) - 1
        out = np.zeros(n, dtype=np.int32)
        largest = self.L.ora_cuthill_mckee(n, p(rowptr), p(col), int(strategy), p(out))
        assert largest >= 0
        return out, largest

    # -- seeded workload inputs --
    def random_uniform(self, seed, n):
        out = np.zeros(int(n))
        self.L.ora_random_uniform(int(seed), int(n), p(out))
        return out

    def random_normal(self, seed, n):
        out = np.zeros(int(n))
        self.L.ora_random_normal(int(seed), int(n), p(out))
        return out

    def kappa_field(self, seed, cells, sigma=1.0, truncation=3):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        out = np.zeros(int(np.prod(cells)))
        self.L.ora_kappa_field(int(seed), len(cells), p(cells), float(sigma), int(truncation), p(out))
        return out

    def structured_boundary(self, dim, order, cells):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        n = int(np.prod(order * cells + 1))
        out = np.zeros(n, dtype=np.uint8)
        self.L.ora_structured_boundary(dim, order, p(cells), p(out))
        return out

    def poisson_system(self, dim, order, cells, seed=0, kappa="lognormal", kappa_seed=None):
        """The seeded Poisson system of the workloads, built on the host without the
        CUDA library: structured Q_order grid of the unit box, CSR pattern, element
        stiffness scattered in the GPU's colour and summation order (reference
        convention), symmetric Dirichlet elimination, RHS uniform [-1, 1] (seed),
        kappa = 1 or the smoothed log-normal field (seed + 1 unless kappa_seed).
        Returns (rowptr, col, val, rhs, isBoundary, kappa)."""
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        assert len(cells) == dim
        dofmap = self.structured_dofmap(dim, order, cells)
        ndofs = int(np.prod(order * cells.astype(np.int64) + 1))
        nb = (order + 1) ** dim
        rowptr, col = self.csr_pattern(int(np.prod(cells)), nb, dofmap, ndofs)
        if isinstance(kappa, str) and kappa == "lognormal":
            k = self.kappa_field(seed + 1 if kappa_seed is None else kappa_seed, cells)
        elif isinstance(kappa, str) and kappa == "one":
            k = np.ones(int(np.prod(cells)))
        else:
            k = np.ascontiguousarray(kappa, dtype=np.float64)
        val = np.zeros(len(col))
        st = self.L.ora_assemble_structured(dim, order, order + 1, p(cells), p(dofmap), p(k), p(rowptr), p(col),
                                            p(val))
        assert st == 0, "element entry missing from the pattern"
        rhs = self.random_uniform(seed, ndofs)
        bnd = self.structured_boundary(dim, order, cells)
        self.L.ora_dirichlet_eliminate(ndofs, p(rowptr), p(col), p(val), p(bnd), p(rhs))
        return rowptr, col, val, rhs, bnd, k


def system_digest(rowptr, col, val, rhs):
    """SHA-256 (first 16 hex digits) over the bytes of a CSR system and its RHS."""
    import hashlib
    h = hashlib.sha256()
    for a, t in ((rowptr, np.int32), (col, np.int32), (val, np.float64), (rhs, np.float64)):
        h.update(np.ascontiguousarray(a, dtype=t).tobytes())
    return h.hexdigest()[:16]


class Reference:
    """The reference's compiled CPU solver (oracle/_ref/libcieref.so)."""

    def __init__(self, threads=None):
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError("oracle/_ref/libcieref.so is not built (needs the reference sources)")
        L = ctypes.CDLL(REF_PATH)
        sig = {
            "cieref_last_error": (_i, [ctypes.c_char_p, _i]),
            "cieref_max_threads": (_i, []),
            "cieref_pool_create": (_P, [_i]),
            "cieref_pool_destroy": (None, [_P]),
            "cieref_spmv": (_i, [_P, _i, _i, _P, _P, _P, _d, _P, _d, _P]),
            "cieref_masked_spmv": (_i, [_P, _i, _i, _P, _P, _P, _P, _u16, _d, _P, _d, _P]),
            "cieref_diag_inverse": (_i, [_i, _P, _P, _P, _P]),
            "cieref_pcg": (_i, [_P, _i, _P, _P, _P, _P, _P, _l, _d, _d, _i, _i, _P, _P]),
            "cieref_jacobi": (_i, [_P, _i, _P, _P, _P, _l, _d, _d, _P, _d, _P]),
            "cieref_pmg": (_i, [_P, _i, _P, _P, _P, _P, _i, _P, _P, _d, _l, _P, _P]),
            "cieref_space_dot": (_i, [_P, _l, _P, _P, _P]),
            "cieref_space_op": (_i, [_P, _i, _l, _P, _P, _d]),
            "cieref_gauss_legendre": (_i, [_i, _P, _P]),
            "cieref_lagrange": (_i, [_i, _P, _i, _i, _P, _P, _P, _P]),
            "cieref_make_reordering": (_i, [_i, _P, _P, _P, _i, _P]),
            "cieref_reorder": (_i, [_i, _P, _P, _P, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L
        self.threads = int(threads) if threads else int(L.cieref_max_threads())
        self.pool = L.cieref_pool_create(self.threads) if self.threads > 1 else None

    def close(self):
        if self.pool:
            self.L.cieref_pool_destroy(self.pool)
            self.pool = None

    def _err(self):
        b = ctypes.create_string_buffer(2048)
        self.L.cieref_last_error(b, 2048)
        return b.value.decode()

    def _check(self, st):
        if st:
            raise RuntimeError("reference: " + self._err())

    def spmv(self, rowptr, col, val, inScale, x, outScale, y, ncols=None):
        y = np.array(y, dtype=np.float64, copy=True)
        n = len(rowptr) - 1
        self._check(self.L.cieref_spmv(self.pool, n, ncols if ncols is not None else len(x), p(rowptr), p(col),
                                       p(val), inScale, p(x), outScale, p(y)))
        return y

    def masked_spmv(self, rowptr, col, val, mask, threshold, inScale, x, outScale, y):
        y = np.array(y, dtype=np.float64, copy=True)
        mask = np.ascontiguousarray(mask, dtype=np.uint16)
        self._check(self.L.cieref_masked_spmv(self.pool, len(rowptr) - 1, len(x), p(rowptr), p(col), p(val),
                                              p(mask), threshold, inScale, p(x), outScale, p(y)))
        return y

    def diag_inverse(self, rowptr, col, val):
        out = np.zeros(len(rowptr) - 1)
        st = self.L.cieref_diag_inverse(len(rowptr) - 1, p(rowptr), p(col), p(val), p(out))
        return out, (self._err() if st else None)

    def pcg(self, rowptr, col, val, b, x0=None, maxit=5000, abstol=0.0, reltol=1e-10, precondition=True):
        n = len(rowptr) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        stats = np.zeros(3)
        secs = ctypes.c_double()
        st = self.L.cieref_pcg(self.pool, n, p(rowptr), p(col), p(val), p(b), p(x), maxit, abstol, reltol,
                               int(precondition), 0, p(stats), ctypes.byref(secs))
        return x, stats, (self._err() if st else None), secs.value

    def jacobi(self, rowptr, col, val, iterations, relaxation, inScale, x, outScale, y):
        y = np.array(y, dtype=np.float64, copy=True)
        self._check(self.L.cieref_jacobi(self.pool, len(rowptr) - 1, p(rowptr), p(col), p(val), iterations,
                                         relaxation, inScale, p(x), outScale, p(y)))
        return y

    def pmg(self, rowptr, col, val, mask, order, b, tol=1e-6, maxCycles=200):
        n = len(rowptr) - 1
        x = np.zeros(n)
        cycles = ctypes.c_long()
        rel = ctypes.c_double()
        self._check(self.L.cieref_pmg(self.pool, n, p(rowptr), p(col), p(val),
                                      p(np.ascontiguousarray(mask, dtype=np.uint16)), order, p(b), p(x), tol,
                                      maxCycles, ctypes.byref(cycles), ctypes.byref(rel)))
        return x, cycles.value, rel.value

    def dot(self, a, b):
        out = ctypes.c_double()
        self._check(self.L.cieref_space_dot(self.pool, len(a), p(a), p(b), ctypes.byref(out)))
        return out.value

    def space_op(self, op, target, source, alpha):
        t = np.array(target, dtype=np.float64, copy=True)
        self._check(self.L.cieref_space_op(self.pool, op, len(t), p(t), p(source), alpha))
        return t

    def gauss_legendre(self, order):
        n, w = np.zeros(order), np.zeros(order)
        self._check(self.L.cieref_gauss_legendre(order, p(n), p(w)))
        return n, w

    def make_reordering(self, rowptr, col, val, strategy):
        """makeReordering (serial): map[new row] = old row; strategy 1 CM, 2 RCM."""
        n = len(rowptr) - 1
        out = np.zeros(n, dtype=np.int32)
        self._check(self.L.cieref_make_reordering(n, p(rowptr), p(col), p(np.ascontiguousarray(val, np.float64)),
                                                  int(strategy), p(out)))
        return out

    def reorder(self, mapping, rowptr, col, val):
        """reorder<int,double,false> on copies: the permuted (rowptr, col, val)."""
        rp, c, v = (np.array(a, copy=True) for a in (rowptr, col, val))
        self._check(self.L.cieref_reorder(len(rp) - 1, p(np.ascontiguousarray(mapping, np.int32)), p(rp), p(c), p(v)))
        return rp, c, v

    # The reference's stream writer crashes (SIGSEGV in the C++ stream's number
    # formatting) in a process that has imported numpy, whose bundled runtime
    # libraries it then shares; so it runs in a child interpreter that loads only
    # ctypes and the reference library, on arrays passed through a file.
    _MM_CHILD = """
import array, ctypes, sys
lib = ctypes.CDLL(sys.argv[1])
kind, src, dst = sys.argv[2], sys.argv[3], sys.argv[4].encode()
with open(src, "rb") as f:
    head = array.array("q"); head.fromfile(f, 3)
    ints = array.array("i"); vals = array.array("d")
    if kind == "csr":
        ints.fromfile(f, head[0] + 1 + head[2])
    vals.fromfile(f, head[2])
ip = (ctypes.c_int * max(len(ints), 1)).from_buffer(ints) if len(ints) else None
vp = (ctypes.c_double * max(len(vals), 1)).from_buffer(vals) if len(vals) else None
P = ctypes.c_void_p
if kind == "csr":
    base = ctypes.addressof(ip)
    st = lib.cieref_matrix_market(ctypes.c_char_p(dst), ctypes.c_int(head[0]), ctypes.c_int(head[1]), P(base),
                                  P(base + 4 * (head[0] + 1)), P(ctypes.addressof(vp) if vp else 0))
else:
    st = lib.cieref_matrix_market_vector(ctypes.c_char_p(dst), ctypes.c_long(head[2]),
                                         P(ctypes.addressof(vp) if vp else 0))
sys.exit(st)
"""

    def _matrix_market_child(self, kind, path, head, ints, vals):
        import sys
        import tempfile
        with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
            np.asarray(head, dtype=np.int64).tofile(f)
            if ints is not None:
                np.ascontiguousarray(ints, dtype=np.int32).tofile(f)
            np.ascontiguousarray(vals, dtype=np.float64).tofile(f)
            name = f.name
        try:
            subprocess.run([sys.executable, "-c", self._MM_CHILD, REF_PATH, kind, name, str(path)], check=True)
        finally:
            os.unlink(name)

    def matrix_market(self, path, rowptr, col, val, columns=None):
        """cie::io::MatrixMarket::Output for a CSR matrix, written to `path`."""
        n = len(rowptr) - 1
        ints = np.concatenate([np.asarray(rowptr, np.int32), np.asarray(col, np.int32)])
        self._matrix_market_child("csr", path, [n, n if columns is None else columns, len(col)], ints, val)

    def matrix_market_vector(self, path, values):
        self._matrix_market_child("vector", path, [0, 0, len(values)], None, values)

    def lagrange(self, nodes, iBase, points):
        """The reference's LagrangePolynomial of node iBase: (ascending coefficients,
        values at points, derivative values at points)."""
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        points = np.ascontiguousarray(points, dtype=np.float64)
        c, v, d = np.zeros(len(nodes)), np.zeros(len(points)), np.zeros(len(points))
        self._check(self.L.cieref_lagrange(len(nodes), p(nodes), int(iBase), len(points), p(points), p(c), p(v),
                                           p(d)))
        return c, v, d


def reference_available():
    return os.path.exists(REF_PATH)
