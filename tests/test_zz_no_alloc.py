"""The allocation-free Jacobi entry point (ciecu_jacobi_f64_static, scratch in a
static device array) against the allocating ciecu_jacobi_f64 with caller-provided
scratch, both called through the C-ABI on the same matrix and inputs.  Each case
makes two calls in a row with different inputs: the second call finds the first
call's iterates in the shared static array and must not depend on them.  Runs
alone in a fresh process as well as after the other tests."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL = ATOL = 1e-13  # the Jacobi parity tolerance of the other GPU tests


def _problem(dim, cells, seed):
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CUDASpace, CSROperator, makeDiagonalOperator
    space = CUDASpace()
    prob = make_poisson(space, dim, 1, cells, seed=seed)
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    return space, A, D.inverseDiagonal, prob.rhs.numel()


def _jacobi(space, A, dinv, mask, thr, iterations, relaxation, si, x, so, y0, static):
    from cie_b200._lib import call
    from cie_b200.linalg import _ptr
    out = y0.clone()
    space.enter()
    if static:
        call("ciecu_jacobi_f64_static", A.csr.handle, _ptr(dinv), _ptr(mask), thr, iterations, relaxation,
             float(si), _ptr(x), float(so), _ptr(out))
    else:
        work = torch.empty(2 * x.numel(), dtype=torch.float64, device="cuda")
        call("ciecu_jacobi_f64", A.csr.handle, _ptr(dinv), _ptr(mask), thr, iterations, relaxation, float(si),
             _ptr(x), float(so), _ptr(out), _ptr(work))
    space.leave()
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("dim,cells,masked", [(2, [90, 90], False), (3, [40, 40, 40], False),
                                              (3, [30, 30, 30], True)])
def test_static_jacobi_matches_allocating_jacobi(dim, cells, masked):
    space, A, dinv, n = _problem(dim, cells, seed=11)
    g = torch.Generator(device="cpu").manual_seed(5)
    mask = torch.randint(1, 5, (n,), generator=g, dtype=torch.int32).to(torch.uint16).cuda() if masked else None
    thr = 4 if masked else 0
    calls = [(5, 2.0 / 3.0, 0.0, 1.0), (3, 0.8, 1.0, -0.5)]  # (sweeps, relaxation, inScale, outScale)
    for iterations, relaxation, si, so in calls:
        x = (torch.rand(n, generator=g, dtype=torch.float64) * 2 - 1).cuda()
        y0 = (torch.rand(n, generator=g, dtype=torch.float64) * 2 - 1).cuda()
        got = _jacobi(space, A, dinv, mask, thr, iterations, relaxation, si, x, so, y0, static=True)
        want = _jacobi(space, A, dinv, mask, thr, iterations, relaxation, si, x, so, y0, static=False)
        assert np.allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=RTOL, atol=ATOL)
        assert torch.count_nonzero(got - y0).item() > 0


def test_static_jacobi_rejects_matrices_beyond_its_scratch():
    from cie_b200._lib import CiecuError
    space, A, dinv, n = _problem(3, [64, 64, 64], seed=12)  # 65^3 = 274625 rows > 262144
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    with pytest.raises(CiecuError, match="exceed the static scratch of 262144 rows"):
        _jacobi(space, A, dinv, None, 0, 2, 1.0, 0.0, x, 1.0, torch.zeros_like(x), static=True)
