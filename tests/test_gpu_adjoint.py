"""Adjoint gradients of J(u) = 1/2 ||u - u_t||^2 for the 3D Q1 Poisson problem on
64^3 cells with log-normal conductivities (u_t: the solve at an independently
seeded field), through the torch.autograd.Function over the GPU path:
  * against the FP64 CPU adjoint built from the reference's compiled CG (forward
    and transposed solves) and the restated element stiffness K_e(kappa = 1);
  * against central finite differences (relative step 1e-6) on 64 random
    elements, and on entries of b."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SEED = 0
CELLS = [64, 64, 64]


@pytest.fixture(scope="module")
def setup():
    from cie_b200.adjoint import DifferentiablePoisson
    from cie_b200.fem import kappa_field, random_uniform
    from cie_b200.linalg import CUDASpace, Statistics
    space = CUDASpace()
    problem = DifferentiablePoisson(space, 3, 1, CELLS, settings=Statistics(20000, 0.0, 1e-13))
    n, nc = problem.n, problem.mesh.ncells
    kappa = torch.as_tensor(kappa_field(SEED + 1, CELLS)).cuda()
    kappa_t = torch.as_tensor(kappa_field(SEED + 2, CELLS)).cuda()
    b = torch.as_tensor(random_uniform(SEED, n)).cuda()
    u_t = problem(kappa_t, b).detach().clone()
    return problem, kappa, b, u_t, n, nc


def objective(problem, kappa, b, u_t):
    u = problem(kappa, b)
    return 0.5 * torch.sum((u - u_t) ** 2), u


def test_adjoint_gradient_vs_cpu_fp64_adjoint(setup, reference, restatement):
    problem, kappa, b, u_t, n, nc = setup
    k = kappa.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    J, u = objective(problem, k, bb, u_t)
    J.backward()
    g_kappa, g_b = k.grad.cpu().numpy(), bb.grad.cpu().numpy()
    assert problem.adjoint_stats.relativeResidual <= 1e-13
    # CPU FP64 adjoint on the same assembled system
    m = problem.matrix
    rp, col, val = m.rowExtents.cpu().numpy(), m.columnIndices.cpu().numpy(), m.entries.cpu().numpy()
    bnd = problem.boundary.cpu().numpy().astype(bool)
    bh = np.where(bnd, 0.0, b.cpu().numpy())
    uc, _, err, _ = reference.pcg(rp, col, val, bh, maxit=20000, abstol=0.0, reltol=1e-13)
    assert err is None
    g = np.where(bnd, 0.0, uc - u_t.cpu().numpy())
    lam, _, err, _ = reference.pcg(rp, col, val, g, maxit=20000, abstol=0.0, reltol=1e-13)
    assert err is None
    mesh = problem.mesh
    Kunit = restatement.element_stiffness(3, 1, 1.0, mesh.h, 0)
    g_ref = restatement.element_gradient(nc, mesh.nb, mesh.dofmap, Kunit, np.where(bnd, 0.0, lam),
                                         np.where(bnd, 0.0, uc))
    e_k = np.linalg.norm(g_kappa - g_ref) / np.linalg.norm(g_ref)
    e_b = np.linalg.norm(g_b - lam) / np.linalg.norm(lam)
    e_u = np.linalg.norm(u.detach().cpu().numpy() - uc) / np.linalg.norm(uc)
    print("dJ/dkappa vs CPU adjoint: %.3e; dJ/db: %.3e; u: %.3e" % (e_k, e_b, e_u))
    assert e_u <= 1e-9 and e_k <= 1e-8 and e_b <= 1e-8


def test_adjoint_gradient_vs_central_differences(setup):
    problem, kappa, b, u_t, n, nc = setup
    k = kappa.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    J, _ = objective(problem, k, bb, u_t)
    J.backward()
    g_kappa, g_b = k.grad.cpu().numpy(), bb.grad.cpu().numpy()
    rng = np.random.default_rng(SEED + 3)
    cells = rng.choice(nc, size=64, replace=False)
    step = 1e-6
    fd = np.empty(len(cells))
    with torch.no_grad():
        for i, e in enumerate(cells):
            kp, km = kappa.clone(), kappa.clone()
            h = step * float(kappa[e])
            kp[e] += h
            km[e] -= h
            Jp, _ = objective(problem, kp, b, u_t)
            Jm, _ = objective(problem, km, b, u_t)
            fd[i] = (float(Jp) - float(Jm)) / (2 * h)
    ga = g_kappa[cells]
    err = np.linalg.norm(fd - ga) / np.linalg.norm(ga)
    print("dJ/dkappa vs central differences on 64 elements: %.3e (|g| max %.3e)" % (err, np.abs(ga).max()))
    assert err <= 1e-5
    # dJ/db on interior entries (boundary entries of b do not enter: gradient 0)
    bnd = problem.boundary.cpu().numpy().astype(bool)
    interior = np.flatnonzero(~bnd)
    idx = rng.choice(interior, size=8, replace=False)
    fdb = np.empty(len(idx))
    with torch.no_grad():
        for i, j in enumerate(idx):
            bp, bm = b.clone(), b.clone()
            bp[j] += 1e-6
            bm[j] -= 1e-6
            fdb[i] = (float(objective(problem, kappa, bp, u_t)[0]) - float(objective(problem, kappa, bm, u_t)[0])) / 2e-6
    errb = np.linalg.norm(fdb - g_b[idx]) / np.linalg.norm(g_b[idx])
    print("dJ/db vs central differences on 8 entries: %.3e" % errb)
    assert errb <= 1e-5
    assert np.all(g_b[bnd] == 0.0)


def test_solve_is_reused_for_the_same_kappa(setup):
    problem, kappa, b, u_t, n, nc = setup
    u1 = problem(kappa, b)
    entries = problem.matrix.entries.clone()
    u2 = problem(kappa.clone(), b)  # same values: no re-assembly, same solve
    assert torch.equal(problem.matrix.entries, entries)
    assert torch.equal(u1, u2)
