"""Differentiation form: adjoint gradient of the pressure misfit with respect to
per-cell log-permeability, against the CPU FP64 oracle gradient and against
central finite differences (step 1e-6). Bar: relative error <= 1e-5."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (12, 22, 6)
TOL = 1e-5


@pytest.fixture(scope="module")
def problem():
    from ml_prec_b200 import adjoint
    prob, theta = adjoint.make_problem(*DIMS, eps=1e-12, fp32=True)
    J, g, lam, p = prob.gradient(theta)
    return prob, theta, J, g, lam, p


def test_gradient_matches_cpu_fp64_oracle(problem):
    from ml_prec_b200 import adjoint
    from oracle import oracle as O
    prob, theta, J, g, lam, p = problem
    nx, ny, nz = DIMS
    kx, ky, kz = adjoint.field_from_theta(nx, ny, nz, theta)
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, 1.0, True)
    P = O.Prec(A, "msplit")
    po, it, rel, rc = O.pcg(A, b, P, 1e-12, maxit=5000, x0_zero=True)
    assert rc == 0
    r = po[prob.obs] - prob.p_obs
    go = np.zeros(A.n)
    go[prob.obs] = r
    lo, it, rel, rc = O.pcg(A, go, P, 1e-12, maxit=5000, x0_zero=True)
    assert rc in (0, -3)
    gref = O.grad_logk(nx, ny, nz, kx, ky, kz, po, lo)
    assert abs(J - 0.5 * np.sum(r ** 2)) <= TOL * J
    assert np.linalg.norm(g - gref) <= TOL * np.linalg.norm(gref)


def test_gradient_matches_central_differences(problem):
    prob, theta, J, g, lam, p = problem
    rng = np.random.default_rng(7)
    # 64 random cells, drawn with probability proportional to |g| so that the
    # sample is not dominated by cells whose sensitivity is below rounding
    w = np.abs(g) / np.abs(g).sum()
    cells = rng.choice(len(g), size=64, replace=False, p=w)
    h = 1e-6
    fd = np.empty(len(cells))
    for t, c in enumerate(cells):
        tp = theta.copy(); tp[c] += h
        tm = theta.copy(); tm[c] -= h
        fd[t] = (prob.objective(tp)[0] - prob.objective(tm)[0]) / (2 * h)
    assert np.linalg.norm(fd - g[cells]) <= TOL * np.linalg.norm(g[cells])


def test_autograd_binding(problem):
    import torch
    from ml_prec_b200 import adjoint
    prob, theta, J, g, lam, p = problem
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    Jt = adjoint.pressure_misfit(th, prob)
    Jt.backward()
    assert abs(Jt.item() - J) <= 1e-12 * J
    assert np.allclose(th.grad.numpy(), g, rtol=1e-10, atol=1e-14 * np.abs(g).max())


def test_full_size_gradient_against_oracle_and_central_differences():
    """60x220x85 (1,122,000 cells): the adjoint gradient over all cells
    against the oracle's FP64 gradient (forward and adjoint solves at 1e-12,
    capped at 300 iterations: the FP64 iteration stagnates near there), and
    central differences (step 1e-6) on 64 uniformly drawn cells and on the 16
    cells of largest sensitivity. With 25 observation cells in a heterogeneous
    field, 99 % of the cells have |dJ/dlnK| below 1e-22 (on this problem the
    uniform draw finds none above 1e-28, against max |g| = 4.3e-9), where an
    error relative to the cell's own value is meaningless; the uniform sample
    is held to 1e-5 of max |g| per cell, the 16 largest to 1e-5 normwise."""
    from ml_prec_b200 import adjoint
    from oracle import oracle as O
    dims = (60, 220, 85)
    prob, theta = adjoint.make_problem(*dims, eps=1e-12, fp32=True)
    J, g, lam, p = prob.gradient(theta)
    kx, ky, kz = adjoint.field_from_theta(*dims, theta)
    A, b = O.assemble(*dims, kx, ky, kz, 1.0, True)
    P = O.Prec(A, "msplit")
    po, _, _, rc = O.pcg(A, b, P, 1e-12, maxit=300, x0_zero=True)
    assert rc in (0, -3)
    r = po[prob.obs] - prob.p_obs
    go = np.zeros(A.n)
    go[prob.obs] = r
    lo, _, _, rc = O.pcg(A, go, P, 1e-12, maxit=300, x0_zero=True)
    assert rc in (0, -3)
    gref = O.grad_logk(*dims, kx, ky, kz, po, lo)
    assert abs(J - 0.5 * np.sum(r ** 2)) <= TOL * J
    assert np.linalg.norm(g - gref) <= TOL * np.linalg.norm(gref)
    rng = np.random.default_rng(11)
    uniform = rng.choice(len(g), size=64, replace=False)
    top = np.argsort(-np.abs(g))[:16]
    h = 1e-6

    def fd(cells):
        out = np.empty(len(cells))
        for t, c in enumerate(cells):
            tp = theta.copy(); tp[c] += h
            tm = theta.copy(); tm[c] -= h
            out[t] = (prob.objective(tp)[0] - prob.objective(tm)[0]) / (2 * h)
        return out

    scale = np.abs(g).max()
    assert np.abs(fd(uniform) - g[uniform]).max() <= TOL * scale
    ft = fd(top)
    assert np.linalg.norm(ft - g[top]) <= TOL * np.linalg.norm(g[top])
