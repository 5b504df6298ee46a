"""The oracle's dT/dlogK gradient (or_grad_logk), CPU only: with the pressure
and the adjoint state from exact dense solves, it must equal central finite
differences of the misfit J(theta) = 0.5 sum_o (p_o - p_obs_o)^2, so the
oracle that checks the GPU gradient is itself pinned to the mathematics."""
import numpy as np

from oracle import oracle as O

DIMS = (6, 8, 4)


def _dense(A):
    M = np.zeros((A.n, A.n))
    for i in range(A.n):
        s, e = A.ia[i], A.ia[i + 1]
        M[i, A.ja[s:e]] = A.a[s:e]
    return M


def _misfit(theta, obs, p_obs, with_state=False):
    from ml_prec_b200.adjoint import field_from_theta
    nx, ny, nz = DIMS
    kx, ky, kz = field_from_theta(nx, ny, nz, theta)
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, 1.0, True)
    M = _dense(A)
    p = np.linalg.solve(M, b)
    r = p[obs] - p_obs
    J = 0.5 * float(r @ r)
    if not with_state:
        return J
    g = np.zeros(A.n)
    g[obs] = r
    lam = np.linalg.solve(M.T, g)
    return J, (kx, ky, kz), p, lam


def test_oracle_gradient_matches_central_differences():
    from ml_prec_b200 import fields
    from ml_prec_b200.adjoint import field_index
    nx, ny, nz = DIMS
    idx = field_index(nx, ny, nz)
    theta = np.log(fields.field("iid", 1)[0])[idx]
    theta_true = np.log(fields.field("iid", 3)[0])[idx]
    rng = np.random.default_rng(2)
    obs = np.sort(rng.choice(theta.size, size=10, replace=False))
    p_true = _misfit(theta_true, obs, np.zeros(10), with_state=True)[2]
    p_obs = p_true[obs]
    J, (kx, ky, kz), p, lam = _misfit(theta, obs, p_obs, with_state=True)
    g = O.grad_logk(nx, ny, nz, kx, ky, kz, p, lam)
    cells = rng.choice(theta.size, size=24, replace=False)
    h = 1e-6
    fd = np.empty(cells.size)
    for t, c in enumerate(cells):
        tp = theta.copy(); tp[c] += h
        tm = theta.copy(); tm[c] -= h
        fd[t] = (_misfit(tp, obs, p_obs) - _misfit(tm, obs, p_obs)) / (2 * h)
    assert np.linalg.norm(fd - g[cells]) <= 1e-6 * np.linalg.norm(g[cells])
