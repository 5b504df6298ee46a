"""Differentiation form: gradient of a pressure misfit with respect to the
per-cell log-permeability, by the adjoint method, with an optional
torch.autograd binding.

    J(theta) = 0.5 * sum_{o in obs} (p_o - p_obs_o)^2,   A(theta) p = b(theta),
    K = exp(theta) per mesh cell, kx = ky = K, kz = 0.1 K.

forward: assemble A(theta) on the GPU, build the (FP32-stored) multi-split
hierarchy, solve A p = b with flexible FP64 PCG. gradient: one more PCG solve
with the same matrix and hierarchy (A is symmetric, so the adjoint system is
A lambda = dJ/dp), then the fused dT/dlogK kernel (mlp_matrix_grad_logk).
The reference has no gradients; this form is this project's addition.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api
from ._capi import Stats, check, lib
from .fields import KN, KNX, KNY

MSPLIT = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="simple_1")


def field_index(nx, ny, nz):
    """SPE10 field entry of every mesh cell (SPEMesh::index_k, mesh.h:57-59)."""
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return ((k * KNY * KNX + j * KNX + i) % KN).reshape(-1)


def field_from_theta(nx, ny, nz, theta, base=None):
    """kx, ky, kz field blocks with K = exp(theta) on the mesh's cells."""
    idx = field_index(nx, ny, nz)
    K = np.ones(KN) if base is None else np.array(base, dtype=np.float64, copy=True)
    K[idx] = np.exp(np.asarray(theta, np.float64))
    return K, K.copy(), 0.1 * K


class MisfitProblem:
    """Pressure-misfit objective on an nx x ny x nz mesh (GPU forward/adjoint).

    x0_zero starts both solves from zero (the forward residual tolerance is then
    relative to ||b||); the adjoint always starts from zero."""

    def __init__(self, nx, ny, nz, obs, p_obs, c=1.0, eps=1e-12, fp32=True, prec_kw=None, x0_zero=True):
        self.dims = (nx, ny, nz)
        self.obs = np.asarray(obs, np.int64)
        self.p_obs = np.asarray(p_obs, np.float64)
        self.c = c
        self.eps = eps
        self.fp32 = fp32
        self.prec_kw = dict(MSPLIT if prec_kw is None else prec_kw)
        self.x0_mode = 1 if x0_zero else 0
        self.stats = {}

    def solve(self, theta):
        """(A, P, p_dev, b) for the field exp(theta); p on the device."""
        import torch
        kx, ky, kz = field_from_theta(*self.dims, theta)
        A, b = api.CSRMatrix.spe(*self.dims, kx, ky, kz, c=self.c, dirichlet=True)
        P = api.MultiSplitPrec(A, fp32=self.fp32, **self.prec_kw)
        b_d = torch.from_numpy(b).cuda()
        p_d = torch.empty_like(b_d)
        st = Stats()
        check(lib().mlp_pcg_device_x0(A.h, C.c_void_p(b_d.data_ptr()), P.h, C.c_void_p(p_d.data_ptr()), self.eps,
                                      0, int(self.fp32), self.x0_mode, C.byref(st), None))
        self.stats["forward"] = dict(niter=st.niter, t_solve_ms=st.t_solve_ms, t_setup_ms=st.t_setup_ms)
        return A, P, p_d, b

    def objective(self, theta):
        A, P, p_d, _ = self.solve(theta)
        p = p_d.cpu().numpy()
        return 0.5 * float(np.sum((p[self.obs] - self.p_obs) ** 2)), p

    def gradient(self, theta):
        """(J, dJ/dtheta, lambda, p) by one forward and one adjoint solve."""
        import torch
        A, P, p_d, _ = self.solve(theta)
        p = p_d.cpu().numpy()
        r = p[self.obs] - self.p_obs
        J = 0.5 * float(np.sum(r ** 2))
        g = np.zeros(A.n)
        np.add.at(g, self.obs, r)
        g_d = torch.from_numpy(g).cuda()
        lam = torch.empty_like(g_d)
        st = Stats()
        rc = lib().mlp_pcg_device_x0(A.h, C.c_void_p(g_d.data_ptr()), P.h, C.c_void_p(lam.data_ptr()), self.eps,
                                     0, int(self.fp32), 1, C.byref(st), None)
        if rc not in (0, 6):  # a tolerance below the rounding floor ends at the cap
            check(rc)
        self.stats["adjoint"] = dict(niter=st.niter, t_solve_ms=st.t_solve_ms)
        grad = torch.empty_like(g_d)
        check(lib().mlp_matrix_grad_logk(A.h, C.c_void_p(p_d.data_ptr()), C.c_void_p(lam.data_ptr()),
                                         C.c_void_p(grad.data_ptr()), None))
        return J, grad.cpu().numpy(), lam.cpu().numpy(), p


def _autograd_fn():
    import torch

    class PressureMisfit(torch.autograd.Function):
        """J = PressureMisfit.apply(theta, problem): theta a float64 tensor of
        per-cell log-permeabilities; backward returns dJ/dtheta."""

        @staticmethod
        def forward(ctx, theta, problem):
            th = theta.detach().cpu().numpy().astype(np.float64)
            J, g, _, _ = problem.gradient(th)
            ctx.save_for_backward(torch.from_numpy(g).to(theta.device, theta.dtype))
            return theta.new_tensor(J)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout * g, None

    return PressureMisfit


_PM = None


def pressure_misfit(theta, problem):
    """torch.autograd entry point: differentiable J(theta)."""
    global _PM
    if _PM is None:
        _PM = _autograd_fn()
    return _PM.apply(theta, problem)


def make_problem(nx, ny, nz, seed_field=1, seed_obs=2, seed_truth=3, nobs=25, c=1.0, **kw):
    """A misfit problem: nobs seeded observation cells, p_obs from the forward
    solve of a second seeded i.i.d. field; returns (problem, theta0)."""
    from . import fields
    rng = np.random.default_rng(seed_obs)
    N = nx * ny * nz
    obs = np.sort(rng.choice(N, size=nobs, replace=False))
    idx = field_index(nx, ny, nz)
    theta_true = np.log(fields.field("iid", seed_truth)[0])[idx]
    prob = MisfitProblem(nx, ny, nz, obs, np.zeros(nobs), c=c, **kw)
    _, p_true = prob.objective(theta_true)
    prob.p_obs = p_true[obs]
    theta0 = np.log(fields.field("iid", seed_field)[0])[idx]
    return prob, theta0
