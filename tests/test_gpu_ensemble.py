"""Batching form: an ensemble of realizations on uneven meshes solved as
parallel branches of one graph launch must give, member by member, what the
single-instance solve gives."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spmv(A, x):
    ia, ja, a = A.arrays()
    rows = np.repeat(np.arange(A.n), np.diff(ia))
    return np.bincount(rows, weights=a * x[ja], minlength=A.n)


def test_ensemble_matches_single_solves():
    from ml_prec_b200 import ensemble
    from ml_prec_b200._capi import Stats, check, lib
    dims = [(7, 11, 5), (12, 22, 6), (30, 17, 4), (9, 40, 3), (16, 22, 8), (5, 5, 30)]
    E = ensemble.Ensemble(dims, fp32=True)
    ms, its = E.forward(eps=1e-8)
    xs = [x.cpu().numpy().copy() for x in E.x]
    for i in range(len(dims)):
        st = Stats()
        check(lib().mlp_pcg_device(E.A[i].h, C.c_void_p(E.b[i].data_ptr()), E.P[i].h,
                                   C.c_void_p(E.x[i].data_ptr()), 1e-8, 0, 1, C.byref(st), None))
        assert st.niter == its[i]
        assert np.array_equal(E.x[i].cpu().numpy(), xs[i])
    # adjoint launch: zero start, misfit right-hand side
    p_obs = [np.zeros(len(o)) for o in E.obs]
    E.adjoint(p_obs, eps=1e-8)
    for i in range(len(dims)):
        g = E.g[i].cpu().numpy()
        r = g - _spmv(E.A[i], E.lam[i].cpu().numpy())
        assert np.linalg.norm(r) <= 1e-7 * np.linalg.norm(g)
    E.close()


def test_gradient_in_one_launch_matches_single_solves_and_oracle():
    """One graph launch runs every member's forward solve, misfit gradient,
    adjoint solve and dJ/dlnK kernel. Member by member it equals the same
    steps done one call at a time through the single-instance entry points
    (zero starts, same handle: bit for bit), and the oracle's FP64 gradient
    within 1e-5."""
    import torch
    from ml_prec_b200 import ensemble, fields
    from ml_prec_b200._capi import Stats, check, lib
    from oracle import oracle as O
    dims = [(7, 11, 5), (12, 22, 6), (16, 22, 8)]
    E = ensemble.Ensemble(dims, fp32=True)
    rng = np.random.default_rng(3)
    p_obs = [rng.standard_normal(len(o)) * 0.1 + 0.5 for o in E.obs]
    ms, itf, ita = E.gradient(p_obs, eps=1e-10)
    assert ms > 0 and min(itf) > 0 and min(ita) > 0
    for i, d in enumerate(dims):
        b = E.b[i]
        p = torch.empty_like(b)
        st = Stats()
        check(lib().mlp_pcg_device_x0(E.A[i].h, C.c_void_p(b.data_ptr()), E.P[i].h, C.c_void_p(p.data_ptr()),
                                      1e-10, 0, 1, 1, C.byref(st), None))
        assert st.niter == itf[i]
        pn = p.cpu().numpy()
        assert np.array_equal(pn, E.p[i].cpu().numpy())
        g = np.zeros(len(pn))
        g[E.obs[i]] = pn[E.obs[i]] - p_obs[i]
        g_d = torch.from_numpy(g).cuda()
        lam = torch.empty_like(g_d)
        check(lib().mlp_pcg_device_x0(E.A[i].h, C.c_void_p(g_d.data_ptr()), E.P[i].h, C.c_void_p(lam.data_ptr()),
                                      1e-10, 0, 1, 1, C.byref(st), None))
        assert st.niter == ita[i]
        assert np.array_equal(lam.cpu().numpy(), E.lam_g[i].cpu().numpy())
        grad = torch.empty_like(g_d)
        check(lib().mlp_matrix_grad_logk(E.A[i].h, C.c_void_p(p.data_ptr()), C.c_void_p(lam.data_ptr()),
                                         C.c_void_p(grad.data_ptr()), None))
        gi = E.grad[i].cpu().numpy()
        assert np.array_equal(grad.cpu().numpy(), gi)
        # the oracle's FP64 gradient of the same member
        kx, ky, kz = fields.field("iid", 100 + i)
        Ao, bo = O.assemble(*d, kx, ky, kz, 1.0, True)
        Po = O.Prec(Ao, "msplit")
        po, _, _, rc = O.pcg(Ao, bo, Po, 1e-12, maxit=2000, x0_zero=True)
        assert rc == 0
        go = np.zeros(Ao.n)
        go[E.obs[i]] = po[E.obs[i]] - p_obs[i]
        lo, _, _, rc = O.pcg(Ao, go, Po, 1e-12, maxit=2000, x0_zero=True)
        assert rc in (0, -3)
        gref = O.grad_logk(*d, kx, ky, kz, po, lo)
        assert np.linalg.norm(gi - gref) <= 1e-5 * np.linalg.norm(gref), i
    E.close()
