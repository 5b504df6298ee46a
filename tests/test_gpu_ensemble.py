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
