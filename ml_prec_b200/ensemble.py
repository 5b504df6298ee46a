"""Batching form: an ensemble of permeability realizations on meshes of uneven
size, solved (forward and adjoint) as parallel branches of one CUDA graph.

Each realization r gets its own mesh nx in [30, 60], ny in [110, 220],
nz in [10, 85] (seeded) and its own i.i.d. log-normal field (the
small-mesh model), its own matrix and FP32-stored multi-split hierarchy; the forward
solves (right-hand side from the Dirichlet faces) and the adjoint solves
(misfit gradient at 25 observation cells) of all realizations each run as one
graph launch (mlp_ensemble_solve). The members' row kernels take their launch
shapes from the build-time autotuner (mlp_prec_cfg.autotune). Sharding the
ensemble over several GPUs
assigns whole realizations to ranks (no data exchange during the solves).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api, fields
from ._capi import Stats, check, lib

MSPLIT = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="simple_1")


def realization_dims(count=64, seed=5):
    rng = np.random.default_rng(seed)
    nx = rng.integers(30, 61, size=count)
    ny = rng.integers(110, 221, size=count)
    nz = rng.integers(10, 86, size=count)
    return [(int(a), int(b), int(c)) for a, b, c in zip(nx, ny, nz)]


def shard(dims, rank, world):
    """Realizations of one rank: greedy balance of the cell counts (largest
    first to the least-loaded rank), the same on every rank."""
    order = sorted(range(len(dims)), key=lambda i: (-int(np.prod(dims[i])), i))
    load = [0] * world
    owner = [0] * len(dims)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(np.prod(dims[i]))
    return [i for i in range(len(dims)) if owner[i] == rank]


class Ensemble:
    """Matrices, hierarchies and the two ensemble graphs (forward, adjoint)."""

    def __init__(self, dims, field_seed0=100, fp32=True, prec_kw=None, nobs=25, obs_seed=9, autotune=True):
        import torch
        self.dims = list(dims)
        self.fp32 = fp32
        kw = dict(MSPLIT if prec_kw is None else prec_kw)
        self.A, self.P, self.b, self.obs = [], [], [], []
        rng = np.random.default_rng(obs_seed)
        for i, (nx, ny, nz) in enumerate(self.dims):
            kx, ky, kz = fields.field("iid", field_seed0 + i)
            A, b = api.CSRMatrix.spe(nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True)
            P = api.MultiSplitPrec(A, fp32=fp32, autotune=autotune, **kw)
            self.A.append(A)
            self.P.append(P)
            self.b.append(torch.from_numpy(b).cuda())
            self.obs.append(np.sort(rng.choice(A.n, size=min(nobs, A.n), replace=False)))
        self.x = [torch.empty_like(b) for b in self.b]
        self.lam = [torch.empty_like(b) for b in self.b]
        self.g = [torch.zeros_like(b) for b in self.b]
        self.fwd = self._make(x0_mode=0)
        self.adj = self._make(x0_mode=1)

    def _make(self, x0_mode):
        arr = (C.c_void_p * len(self.P))(*[P.h.value for P in self.P])
        h = C.c_void_p()
        check(lib().mlp_ensemble_create(len(self.P), arr, int(self.fp32), x0_mode, C.byref(h)))
        return h

    def _solve(self, h, b, x, eps):
        K = len(self.P)
        bp = (C.c_void_p * K)(*[t.data_ptr() for t in b])
        xp = (C.c_void_p * K)(*[t.data_ptr() for t in x])
        st = (Stats * K)()
        t = C.c_double()
        check(lib().mlp_ensemble_solve(h, bp, xp, eps, 0, st, C.byref(t), None))
        return t.value, [st[i].niter for i in range(K)]

    def forward(self, eps=1e-8):
        """All forward solves in one launch; returns (ms, iterations)."""
        return self._solve(self.fwd, self.b, self.x, eps)

    def adjoint(self, p_obs, eps=1e-8):
        """All adjoint solves A lambda = dJ/dp in one launch (J = 0.5 sum over the
        observation cells of (p - p_obs)^2), from the current forward solutions."""
        import torch
        for i in range(len(self.P)):
            p = self.x[i].cpu().numpy()
            g = np.zeros(self.A[i].n)
            g[self.obs[i]] = p[self.obs[i]] - p_obs[i]
            self.g[i].copy_(torch.from_numpy(g))
        return self._solve(self.adj, self.g, self.lam, eps)

    def gradient(self, p_obs, eps=1e-8):
        """Forward solve, misfit gradient, adjoint solve and dJ/dlnK of every
        member in ONE graph launch (mlp_ensemble_gradient_create); both solves
        start from zero. Fills self.p, self.lam_g and self.grad; returns (ms,
        forward iterations, adjoint iterations)."""
        import torch
        K = len(self.P)
        if getattr(self, "grad_h", None) is None or self._pobs_shape != [len(o) for o in p_obs]:
            if getattr(self, "grad_h", None):
                lib().mlp_ensemble_destroy(self.grad_h)
            self.obs_d = [torch.from_numpy(o.astype(np.uint32)).cuda() for o in self.obs]
            self.pobs_d = [torch.zeros(len(o), dtype=torch.float64, device="cuda") for o in self.obs]
            self.p = [torch.empty_like(b) for b in self.b]
            self.lam_g = [torch.empty_like(b) for b in self.b]
            self.grad = [torch.empty_like(b) for b in self.b]
            vp = C.c_void_p
            arr = lambda ts: (vp * K)(*[t.data_ptr() for t in ts])
            h = C.c_void_p()
            nobs = np.array([len(o) for o in self.obs], np.uint32)
            check(lib().mlp_ensemble_gradient_create(
                K, (vp * K)(*[A.h.value for A in self.A]), (vp * K)(*[P.h.value for P in self.P]),
                arr(self.obs_d), nobs.ctypes.data_as(C.POINTER(C.c_uint32)), arr(self.pobs_d), arr(self.p),
                arr(self.lam_g), arr(self.grad), int(self.fp32), C.byref(h)))
            self.grad_h = h
            self._pobs_shape = [len(o) for o in p_obs]
        for i in range(K):
            self.pobs_d[i].copy_(torch.from_numpy(np.asarray(p_obs[i], np.float64)))
        bp = (C.c_void_p * K)(*[t.data_ptr() for t in self.b])
        st = (Stats * (2 * K))()
        t = C.c_double()
        check(lib().mlp_ensemble_solve(self.grad_h, bp, None, eps, 0, st, C.byref(t), None))
        return t.value, [st[i].niter for i in range(K)], [st[K + i].niter for i in range(K)]

    def looped_forward(self, eps=1e-8):
        """The same forward solves one handle at a time (single-instance path)."""
        import time
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its = []
        for i in range(len(self.P)):
            st = Stats()
            check(lib().mlp_pcg_device(self.A[i].h, C.c_void_p(self.b[i].data_ptr()), self.P[i].h,
                                       C.c_void_p(self.x[i].data_ptr()), eps, 0, int(self.fp32), C.byref(st),
                                       None))
            its.append(st.niter)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3, its

    def close(self):
        for h in (getattr(self, "fwd", None), getattr(self, "adj", None), getattr(self, "grad_h", None)):
            if h:
                lib().mlp_ensemble_destroy(h)
        self.fwd = self.adj = self.grad_h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
