"""The benchmark configurations at their own sizes on the GPU, against the
oracle. The oracle equals the reference on the same problems: bit for bit on
the golden fixtures, and run side by side in tests/test_oracle_vs_reference.py
(including the 2-level 60x220x10 problem with the direct coarsest solve).

* 60x220x10 (132,000 cells, i.i.d. field), 2 levels with the dense coarsest
  solve (about 1,600 unknowns): hierarchy bit-exact, PCG to 1e-8 within one
  iteration and 1e-10 of the oracle's solution.
* The FP32 form on that matrix (hierarchy stored and applied in FP32, the
  coarsest solve in FP64, flexible FP64 PCG) at 1e-8 and 1e-10: iterations and
  the solution error against the oracle's FP64 solution at 1e-12.
* uh_cheb (sigma 3, degree 4) on the 60x220x85 layered field: hierarchy
  bit-exact, PCG within one iteration and 1e-10; its merged residual + phase-1
  launches bit-identical to the separate ones.
* The FP32 form on the 60x220x85 multi-split problem against the oracle (at
  1e-8 and 1e-9: there the FP64 iteration itself stagnates near 5.6e-10).
* Ensemble members against the oracle, forward and adjoint (FP64 members to
  1e-10; the FP32 form by true residual and to 1e-4).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MS2 = dict(q=(0.8,), niter=(5,), max_levels=2, degree_max=2)
MS = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2)


@pytest.fixture(scope="module")
def M():
    import ml_prec_b200 as M
    return M


def hierarchy_equal(P, Po):
    assert P.nlevels == Po.nlevels
    for l in range(Po.nlevels):
        lv, lo = P.level(l), Po.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == lo[k], (l, k, lv[k], lo[k])
        if "map" in lo and not lv["direct"]:
            assert np.array_equal(lv["map"], lo["map"]), l
            for m in ("L", "U"):
                for t in range(3):
                    assert np.array_equal(lv[m][t], lo[m][t]), (l, m, t)
        if l > 0:
            for t in range(3):
                assert np.array_equal(lv["A"][t], lo["A"][t]), (l, "A", t)


@pytest.fixture(scope="module")
def config1():
    import ml_prec_b200 as M
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("iid", 1)
    A, b = M.CSRMatrix.spe(60, 220, 10, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(60, 220, 10, kx, ky, kz, 1.0, True)
    Po = O.Prec(Ao, "msplit", **MS2)
    x12, it12, _, rc = O.pcg(Ao, bo, Po, 1e-12, maxit=500)
    assert rc == 0
    return A, b, Ao, bo, Po, x12


def test_config1_two_level_direct_coarse(M, config1):
    from oracle import oracle as O
    A, b, Ao, bo, Po, _ = config1
    P = M.MultiSplitPrec(A, **MS2)
    assert P.nlevels == 2 and P.level(1)["direct"] and P.level(1)["N"] <= 4000
    hierarchy_equal(P, Po)
    st = M.SolverStats()
    x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
    xo, it, _, rc = O.pcg(Ao, bo, Po, 1e-8)
    assert rc == 0 and abs(st.niter - it) <= 1
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


@pytest.mark.parametrize("eps,bound", [(1e-8, 1e-5), (1e-10, 1e-7)])
def test_config3_fp32_form_against_fp64_oracle(M, config1, eps, bound):
    """Solution error of the FP32-stored hierarchy in flexible FP64 PCG
    against the FP64 oracle solved to 1e-12; the FP64 GPU path at the same
    tolerance is held to the same bound."""
    A, b, Ao, bo, Po, x12 = config1
    nrm = np.linalg.norm(x12)
    P32 = M.MultiSplitPrec(A, fp32=True, **MS2)
    st = M.SolverStats()
    x32 = M.PCGSolver(A, b, P32, stats=st, eps=eps, flexible=True)
    assert st.final_rel <= eps
    x64 = M.PCGSolver(A, b, M.MultiSplitPrec(A, **MS2), eps=eps)
    e32 = np.linalg.norm(x32 - x12) / nrm
    e64 = np.linalg.norm(x64 - x12) / nrm
    print(f"eps {eps:g}: FP32 form {st.niter} iterations, error {e32:.2e}; FP64 error {e64:.2e}")
    assert e32 <= bound and e64 <= bound


def test_uh_cheb_full_size(M):
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(60, 220, 85, kx, ky, kz, 1.0, True)
    kw = dict(sigma=(3.0,), ncheb=(4,), use_tails=True)
    P = M.Prec(A, **kw)
    Po = O.Prec(Ao, "cheb", **kw)
    hierarchy_equal(P, Po)
    st = M.SolverStats()
    x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
    xo, it, _, rc = O.pcg(Ao, bo, Po, 1e-8)
    assert rc == 0 and abs(st.niter - it) <= 1
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


@pytest.mark.parametrize("fp32", [False, True])
def test_uh_cheb_merged_residual_is_bit_identical(M, fp32, monkeypatch):
    """uh_cheb (sigma 3, degree 4) on the 60x220x85 layered field, whose level
    4 (11,452 rows) is called 256 times per application: the Chebyshev
    residual F - As u and phase 1 of the level call after it as one launch
    (k_merge_a with As), and each call of the tabulated small levels with the
    Chebyshev update after it as one launch (k_dense_gemv_epi), give the same
    application and PCG iterates, bit for bit, as the separate launches
    (MLP_MERGE=0)."""
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    f = np.random.default_rng(7).standard_normal(A.n)
    out = []
    for env in ("1", "0"):
        monkeypatch.setenv("MLP_MERGE", env)
        P = M.Prec(A, fp32=fp32, sigma=(3.0,), ncheb=(4,), use_tails=True)
        z = P.solve(f)
        names = [nm for nm, _, _ in P.profile(1)]
        st = M.SolverStats()
        x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
        out.append((names, z, st.niter, x))
        del P
    (n1, z1, it1, x1), (n0, z0, it0, x0) = out
    assert "merge_a L4" in n1 and not any(nm.startswith("merge_a") for nm in n0)
    assert any(nm.startswith("dense_step") for nm in n1) and not any(nm.startswith("dense_step") for nm in n0)
    assert len(n1) < len(n0)
    assert np.array_equal(z1, z0)
    assert it1 == it0 and np.array_equal(x1, x0)


def test_fp32_form_full_size_against_oracle(M):
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(60, 220, 85, kx, ky, kz, 1.0, True)
    # 1e-9: at this size and contrast the FP64 iteration (the oracle's, like
    # the reference's) stagnates near 5.6e-10 (rounding; 81 iterations reach
    # 1e-9, 300 stop at 5.6e-10), so a tighter tolerance only runs into the cap
    xo, it, rel, rc = O.pcg(Ao, bo, O.Prec(Ao, "msplit", **MS), 1e-9, maxit=300)
    assert rc == 0 and rel <= 1e-9
    P32 = M.MultiSplitPrec(A, fp32=True, **MS)
    nrm = np.linalg.norm(xo)
    for eps, bound in ((1e-8, 1e-4), (1e-9, 1e-5)):
        st = M.SolverStats()
        x = M.PCGSolver(A, b, P32, stats=st, eps=eps, flexible=True)
        err = np.linalg.norm(x - xo) / nrm
        print(f"60x220x85 FP32 form eps {eps:g}: {st.niter} iterations, error {err:.2e}")
        assert st.final_rel <= eps and err <= bound


def test_ensemble_members_against_oracle():
    """FP64 members (fixed launch shapes) equal the oracle's solves like single
    solves do (iterations within 1, solution within 1e-10). The FP32 autotuned
    ensemble runs another iteration (FP32 preconditioner, flexible PCG), so it
    is held to what the tolerance promises: a true FP64 residual within 10x
    of the oracle's own, and a solution within 1e-4 of the oracle's (two
    solutions with relative residual 1e-8 differ by up to cond(A) 1e-8),
    forward and adjoint."""
    from ml_prec_b200 import ensemble, fields
    from oracle import oracle as O
    dims = [(30, 110, 10), (7, 11, 5), (12, 22, 6), (31, 17, 9), (16, 40, 12)]
    ref = []
    for i, d in enumerate(dims):
        kx, ky, kz = fields.field("iid", 100 + i)
        Ao, bo = O.assemble(*d, kx, ky, kz, 1.0, True)
        Po = O.Prec(Ao, "msplit", **MS)
        xo, it, _, rc = O.pcg(Ao, bo, Po, 1e-8)
        assert rc == 0
        ref.append((Ao, Po, xo, it, bo))
    E = ensemble.Ensemble(dims, fp32=False, autotune=False)
    _, its = E.forward(eps=1e-8)
    for i, (Ao, Po, xo, it, bo) in enumerate(ref):
        x = E.x[i].cpu().numpy()
        assert abs(its[i] - it) <= 1, i
        assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo), i
    E.close()
    E = ensemble.Ensemble(dims, fp32=True)
    E.forward(eps=1e-8)
    p_obs = [np.zeros(len(o)) for o in E.obs]
    E.adjoint(p_obs, eps=1e-8)
    def res(A, b, x):
        return np.linalg.norm(b - O.spmv(A, x))

    for i, (Ao, Po, xo, it, bo) in enumerate(ref):
        x = E.x[i].cpu().numpy()
        assert res(Ao, bo, x) <= 10 * res(Ao, bo, xo), i
        assert np.linalg.norm(x - xo) <= 1e-4 * np.linalg.norm(xo), i
        g = E.g[i].cpu().numpy()
        lo, _, _, rc = O.pcg(Ao, g, Po, 1e-8, x0_zero=True)
        assert rc == 0
        lam = E.lam[i].cpu().numpy()
        assert res(Ao, g, lam) <= 10 * res(Ao, g, lo), i
        assert np.linalg.norm(lam - lo) <= 1e-4 * np.linalg.norm(lo), i
    E.close()
