"""Failure paths of the solver through the C ABI.

Every failure here is made on the host with inputs that a GPU computes on
without faulting: an indefinite matrix, a right-hand side holding a NaN, a
mesh without the reaction term. Each must come back as the documented status
code with the reference's message, and the device context must stay usable
afterwards (the last test solves a normal system on it).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MSPLIT = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2)


@pytest.fixture(scope="module")
def M():
    import ml_prec_b200 as M
    return M


def test_indefinite_matrix_stops_on_curvature(M):
    """<Ap, p> <= 0 throws in the reference (pcg.cc:51-55). A negative
    diagonal matrix makes a one-level hierarchy whose apply is A^{-1}, so the
    first <Ap, p> = <r0, A^{-1} r0> is negative; the oracle fails the same way."""
    from oracle import oracle as O
    n = 64
    rng = np.random.default_rng(0)
    ia = np.arange(n + 1, dtype=np.uint32)
    ja = np.arange(n, dtype=np.uint32)
    a = -(1 + rng.random(n))
    b = rng.standard_normal(n)
    Ao = O.Matrix(ia, ja, a)
    _, it, _, rc = O.pcg(Ao, b, O.Prec(Ao, "msplit", **MSPLIT), 1e-8)
    assert rc != 0 and it == 0
    A = M.CSRMatrix.from_arrays(ia, ja, a)
    P = M.MultiSplitPrec(A, **MSPLIT)
    with pytest.raises(M.MlpError) as e:
        M.PCGSolver(A, b, P, eps=1e-8)
    assert e.value.code == 4  # MLP_ERR_CURVATURE
    assert "<Ap, p>" in str(e.value)


def test_nan_in_right_hand_side_is_reported(M):
    """A NaN in b makes the initial residual norm non-finite: the solve stops
    before its first iteration with MLP_ERR_NOT_FINITE instead of iterating on
    NaNs or claiming "No need to iterate"."""
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("iid", 1)
    A, b = M.CSRMatrix.spe(12, 22, 6, kx, ky, kz, c=1.0)
    P = M.MultiSplitPrec(A, **MSPLIT)
    b = b.copy()
    b[17] = np.nan
    with pytest.raises(M.MlpError) as e:
        M.PCGSolver(A, b, P, eps=1e-8)
    assert e.value.code == 5  # MLP_ERR_NOT_FINITE


def test_uh_cheb_without_reaction_term_has_too_many_levels(M):
    """With c = 0 on a Neumann mesh uh_cheb never coarsens enough and the
    reference throws "Too many levels" (cheb_constr.cc:282-283); so do the
    oracle and the GPU build (MLP_ERR_LEVELS)."""
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("iid", 1)
    Ao, _ = O.assemble(12, 22, 6, kx, ky, kz, 0.0, False)
    with pytest.raises(Exception, match="Too many levels"):
        O.Prec(Ao, "cheb", sigma=(3.0,), ncheb=(2,), use_tails=True)
    A, _ = M.CSRMatrix.spe(12, 22, 6, kx, ky, kz, c=0.0, dirichlet=False)
    with pytest.raises(M.MlpError) as e:
        M.Prec(A, sigma=(3.0,), ncheb=(2,), use_tails=True)
    assert e.value.code == 3  # MLP_ERR_LEVELS
    assert "Too many levels" in str(e.value)


def test_multisplit_without_reaction_term_ends_in_the_direct_level(M):
    """Multi-split with c = 0 on a Neumann mesh drops no link, so every level
    keeps all 1,584 unknowns until max_levels; like the reference built with
    its coarsest-level direct solver (multi_split_constr.cc:46-55 with
    HAVE_UMFPACK), the last level is then solved directly. Level sizes equal
    the oracle's. With one inner iteration per level the application is a
    chain of 15 levels; with five it would be 5^14 coarsest solves per
    application, and the GPU build refuses that plan with MLP_ERR_LIMIT
    instead of recording it."""
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("iid", 1)
    one = dict(MSPLIT, niter=(1,))
    Ao, _ = O.assemble(12, 22, 6, kx, ky, kz, 0.0, False)
    Po = O.Prec(Ao, "msplit", **one)
    A, _ = M.CSRMatrix.spe(12, 22, 6, kx, ky, kz, c=0.0, dirichlet=False)
    P = M.MultiSplitPrec(A, **one)
    assert P.nlevels == Po.nlevels == 15
    assert [P.level(l)["N"] for l in range(15)] == [Po.level(l)["N"] for l in range(15)]
    assert P.level(14)["direct"]
    assert np.isfinite(P.solve(np.random.default_rng(3).standard_normal(A.n))).all()
    with pytest.raises(M.MlpError) as e:
        M.MultiSplitPrec(A, **MSPLIT)
    assert e.value.code == 9  # MLP_ERR_LIMIT


def test_context_survives_the_failures(M):
    """After the failures above, a normal solve on the same device still
    matches the oracle (iterations within 1, solution within 1e-10)."""
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("iid", 1)
    A, b = M.CSRMatrix.spe(12, 22, 6, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(12, 22, 6, kx, ky, kz, 1.0, True)
    st = M.SolverStats()
    x = M.PCGSolver(A, b, M.MultiSplitPrec(A, **MSPLIT), stats=st, eps=1e-8)
    xo, it, _, rc = O.pcg(Ao, bo, O.Prec(Ao, "msplit", **MSPLIT), 1e-8)
    assert rc == 0 and abs(st.niter - it) <= 1
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
