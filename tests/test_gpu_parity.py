"""CUDA path against the reference's outputs (golden fixtures) and the oracle.

Bar: integer work (hierarchy shape, node permutation, factor and coarse-matrix
sparsity) bit-exact; factor and coarse-matrix values bit-exact too (the setup
kernels are compiled without FMA contraction and keep the reference's operation
order); preconditioner apply within 1e-12 relative (parallel reductions change
the rounding); PCG iteration count within +-1 and solution within 1e-10
relative of the reference's.
"""
import numpy as np
import pytest

from conftest import golden_cases
from util import gpu_prec, load_golden, oracle_prec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import ml_prec_b200 as M
    return M


@pytest.fixture(params=["persistent", "persist_split", "dense", "nofold", "separate", "small", "explicit", "waves"])
def apply_path(request, monkeypatch):
    """Run each case through every apply path: the whole apply as one
    persistent launch (MLP_PERSIST=1 at these sizes), the finest level as separate
    launches around a persistent launch of the levels below it, the tabulated
    small-level operator with separate launches and the correction and
    phase-1 steps of the small levels merged (the coarse product folded into
    phase 2, and not), the same with every sweep step a
    separate kernel, the shared-memory small-level kernel (tabulation off),
    the launch path with explicit triangular solves (small kernel off), and
    the launch path with wavefront triangular solves."""
    if request.param in ("persistent", "persist_split"):
        monkeypatch.setenv("MLP_PERSIST", "1")
    if request.param == "persist_split":
        monkeypatch.setenv("MLP_PERSIST_MAX_N", "1200")
    if request.param in ("dense", "nofold", "separate", "small", "explicit", "waves"):
        monkeypatch.setenv("MLP_PERSIST", "0")
    if request.param == "nofold":
        monkeypatch.setenv("MLP_FOLD", "0")
    if request.param == "separate":
        monkeypatch.setenv("MLP_MERGE", "0")
    if request.param == "small":
        monkeypatch.setenv("MLP_DENSE_OP_MAX", "0")
    if request.param in ("explicit", "waves"):
        monkeypatch.setenv("MLP_SMALL_BUDGET", "0")
    if request.param == "waves":
        monkeypatch.setenv("MLP_EXPLICIT", "0")
    return request.param


def gpu_matrix(M, g):
    return M.CSRMatrix.from_arrays(g["A_ia"], g["A_ja"], g["A_a"])


@pytest.mark.parametrize("name", golden_cases())
def test_hierarchy_bit_exact(M, name):
    g = load_golden(name)
    A = gpu_matrix(M, g)
    P = gpu_prec(A, g)
    assert P.nlevels == int(g["nlevels"])
    for l, ref in enumerate(g["levels"]):
        lv = P.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == ref[k], (l, k, lv[k], ref[k])
        if not lv["direct"] and f"l{l}_map" in g and g[f"l{l}_map"].size:
            assert np.array_equal(lv["map"], g[f"l{l}_map"]), l
            assert np.array_equal(lv["dval"], g[f"l{l}_dval"]), l
            for m in ("L", "U"):
                ia, ja, a = lv[m]
                assert np.array_equal(ia, g[f"l{l}_{m}_ia"]), (l, m)
                assert np.array_equal(ja, g[f"l{l}_{m}_ja"]), (l, m)
                assert np.array_equal(a, g[f"l{l}_{m}_a"]), (l, m)
        if l > 0:
            ia, ja, a = lv["A"]
            assert np.array_equal(ia, g[f"l{l}_A_ia"]), l
            assert np.array_equal(ja, g[f"l{l}_A_ja"]), l
            assert np.array_equal(a, g[f"l{l}_A_a"]), l


def launch_path_refuses_dynamic(M, g, A, apply_path):
    """Dynamic inner iterations (inner_iter = dynamic) decide the number of
    sweeps on the device inside the persistent launch; the launch-per-step
    paths refuse them with MLP_ERR_CONFIG. Returns True when that was checked."""
    if "level_eps" not in g["options"] or apply_path in ("persistent", "persist_split"):
        return False
    with pytest.raises(M.MlpError) as e:
        gpu_prec(A, g)
    assert e.value.code == 2 and "persistent" in str(e.value)
    return True


@pytest.mark.parametrize("name", golden_cases())
def test_apply_matches_reference(M, name, apply_path):
    g = load_golden(name)
    A = gpu_matrix(M, g)
    if launch_path_refuses_dynamic(M, g, A, apply_path):
        return
    P = gpu_prec(A, g)
    z = P.solve(g["f_in"])
    ref = g["apply_out"]
    assert np.linalg.norm(z - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("name", golden_cases())
def test_pcg_matches_reference(M, name, apply_path):
    g = load_golden(name)
    A = gpu_matrix(M, g)
    if launch_path_refuses_dynamic(M, g, A, apply_path):
        return
    P = gpu_prec(A, g)
    st = M.SolverStats()
    if g["options"].get("solver") == "cheb":  # ChebSolver as the outer iteration (cheb.cc:9-100)
        x = M.ChebSolver(A, P.lmin(), P.lmax(), g["b"], P, stats=st, eps=1e-8)
    else:
        x = M.PCGSolver(A, g["b"], P, stats=st, eps=1e-8)
    assert abs(st.niter - int(g["niter"])) <= 1
    assert np.linalg.norm(x - g["x"]) <= 1e-10 * np.linalg.norm(g["x"])


@pytest.mark.parametrize("model,seed,dims,c", [("iid", 1, (12, 22, 6), 1.0), ("layered", 2, (60, 220, 85), 1.0),
                                                ("layered", 7, (31, 17, 9), 0.1)])
def test_assembly_bit_exact(M, model, seed, dims, c):
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field(model, seed)
    A, b = M.CSRMatrix.spe(*dims, kx, ky, kz, c=c, dirichlet=True)
    Ao, bo = O.assemble(*dims, kx, ky, kz, c, True)
    ia, ja, a = A.arrays()
    assert np.array_equal(ia, Ao.ia) and np.array_equal(ja, Ao.ja)
    assert np.array_equal(a, Ao.a)
    assert np.array_equal(b, bo)


def test_full_size_hierarchy_and_pcg_against_oracle(M):
    """60x220x85 layered field (1,122,000 cells): hierarchy bit-exact on every
    level, PCG iterations within +-1 of the oracle's."""
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(60, 220, 85, kx, ky, kz, 1.0, True)
    P = M.MultiSplitPrec(A, q=(0.8,), niter=(5,), max_levels=15, degree_max=2)
    Po = O.Prec(Ao, "msplit", q=(0.8,), niter=(5,), max_levels=15, degree_max=2)
    assert P.nlevels == Po.nlevels
    for l in range(Po.nlevels):
        lv, lo = P.level(l), Po.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == lo[k], (l, k)
        if "map" in lo:
            assert np.array_equal(lv["map"], lo["map"])
            for m in ("L", "U"):
                for t in range(3):
                    assert np.array_equal(lv[m][t], lo[m][t]), (l, m, t)
    st = M.SolverStats()
    x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
    xo, it, rel, rc = O.pcg(Ao, bo, Po, 1e-8)
    assert rc == 0 and abs(st.niter - it) <= 1
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


@pytest.mark.parametrize("fp32", [False, True])
def test_device_loop_matches_host_loop(M, fp32, monkeypatch):
    """A solve runs as one graph launch (start, conditional WHILE loop,
    scatter); the host-driven loop (one round trip per iteration) must give the
    same iterates."""
    g = load_golden("ms_layered_16x22x8_c01")
    A = gpu_matrix(M, g)
    P = gpu_prec(A, g, fp32=fp32)
    st1 = M.SolverStats()
    x1 = M.PCGSolver(A, g["b"], P, stats=st1, eps=1e-8)
    monkeypatch.setenv("MLP_PCG_HOSTLOOP", "1")
    st2 = M.SolverStats()
    x2 = M.PCGSolver(A, g["b"], P, stats=st2, eps=1e-8)
    assert st1.niter == st2.niter
    assert np.array_equal(x1, x2)


def test_iteration_cap_ends_the_device_loop(M):
    """An unreachable tolerance stops at the cap with MLP_ERR_MAXIT."""
    g = load_golden("ms_iid_12x22x6")
    A = gpu_matrix(M, g)
    P = gpu_prec(A, g)
    with pytest.raises(M.MlpError) as e:
        M.PCGSolver(A, g["b"], P, eps=1e-30, maxit=7)
    assert e.value.code == 6


@pytest.mark.parametrize("fp32", [False, True])
def test_apply_forms_are_bit_identical(M, fp32, monkeypatch):
    """60x220x85 layered field: the levels below the finest one run as one
    persistent launch (MLP_PERSIST=1); as separate launches with the
    correction and phase-1 steps of the small levels merged; and as separate
    launches with every sweep step its own kernel (both with the coarse
    product as its own launch, MLP_FOLD=0). All three repeat the same
    arithmetic (same products, lane split and butterfly order), so the apply
    and the PCG iterates are bit-identical. The default folds the coarse
    product into phase 2 ((G_C C) w_C in place of G_C (C w_C)), which changes
    the rounding: test_folded_coarse_product holds it to the unfolded form."""
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    f = np.random.default_rng(5).standard_normal(A.n)
    kw = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, fp32=fp32)
    out = []
    for env in ({"MLP_PERSIST": "1"}, {"MLP_FOLD": "0"}, {"MLP_FOLD": "0", "MLP_MERGE": "0"}):
        for k in ("MLP_PERSIST", "MLP_MERGE", "MLP_FOLD"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        P = M.MultiSplitPrec(A, **kw)
        z = P.solve(f)
        st = M.SolverStats()
        x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
        out.append((z, st.niter, x))
    for z, it, x in out[1:]:
        assert np.array_equal(z, out[0][0])
        assert it == out[0][1] and np.array_equal(x, out[0][2])


@pytest.mark.parametrize("name", ["ms_iid_12x22x6", "ms_layered_16x22x8_c01"])
def test_autotuned_launch_shapes_match_reference(M, name):
    """Plans whose row kernels take their launch shapes from the build-time
    autotuner (lanes per row, block size) give the reference's PCG result:
    iterations within 1, solution within 1e-10 relative."""
    g = load_golden(name)
    A = gpu_matrix(M, g)
    kw = dict(q=(0.8,), niter=tuple(int(t) for t in str(g["options"].get("level_niter", "5")).split()),
              max_levels=g["options"].get("max_levels", 15), degree_max=g["options"].get("degree_max", 2))
    P = M.MultiSplitPrec(A, autotune=True, **kw)
    st = M.SolverStats()
    x = M.PCGSolver(A, g["b"], P, stats=st, eps=1e-8)
    assert abs(st.niter - int(g["niter"])) <= 1
    assert np.linalg.norm(x - g["x"]) <= 1e-10 * np.linalg.norm(g["x"])


def test_autotuned_full_size_pcg(M):
    """60x220x85: autotuned plan against the fixed-heuristic plan, same
    tolerance and iterations within 1."""
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    kw = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2)
    st1, st2 = M.SolverStats(), M.SolverStats()
    x1 = M.PCGSolver(A, b, M.MultiSplitPrec(A, autotune=True, **kw), stats=st1, eps=1e-8)
    x2 = M.PCGSolver(A, b, M.MultiSplitPrec(A, **kw), stats=st2, eps=1e-8)
    assert abs(st1.niter - st2.niter) <= 1 and st1.final_rel <= 1e-8
    assert np.linalg.norm(x1 - x2) <= 1e-9 * np.linalg.norm(x2)


def test_in_graph_timeline(M, monkeypatch):
    """mlp_prec_timeline gives one positive in-graph time per launch of the
    plan (names and bytes as the launch-by-launch profile), mlp_pcg_timeline
    one per launch of a PCG iteration; a plan with a
    launch that stamps no time (the persistent kernel) is refused with
    MLP_ERR_INTERNAL instead of returning misattributed times."""
    g = load_golden("ms_layered_16x22x8_c01")
    A = gpu_matrix(M, g)
    monkeypatch.setenv("MLP_PERSIST", "0")
    P = gpu_prec(A, g)
    P.solve(g["f_in"])
    tl = P.timeline(4)
    prof = P.profile(1)
    assert [t[0] for t in tl] == [p[0] for p in prof]
    assert all(us > 0 for _, us, _ in tl)
    import torch
    b = torch.from_numpy(np.ascontiguousarray(g["b"], dtype=np.float64)).cuda()
    x = torch.empty_like(b)
    pt = P.pcg_timeline(A, b, x, 1e-8)
    assert [t[0] for t in pt] == ["pcg spmv_dot", "pcg update"] + [p[0] for p in prof] + ["pcg dot_rz", "pcg p"]
    assert all(us > 0 for _, us in pt)
    monkeypatch.setenv("MLP_PERSIST", "1")
    P1 = gpu_prec(A, g)
    P1.solve(g["f_in"])
    with pytest.raises(M.MlpError) as e:
        P1.timeline(4)
    assert e.value.code == 10


@pytest.mark.parametrize("fp32", [False, True])
def test_folded_coarse_product(M, fp32, monkeypatch):
    """60x220x85 layered field: the default plan folds the tabulated 422-row
    coarse operator into phase 2 of level 2 (one launch less per level-2
    sweep). Against the unfolded plan: the apply within 1e-13 (FP64) / 1e-6
    (FP32 form) relative, PCG within one iteration and 1e-10 / 1e-6."""
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    f = np.random.default_rng(5).standard_normal(A.n)
    kw = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, fp32=fp32)
    out = []
    for env in ({}, {"MLP_FOLD": "0"}):
        monkeypatch.delenv("MLP_FOLD", raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        P = M.MultiSplitPrec(A, **kw)
        z = P.solve(f)
        names = [t[0] for t in P.profile(1)]
        st = M.SolverStats()
        x = M.PCGSolver(A, b, P, stats=st, eps=1e-8, flexible=fp32)
        out.append((z, st.niter, x, names))
    (zf, itf, xf, nf), (zu, itu, xu, nu) = out
    assert any(n.startswith("phase2_fold") for n in nf) and not any(n.startswith("phase2_fold") for n in nu)
    assert len(nf) < len(nu)
    tol = 1e-6 if fp32 else 1e-13
    assert np.linalg.norm(zf - zu) <= tol * np.linalg.norm(zu)
    assert abs(itf - itu) <= 1
    assert np.linalg.norm(xf - xu) <= (1e-6 if fp32 else 1e-10) * np.linalg.norm(xu)
