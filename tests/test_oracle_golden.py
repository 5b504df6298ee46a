"""The CPU restatement (oracle/) against the reference's own outputs.

The golden fixtures were written by tests/golden/make_golden.py, which runs
the reference compiled from its own sources. Integer work (hierarchy shape,
permutation, factor patterns) and every factor value must match bit for bit;
the PCG iteration count and solution too, because the restatement keeps the
reference's operation order.
"""
import numpy as np
import pytest

from conftest import golden_cases
from oracle import oracle as O
from util import load_golden, oracle_prec


@pytest.mark.parametrize("name", golden_cases())
def test_hierarchy_bit_exact(name):
    g = load_golden(name)
    A = O.Matrix(g["A_ia"], g["A_ja"], g["A_a"])
    P = oracle_prec(A, g)
    assert P.nlevels == int(g["nlevels"])
    for l, ref in enumerate(g["levels"]):
        lv = P.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == ref[k], (l, k)
        if f"l{l}_map" in g and g[f"l{l}_map"].size:
            assert np.array_equal(lv["map"], g[f"l{l}_map"])
            assert np.array_equal(lv["dval"], g[f"l{l}_dval"])
            for m in ("L", "U"):
                ia, ja, a = lv[m]
                assert np.array_equal(ia, g[f"l{l}_{m}_ia"]), (l, m)
                assert np.array_equal(ja, g[f"l{l}_{m}_ja"]), (l, m)
                assert np.array_equal(a, g[f"l{l}_{m}_a"]), (l, m)
        if l > 0:
            ia, ja, a = lv["A"]
            assert np.array_equal(ia, g[f"l{l}_A_ia"])
            assert np.array_equal(ja, g[f"l{l}_A_ja"])
            assert np.array_equal(a, g[f"l{l}_A_a"])


@pytest.mark.parametrize("name", golden_cases())
def test_apply_and_pcg_bit_exact(name):
    g = load_golden(name)
    A = O.Matrix(g["A_ia"], g["A_ja"], g["A_a"])
    P = oracle_prec(A, g)
    z = P.apply(g["f_in"])
    assert np.array_equal(z, g["apply_out"])
    if g["options"].get("solver") == "cheb":
        lv = P.level(0)
        x, it, rel, rc = O.cheb_solve(A, g["b"], P, lv["lmin"], lv["lmax"], 1e-8)
    else:
        x, it, rel, rc = O.pcg(A, g["b"], P, 1e-8)
    assert rc == 0
    assert it == int(g["niter"])
    assert np.array_equal(x, g["x"])


@pytest.mark.parametrize("name", ["ms_iid_12x22x6", "ms_layered_16x22x8_c01", "ch_layered_16x22x8"])
def test_assembly_bit_exact(name):
    from ml_prec_b200 import fields
    g = load_golden(name)
    kx, ky, kz = fields.field(str(g["model"]), int(g["seed"]))
    A, b = O.assemble(int(g["nx"]), int(g["ny"]), int(g["nz"]), kx, ky, kz, float(g["c"]), True)
    # the field generator must reproduce the fixture's matrix exactly, or the
    # comparison below would only test numpy's pow
    assert np.array_equal(A.ia, g["A_ia"]) and np.array_equal(A.ja, g["A_ja"])
    assert np.array_equal(A.a, g["A_a"])
    assert np.array_equal(b, g["b"])


def test_generate_x0_matches_glibc_stream():
    x = O.generate_x0(5)
    # x_i = 20*(random()-RAND_MAX/2)/RAND_MAX + 100 lies in [90, 110]
    assert np.all((x >= 90) & (x <= 110))
    assert np.array_equal(O.generate_x0(5), x)
