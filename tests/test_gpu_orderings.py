"""The node orderings of the multi-split level build (msplit.cfg key
elim_order, multi_split_mark.cc) on the GPU beyond the golden cases.

* original (multi_split_mark.cc:27-154), with and without its tail group, at
  the full 60x220x85 size: every level's permutation and factors bit-exact
  against the oracle (which equals the reference on the original golden cases
  and in tests/test_oracle_vs_reference.py), PCG iterations within 1 and the
  solution within 1e-10.
* block (multi_split_mark.cc:193-252) accepts only the 60x220x85 mesh, so the
  reference fails on every other mesh at level 0 and on every mesh at level 1;
  the library must fail with the reference's message (recorded from the
  reference by tests/golden/make_golden.py). The level-1 size in that message
  is what the level-0 block ordering left over.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import ml_prec_b200 as M
    return M


@pytest.mark.parametrize("name", ["err_block_60x220x85", "err_block_16x22x8"])
def test_block_ordering_fails_like_the_reference(M, name):
    from ml_prec_b200 import fields
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        rec = json.load(f)
    kx, ky, kz = fields.field(rec["model"], rec["seed"])
    A, _ = M.CSRMatrix.spe(rec["nx"], rec["ny"], rec["nz"], kx, ky, kz, c=rec["c"])
    with pytest.raises(M.MlpError) as e:
        M.MultiSplitPrec(A, q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="block")
    assert e.value.code == 2  # MLP_ERR_CONFIG
    assert rec["message"] in str(e.value), (rec["message"], str(e.value))


@pytest.mark.parametrize("tails", [True, False])
def test_original_ordering_full_size(M, tails):
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("layered", 2)
    A, b = M.CSRMatrix.spe(60, 220, 85, kx, ky, kz, c=1.0)
    Ao, bo = O.assemble(60, 220, 85, kx, ky, kz, 1.0, True)
    kw = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="original", use_tails=tails)
    P = M.MultiSplitPrec(A, **kw)
    Po = O.Prec(Ao, "msplit", **kw)
    assert P.nlevels == Po.nlevels
    for l in range(Po.nlevels):
        lv, lo = P.level(l), Po.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == lo[k], (l, k)
        if "map" in lo:
            assert np.array_equal(lv["map"], lo["map"]), l
            for m in ("L", "U"):
                for t in range(3):
                    assert np.array_equal(lv[m][t], lo[m][t]), (l, m, t)
    st = M.SolverStats()
    x = M.PCGSolver(A, b, P, stats=st, eps=1e-8)
    xo, it, _, rc = O.pcg(Ao, bo, Po, 1e-8)
    assert rc == 0 and abs(st.niter - it) <= 1
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
