"""The oracle against the reference itself at sizes beyond the golden
fixtures: the reference compiled from its own sources (oracle/_ref/ref_driver,
built by `make -C oracle ref`) and the oracle run on the same seeded problems;
hierarchy shape per level, PCG iteration count and the solution must agree
exactly. CPU only; skipped where the reference driver was not built."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

# (model, seed, nx, ny, nz, c, elim_order, use_tails, max_levels); the last case
# is the 2-level problem with the direct coarsest solve on the 60x220x10 mesh
CASES = [("layered", 2, 40, 60, 20, 1.0, "simple_1", None, 15), ("iid", 4, 30, 44, 16, 0.1, "simple_1", None, 15),
         ("layered", 2, 30, 40, 20, 1.0, "original", 1, 15), ("iid", 4, 30, 44, 16, 1.0, "original", 0, 15),
         ("iid", 1, 60, 220, 10, 1.0, "simple_1", None, 2)]


@pytest.mark.parametrize("model,seed,nx,ny,nz,c,order,tails,max_levels", CASES)
def test_oracle_equals_reference(tmp_path, model, seed, nx, ny, nz, c, order, tails, max_levels):
    if not O.ref_available():
        pytest.skip("reference driver not built")
    from ml_prec_b200 import fields
    kx, ky, kz = fields.field(model, seed)
    perm = str(tmp_path / "perm.bin")
    fields.write_perm_bin(perm, kx, ky, kz)
    cfg = str(tmp_path / "msplit.cfg")
    with open(cfg, "w") as f:
        f.write(O.msplit_cfg_text(elim_order=order, max_levels=max_levels))
    out = str(tmp_path / "out")
    r = O.run_ref(out, perm=perm, nx=nx, ny=ny, nz=nz, c=c, prec="msplit", cfg=cfg, eps=1e-8, timeout=600,
                  dump=True, ms_use_tails=tails)
    xr = np.fromfile(os.path.join(out, "x.f64"))
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, c, True)
    P = O.Prec(A, "msplit", q=(0.8,), niter=(5,), max_levels=max_levels, degree_max=2, order=order,
               use_tails=bool(tails))
    assert P.nlevels == r["nlevels"]
    levels = r["levels"] if isinstance(r["levels"], list) else json.loads(r["levels"])
    for l, ref in enumerate(levels):
        lv = P.level(l)
        for k in ("N", "nnz", "M", "Md"):
            assert lv[k] == ref[k], (l, k)
        if "map" in lv:
            assert np.array_equal(lv["map"], np.fromfile(os.path.join(out, f"l{l}_map.u32"), np.uint32)), l
    x, it, rel, rc = O.pcg(A, b, P, 1e-8)
    assert rc == 0 and it == r["niter"]
    assert np.array_equal(x, xr)
