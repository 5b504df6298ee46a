"""Writes the golden fixtures of tests/golden/ by running the reference itself.

The reference (ml_prec) is compiled from its own sources by `make -C oracle ref`
into oracle/_ref/ref_driver (a driver of this project linked against the
unmodified reference objects). For each case below the driver builds the
matrix with SPEMesh::construct_matrix from a seeded synthetic field, constructs
the preconditioner, runs one preconditioner apply on a seeded vector and a PCG
solve, and dumps the hierarchy. This script stores the inputs and those outputs
as compressed .npz files. It needs the reference sources (REF below) and is run
only when the fixtures are regenerated; the tests read the .npz files.

    python tests/golden/make_golden.py [case ...]   # all cases by default
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ml_prec_b200 import fields  # noqa: E402
from oracle import oracle as O  # noqa: E402

# the reference tree: MLP_REF_SRC, else the `reference` tree beside this repository
REF = os.environ.get("MLP_REF_SRC", os.path.join(os.path.dirname(ROOT), "reference"))
OUT = os.path.dirname(os.path.abspath(__file__))

# name: (field model, field seed, nx, ny, nz, c, prec, options)
CASES = {
    "ms_iid_12x22x6": ("iid", 1, 12, 22, 6, 1.0, "msplit", {}),
    "ms_layered_16x22x8_c01": ("layered", 2, 16, 22, 8, 0.1, "msplit", {}),
    "ms_direct_20x22x6": ("iid", 3, 20, 22, 6, 1.0, "msplit", {"max_levels": 2}),
    "ms_deg1_12x22x6": ("iid", 5, 12, 22, 6, 1.0, "msplit", {"degree_max": 1, "level_niter": "3 4"}),
    "ms_tiny_1x1x1": ("iid", 1, 1, 1, 1, 1.0, "msplit", {}),
    "ms_line_1x1x7": ("iid", 1, 1, 1, 7, 1.0, "msplit", {}),
    "ms_none_12x22x6": ("iid", 1, 12, 22, 6, 1.0, "msplit", {"elim_order": "none", "max_levels": 3}),
    "ms_original_16x22x8": ("layered", 2, 16, 22, 8, 1.0, "msplit", {"elim_order": "original", "use_tails": 1}),
    "ms_original_notails_20x22x10": ("iid", 6, 20, 22, 10, 1.0, "msplit",
                                     {"elim_order": "original", "use_tails": 0}),
    "ms_dynamic_16x22x8_c01": ("layered", 2, 16, 22, 8, 0.1, "msplit", {"level_eps": "0 1e-2"}),
    "ms_dynamic_12x22x6": ("iid", 1, 12, 22, 6, 1.0, "msplit", {"level_eps": "0 1e-1 1e-3"}),
    "ch_layered_16x22x8": ("layered", 2, 16, 22, 8, 1.0, "cheb", {"sigmas": [3.0], "niters": [4]}),
    "ch_iid_12x22x6": ("iid", 4, 12, 22, 6, 1.0, "cheb", {"sigmas": [3.0, 2.5], "niters": [2, 3]}),
    # SymPrec (sym_prec.cc): uh_cheb of the symmetric part applied as a PCG solve to 1e-14
    "sym_layered_16x22x8": ("layered", 2, 16, 22, 8, 1.0, "sym", {"sigmas": [3.0], "niters": [4]}),
    # the same preconditioner with ChebSolver as the outer iteration (x, niter are ChebSolver's)
    "chs_layered_16x22x8": ("layered", 2, 16, 22, 8, 1.0, "cheb", {"sigmas": [3.0], "niters": [4], "solver": "cheb"}),
}

# Configurations the reference rejects while it builds the hierarchy: the
# message of its exception is stored (name.json) and the library must fail
# with the same message. elim_order = block accepts only the 60x220x85 mesh,
# so it fails on any other mesh at level 0 and on every mesh at level 1
# (multi_split_mark.cc:201-203); the size in the level-1 message is what
# level 0 left over, which pins the level-0 block ordering's M + Md.
ERRORS = {
    "err_block_60x220x85": ("layered", 2, 60, 220, 85, 1.0, {"elim_order": "block"}),
    "err_block_16x22x8": ("layered", 2, 16, 22, 8, 1.0, {"elim_order": "block"}),
}


def run_errors(td, wanted):
    import re
    for name, (model, seed, nx, ny, nz, c, opt) in ERRORS.items():
        if name not in wanted:
            continue
        kx, ky, kz = fields.field(model, seed)
        od = os.path.join(td, name)
        os.makedirs(od)
        fn = os.path.join(od, "perm.bin")
        fields.write_perm_bin(fn, kx, ky, kz)
        cfg = os.path.join(od, "msplit.cfg")
        with open(cfg, "w") as fh:
            fh.write(O.msplit_cfg_text(elim_order=opt["elim_order"]))
        r = subprocess.run([O.REF_DRIVER, "--out", od, "--perm", fn, "--nx", str(nx), "--ny", str(ny), "--nz",
                            str(nz), "--c", repr(float(c)), "--prec", "msplit", "--cfg", cfg, "--no-solve"],
                           capture_output=True, text=True)
        assert r.returncode != 0, f"{name}: the reference accepted the configuration"
        m = re.search(r"EXCEPTION \(([^)]*)\): (.*)", r.stderr)
        assert m, r.stderr[-2000:]
        where = m.group(1).replace(os.path.join(REF, ""), "")
        rec = dict(model=model, seed=seed, nx=nx, ny=ny, nz=nz, c=c, options=opt, where=where,
                   message=m.group(2).strip())
        with open(os.path.join(OUT, f"{name}.json"), "w") as fh:
            json.dump(rec, fh, indent=1)
        print(name, rec["message"], flush=True)


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    with tempfile.TemporaryDirectory() as td:
        perms = {}
        wanted = sys.argv[1:] or list(CASES) + list(ERRORS)
        run_errors(td, wanted)
        for name, (model, seed, nx, ny, nz, c, prec, opt) in CASES.items():
            if name not in wanted:
                continue
            key = (model, seed)
            if key not in perms:
                kx, ky, kz = fields.field(model, seed)
                fn = os.path.join(td, f"perm_{model}_{seed}.bin")
                fields.write_perm_bin(fn, kx, ky, kz)
                perms[key] = fn
            od = os.path.join(td, name)
            os.makedirs(od)
            N = nx * ny * nz
            f = np.random.default_rng(1234).standard_normal(N)
            f.tofile(os.path.join(od, "f_in.f64"))
            kw = {}
            if prec == "msplit":
                cfg = os.path.join(od, "msplit.cfg")
                with open(cfg, "w") as fh:
                    fh.write(O.msplit_cfg_text(level_niter=opt.get("level_niter", "5"),
                                               elim_order=opt.get("elim_order", "simple_1"),
                                               degree_max=opt.get("degree_max", 2),
                                               max_levels=opt.get("max_levels", 15),
                                               level_eps=opt.get("level_eps")))
                kw["cfg"] = cfg
                if "use_tails" in opt:
                    # MultiSplitPrec reads use_tails without setting it (multi_split_prec.h:17);
                    # the driver pins it for the case
                    kw["ms_use_tails"] = opt["use_tails"]
            else:
                kw["sigmas"] = opt["sigmas"]
                kw["niters"] = opt["niters"]
                if "solver" in opt:
                    kw["solver"] = opt["solver"]
            res = O.run_ref(od, perm=perms[key], nx=nx, ny=ny, nz=nz, c=c, prec=prec, eps=1e-8, dump=True,
                            apply=os.path.join(od, "f_in.f64"), **kw)
            _, _, ia, ja, a = O.read_csr(os.path.join(od, "A0.csr"))
            d = dict(nx=nx, ny=ny, nz=nz, c=c, model=model, seed=seed, prec=prec,
                     options=json.dumps(opt), A_ia=ia, A_ja=ja, A_a=a,
                     b=np.fromfile(os.path.join(od, "b.f64")), f_in=f,
                     apply_out=np.fromfile(os.path.join(od, "apply_out.f64")),
                     x=np.fromfile(os.path.join(od, "x.f64")), niter=res["niter"],
                     nlevels=res["nlevels"], levels=json.dumps(res["levels"]))
            for l in range(res["nlevels"]):
                p = lambda s: os.path.join(od, f"l{l}_{s}")
                if os.path.exists(p("map.u32")):
                    d[f"l{l}_map"] = np.fromfile(p("map.u32"), np.uint32)
                    d[f"l{l}_dval"] = np.fromfile(p("dval.f64"))
                    for m in ("L", "U"):
                        _, _, i2, j2, a2 = O.read_csr(p(f"{m}.csr"))
                        d[f"l{l}_{m}_ia"], d[f"l{l}_{m}_ja"], d[f"l{l}_{m}_a"] = i2, j2, a2
                if l > 0:
                    _, _, i2, j2, a2 = O.read_csr(p("A.csr"))
                    d[f"l{l}_A_ia"], d[f"l{l}_A_ja"], d[f"l{l}_A_a"] = i2, j2, a2
            np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **d)
            print(name, "N", N, "levels", res["nlevels"], "niter", res["niter"], flush=True)


if __name__ == "__main__":
    main()
