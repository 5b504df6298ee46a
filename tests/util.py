"""Helpers shared by the tests: golden fixtures and oracle configurations."""
import json
import os

import numpy as np

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_golden(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    d["options"] = json.loads(str(d["options"]))
    d["levels"] = json.loads(str(d["levels"]))
    d["prec"] = str(d["prec"])
    return d


def prec_kwargs(g):
    """Keyword arguments of the preconditioner a golden case was made with."""
    o = g["options"]
    if g["prec"] == "msplit":
        return dict(kind="msplit", q=(0.8,), niter=tuple(int(t) for t in str(o.get("level_niter", "5")).split()),
                    max_levels=o.get("max_levels", 15), degree_max=o.get("degree_max", 2),
                    order=o.get("elim_order", "simple_1"), use_tails=bool(o.get("use_tails", 1)),
                    level_eps=(tuple(float(t) for t in o["level_eps"].split()) if "level_eps" in o else None))
    return dict(kind=g["prec"], sigma=tuple(o["sigmas"]), ncheb=tuple(o["niters"]), use_tails=True)


def oracle_prec(A, g):
    kw = prec_kwargs(g)
    kind = kw.pop("kind")
    return O.Prec(A, kind, **kw)


def gpu_prec(A, g, fp32=False):
    import ml_prec_b200 as M
    kw = prec_kwargs(g)
    kind = kw.pop("kind")
    if kind == "msplit":
        return M.MultiSplitPrec(A, fp32=fp32, **kw)
    if kind == "sym":
        return M.SymPrec(A, fp32=fp32, **kw)
    return M.Prec(A, fp32=fp32, **kw)
