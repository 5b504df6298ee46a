"""Python mirror of the reference's host interface for the hot path.

Names follow ml_prec: ``CSRMatrix`` (matrix.h:187-262), ``Config``
(project/config.h:54-86), ``ConfigFile`` key = value parsing
(modules/config_file/config_file.cc:68-142), ``MultiSplitPrec``
(multi_split_prec.h:105), ``Prec`` (uh_cheb, cheb_prec.h:115), ``PCGSolver``
(solvers.h:31-32) with ``SolverStats`` (solvers.h:15-28). Everything runs on
the GPU through the C ABI (include/mlp_b200.h); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import List, Optional

import numpy as np

from ._capi import (LevelInfo, PrecCfg, Stats, check, f64p, lib, ptr, u32p)

ORDERS = {"none": 0, "original": 1, "block": 2, "simple_1": 3}


class ConfigError(ValueError):
    pass


# ---------------------------------------------------------------------------
# ConfigFile (config_file.cc:68-142): "key = value" lines, '#' comments, values
# may continue on following lines that hold no delimiter; keys and values are
# trimmed; a repeated key overwrites the earlier one.
# ---------------------------------------------------------------------------
class ConfigFile:
    def __init__(self, filename: str, delimiter: str = "=", comment: str = "#",
                 sentry: str = "EndConfigFile"):
        if not os.path.exists(filename):
            raise FileNotFoundError(filename)
        self.contents = {}
        with open(filename) as f:
            lines = f.read().split("\n")
        i = 0
        n = len(lines)
        while i < n:
            line = lines[i].split(comment, 1)[0]
            i += 1
            if sentry and sentry in line:
                break
            if delimiter not in line:
                continue
            key, val = line.split(delimiter, 1)
            # continuation lines: no delimiter, not blank, not the sentry
            while i < n:
                nxt = lines[i]
                if nxt.strip() == "":
                    i += 1
                    break
                nxt = nxt.split(comment, 1)[0]
                if delimiter in nxt or (sentry and sentry in nxt):
                    break
                if nxt.strip():
                    val += "\n"
                val += nxt
                i += 1
            self.contents[key.strip()] = val.strip()

    def read(self, key, default):
        if key not in self.contents:
            return default
        v = self.contents[key]
        t = type(default)
        if t is str:
            return v
        if t is int:
            return int(v.split()[0])
        if t is float:
            return float(v.split()[0])
        return v


@dataclasses.dataclass
class Config:
    """project/config.h:54-86 (the fields the hot path reads); defaults of
    set_params (main_helper.cc:61-84)."""
    niters: List[int] = dataclasses.field(default_factory=lambda: [2])
    sigmas: List[float] = dataclasses.field(default_factory=lambda: [3.0])
    c: float = 1.0
    nx: int = 60
    ny: int = 220
    nz: int = 85
    use_tails: bool = True
    coarse_n: int = 0
    max_levels: int = 30
    prec_conf_file: str = ""
    fp32: bool = False  # reduced-precision hierarchy (this project's form (b))


def msplit_params(cfg: Config) -> dict:
    """MultiSplitPrec constructor parameter logic (multi_split_constr.cc:170-266).

    A config file overrides the command-line values (:179-180). Cases the
    reference leaves undefined are errors here: a missing config file (the
    reference continues with an empty q list, :230-232 then :256). Dynamic
    inner iterations (inner_iter = dynamic, level_eps) are capped on the device
    (the reference loops without a cap)."""
    if cfg.prec_conf_file:
        try:
            f = ConfigFile(cfg.prec_conf_file)
        except FileNotFoundError:
            raise ConfigError(f'Config file "{cfg.prec_conf_file}" is absent')
        qs = [float(t) for t in f.read("q", "0.8").split()]
        inner = f.read("inner_iter", "fixed")
        lu = f.read("lu_method", "exact")
        order = f.read("elim_order", "original")
        stop = f.read("elim_stop", "degree")
        coarse_n = f.read("coarse_n", 0)
        nlevels = f.read("max_levels", 15)
        level_eps = None
        if inner == "fixed":
            niters = [int(float(t)) for t in f.read("level_niter", "5").split()]
        elif inner == "dynamic":
            niters = [5]
            level_eps = [float(t) for t in f.read("level_eps", "1e-2").split()]
        else:
            raise ConfigError(f"Unknown inner_iter type: {inner}")
        if lu not in ("exact", "ilut"):
            raise ConfigError(f"Unknown lu type: {lu}")
        if order not in ORDERS:
            raise ConfigError(f"Unknown elim_order type: {order}")
        if stop == "degree":
            degree_max = f.read("degree_max", 3)
        elif stop == "goal":
            degree_max = 0  # level_ratio is read but never used (:225-226)
        else:
            raise ConfigError(f"Unknown elim_stop type: {stop}")
    else:
        level_eps = None
        qs = list(cfg.sigmas)
        niters = list(cfg.niters)
        order = "original" if cfg.use_tails else "none"
        coarse_n = cfg.coarse_n
        nlevels = cfg.max_levels
        degree_max = 3
        if any(q >= 1 for q in qs):
            raise ConfigError("All sigmas must be < 1")  # main_helper.cc:239-242
    if not qs:
        raise ConfigError("empty q list")
    return dict(q=qs, niter=niters, order=order, coarse_n=coarse_n, max_levels=nlevels,
                degree_max=degree_max, level_eps=level_eps, use_tails=cfg.use_tails)


class CSRMatrix:
    """Device-resident CSR matrix with the reference's layout (diagonal first)."""

    def __init__(self, handle, n, nnz):
        self.h = handle
        self.n = n
        self.nnz_ = nnz

    @classmethod
    def from_arrays(cls, ia, ja, a):
        ia = np.ascontiguousarray(ia, np.uint32)
        ja = np.ascontiguousarray(ja, np.uint32)
        a = np.ascontiguousarray(a, np.float64)
        h = C.c_void_p()
        check(lib().mlp_matrix_create(len(ia) - 1, ptr(ia, u32p), ptr(ja, u32p), ptr(a, f64p), C.byref(h)))
        return cls(h, len(ia) - 1, int(ia[-1]))

    @classmethod
    def spe(cls, nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True):
        """SPEMesh + construct_matrix on the device; returns (A, b)."""
        kx = np.ascontiguousarray(kx, np.float64)
        ky = np.ascontiguousarray(ky, np.float64)
        kz = np.ascontiguousarray(kz, np.float64)
        b = np.zeros(nx * ny * nz)
        h = C.c_void_p()
        check(lib().mlp_matrix_create_spe(nx, ny, nz, ptr(kx, f64p), ptr(ky, f64p), ptr(kz, f64p), c,
                                          int(dirichlet), C.byref(h), ptr(b, f64p)))
        n = C.c_uint32()
        z = C.c_uint32()
        check(lib().mlp_matrix_size(h, C.byref(n), C.byref(z)))
        return cls(h, n.value, z.value), b

    def size(self):
        return self.n

    def nnz(self):
        return self.nnz_

    def arrays(self):
        ia = np.empty(self.n + 1, np.uint32)
        ja = np.empty(self.nnz_, np.uint32)
        a = np.empty(self.nnz_)
        check(lib().mlp_matrix_download(self.h, ptr(ia, u32p), ptr(ja, u32p), ptr(a, f64p)))
        return ia, ja, a

    def __del__(self):
        if getattr(self, "h", None):
            lib().mlp_matrix_destroy(self.h)
            self.h = None


class PrecBase:
    """PrecBase::solve(f, x) (prec_base.h:8-12) on host numpy vectors."""

    h = None

    def solve(self, f, x=None):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f) if x is None else x
        check(lib().mlp_prec_apply_host(self.h, ptr(f, f64p), ptr(out, f64p)))
        return out

    @property
    def nlevels(self):
        n = C.c_uint32()
        check(lib().mlp_prec_nlevels(self.h, C.byref(n)))
        return n.value

    def level_info(self, l) -> dict:
        li = LevelInfo()
        check(lib().mlp_prec_level_info(self.h, l, C.byref(li)))
        return {k: getattr(li, k) for k, _ in LevelInfo._fields_}

    def level(self, l) -> dict:
        """Level data in the reference's indexing (map, L, U, A, dval)."""
        i = self.level_info(l)
        N, M, Md, nnz = i["N"], i["M"], i["Md"], i["nnz"]
        d = dict(i)
        Aia = np.empty(N + 1, np.uint32)
        Aja = np.empty(max(nnz, 1), np.uint32)
        Aa = np.empty(max(nnz, 1))
        if i["direct"]:
            check(lib().mlp_prec_level_export(self.h, l, None, None, None, None, None, None, None,
                                              ptr(Aia, u32p), ptr(Aja, u32p), ptr(Aa, f64p), None))
            d["A"] = (Aia, Aja[:nnz], Aa[:nnz])
            return d
        R = N - Md
        mp = np.empty(max(N, 1), np.uint32)
        Lia = np.empty(R + 1, np.uint32)
        Lja = np.empty(max(i["L_nnz"], 1), np.uint32)
        La = np.empty(max(i["L_nnz"], 1))
        Uia = np.empty(M + 1, np.uint32)
        Uja = np.empty(max(i["U_nnz"], 1), np.uint32)
        Ua = np.empty(max(i["U_nnz"], 1))
        dv = np.empty(max(Md, 1))
        check(lib().mlp_prec_level_export(self.h, l, ptr(mp, u32p), ptr(Lia, u32p), ptr(Lja, u32p), ptr(La, f64p),
                                          ptr(Uia, u32p), ptr(Uja, u32p), ptr(Ua, f64p), ptr(Aia, u32p),
                                          ptr(Aja, u32p), ptr(Aa, f64p), ptr(dv, f64p)))
        d["map"] = mp[:N]
        d["L"] = (Lia, Lja[:i["L_nnz"]], La[:i["L_nnz"]])
        d["U"] = (Uia, Uja[:i["U_nnz"]], Ua[:i["U_nnz"]])
        d["A"] = (Aia, Aja[:nnz], Aa[:nnz])
        d["dval"] = dv[:Md]
        return d

    def profile(self, reps=3):
        """Per launch of the apply: (name, mean ms, algorithmic bytes), timed
        launch by launch with CUDA events (mlp_prec_profile); run an apply
        first, the replay uses its input."""
        n = C.c_uint32()
        check(lib().mlp_prec_profile(self.h, reps, 0, C.byref(n), None, None, None, 0))
        cap = n.value
        ms = np.zeros(max(cap, 1))
        by = (C.c_uint64 * max(cap, 1))()
        names = C.create_string_buffer(64 * max(cap, 1))
        check(lib().mlp_prec_profile(self.h, reps, cap, C.byref(n), ptr(ms, f64p), by, names, 64))
        raw = names.raw
        return [(raw[64 * k:64 * (k + 1)].split(b"\0", 1)[0].decode(), float(ms[k]), int(by[k]))
                for k in range(cap)]

    def timeline(self, reps=5):
        """Per launch of the apply: (name, mean us inside the apply graph,
        algorithmic bytes), from %globaltimer stamps over reps back-to-back
        graph replays (mlp_prec_timeline); names and bytes as profile()."""
        prof = self.profile(1)
        n = C.c_uint32()
        us = np.zeros(max(len(prof), 1))
        check(lib().mlp_prec_timeline(self.h, reps, len(prof), C.byref(n), ptr(us, f64p)))
        if n.value != len(prof):
            raise RuntimeError("timeline and profile disagree on the number of launches")
        return [(nm, float(us[k]), by) for k, (nm, _, by) in enumerate(prof)]

    def pcg_timeline(self, A, b_dev, x_dev, eps=1e-8, flexible=False):
        """One device solve (torch CUDA tensors b_dev, x_dev) with the in-graph
        timeline on: per launch of one iteration near the end, (name, us)
        (mlp_pcg_timeline)."""
        cap = 4096
        n = C.c_uint32()
        us = np.zeros(cap)
        names = C.create_string_buffer(64 * cap)
        check(lib().mlp_pcg_timeline(A.h, C.c_void_p(b_dev.data_ptr()), self.h, C.c_void_p(x_dev.data_ptr()), eps,
                                     int(flexible), cap, C.byref(n), ptr(us, f64p), names, 64))
        raw = names.raw
        return [(raw[64 * k:64 * (k + 1)].split(b"\0", 1)[0].decode(), float(us[k])) for k in range(min(n.value, cap))]

    @property
    def bytes_per_apply(self):
        b = C.c_uint64()
        check(lib().mlp_prec_bytes_per_apply(self.h, C.byref(b)))
        return b.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().mlp_prec_destroy(self.h)
            self.h = None


def _make(A: CSRMatrix, kind, fp32=False, q=(0.8,), niter=(5,), coarse_n=0, max_levels=15, degree_max=2,
          order="simple_1", use_tails=True, sigma=(3.0,), ncheb=(2,), autotune=False, level_eps=None):
    qa = np.asarray(q, np.float64)
    na = np.asarray(niter, np.uint32)
    sa = np.asarray(sigma, np.float64)
    ca = np.asarray(ncheb, np.uint32)
    ea = np.asarray(level_eps if level_eps is not None else [], np.float64)
    cfg = PrecCfg(kind, len(qa), ptr(qa, f64p), len(na), ptr(na, u32p), coarse_n, max_levels, degree_max,
                  ORDERS[order] if isinstance(order, str) else order, int(use_tails),
                  len(sa), ptr(sa, f64p), len(ca), ptr(ca, u32p), int(fp32), int(autotune),
                  len(ea), ptr(ea, f64p) if len(ea) else None)
    h = C.c_void_p()
    check(lib().mlp_prec_create(A.h, C.byref(cfg), C.byref(h)))
    return h


class MultiSplitPrec(PrecBase):
    """MultiSplitPrec(A, cfg) (multi_split_prec.h:105) built on the GPU.

    Either pass a ``Config`` (msplit.cfg via ``prec_conf_file`` or the
    command-line fields) or the parameters directly as keywords."""

    def __init__(self, A: CSRMatrix, cfg: Optional[Config] = None, fp32: bool = False, **kw):
        if cfg is not None:
            p = msplit_params(cfg)
            fp32 = fp32 or cfg.fp32
            p.update(kw)
            kw = p
        self.A = A
        self.fp32 = fp32
        self.h = _make(A, 0, fp32=fp32, **kw)


class Prec(PrecBase):
    """uh_cheb Prec(A, cfg) (cheb_prec.h:115) built on the GPU: sigma (= beta)
    per level from Config.sigmas, Chebyshev degree from Config.niters."""

    def __init__(self, A: CSRMatrix, cfg: Optional[Config] = None, fp32: bool = False, **kw):
        if cfg is not None:
            if any(s <= 1 for s in cfg.sigmas):
                raise ConfigError("All sigmas must be > 1")
            kw.setdefault("sigma", tuple(cfg.sigmas))
            kw.setdefault("ncheb", tuple(cfg.niters))
            kw.setdefault("use_tails", cfg.use_tails)
            fp32 = fp32 or cfg.fp32
        self.A = A
        self.fp32 = fp32
        self.h = _make(A, 1, fp32=fp32, **kw)

    def lmin(self):
        """Lower spectral bound of level 0 (Prec::lmin, cheb_prec.h:121)."""
        return self.level_info(0)["lmin"]

    def lmax(self):
        """Upper spectral bound of level 0 (Prec::lmax, cheb_prec.h:122)."""
        return self.level_info(0)["lmax"]


class SymPrec(PrecBase):
    """SymPrec(A, cfg) (sym_prec.h:13-27) built on the GPU: the uh_cheb Prec of
    the symmetric part of A (a_ij = max(a_ij, a_ji) off the diagonal), applied
    as a PCG solve to 1e-14 (sym_prec.cc:8-40)."""

    def __init__(self, A: CSRMatrix, cfg: Optional[Config] = None, fp32: bool = False, **kw):
        if cfg is not None:
            if any(s <= 1 for s in cfg.sigmas):
                raise ConfigError("All sigmas must be > 1")
            kw.setdefault("sigma", tuple(cfg.sigmas))
            kw.setdefault("ncheb", tuple(cfg.niters))
            kw.setdefault("use_tails", cfg.use_tails)
            fp32 = fp32 or cfg.fp32
        self.A = A
        self.fp32 = fp32
        self.h = _make(A, 2, fp32=fp32, **kw)


@dataclasses.dataclass
class SolverStats:
    niter: int = 0
    napply: int = 0
    init_norm: float = 0.0
    final_norm: float = 0.0
    final_rel: float = 0.0
    t_sol: float = 0.0     # seconds (device time of the PCG call)
    t_const: float = 0.0   # seconds (device time of the preconditioner build)


def PCGSolver(A: CSRMatrix, b, B: PrecBase, x=None, stats: Optional[SolverStats] = None, eps: float = 1e-10,
              maxit: int = 0, flexible: Optional[bool] = None):
    """PCGSolver(A, b, B, x, stats, eps) (pcg.cc:8-102) with host vectors.

    flexible defaults to True for an FP32 hierarchy (Polak-Ribiere beta)."""
    b = np.ascontiguousarray(b, np.float64)
    out = np.empty_like(b) if x is None else x
    if flexible is None:
        flexible = bool(getattr(B, "fp32", False))
    st = Stats()
    check(lib().mlp_pcg(A.h, ptr(b, f64p), B.h, ptr(out, f64p), eps, maxit, int(flexible), C.byref(st)))
    if stats is not None:
        stats.niter = st.niter
        stats.napply = st.napply
        stats.init_norm = st.init_norm
        stats.final_norm = st.final_norm
        stats.final_rel = st.final_rel
        stats.t_sol = st.t_solve_ms / 1e3
        stats.t_const = st.t_setup_ms / 1e3
    return out


def ChebSolver(A: CSRMatrix, lmin: float, lmax: float, b, B: PrecBase, x=None,
               stats: Optional[SolverStats] = None, eps: float = 1e-10, maxit: int = 0):
    """ChebSolver(A, lmin, lmax, b, B, x, eps) (solvers.h:42-43, cheb.cc:9-100)
    with host vectors; lmin, lmax bound the spectrum of B A (uh_cheb's level-0
    bounds, Prec.lmin / Prec.lmax)."""
    b = np.ascontiguousarray(b, np.float64)
    out = np.empty_like(b) if x is None else x
    st = Stats()
    check(lib().mlp_cheb_solve(A.h, ptr(b, f64p), B.h, ptr(out, f64p), lmin, lmax, eps, maxit, C.byref(st)))
    if stats is not None:
        stats.niter = st.niter
        stats.napply = st.napply
        stats.init_norm = st.init_norm
        stats.final_norm = st.final_norm
        stats.final_rel = st.final_rel
        stats.t_sol = st.t_solve_ms / 1e3
        stats.t_const = st.t_setup_ms / 1e3
    return out


def generate_x0(n):
    x = np.empty(n)
    check(lib().mlp_generate_x0(ptr(x, f64p), n))
    return x
