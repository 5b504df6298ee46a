"""ctypes binding of the CPU restatement (oracle/mlp_oracle.c) and a runner for the
compiled reference driver (oracle/_ref/ref_driver).

TEST INFRASTRUCTURE ONLY: imported by tests/, tests/golden/make_golden.py,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, where it is the checker.
The product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmlp_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

u32p = C.POINTER(C.c_uint32)
f64p = C.POINTER(C.c_double)


class CSR(C.Structure):
    _fields_ = [("nrow", C.c_uint32), ("ncol", C.c_uint32), ("ia", u32p), ("ja", u32p), ("a", f64p)]


class PrecCfg(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("nq", C.c_uint32), ("q", f64p),
        ("nnit", C.c_uint32), ("niter", u32p),
        ("coarse_n", C.c_uint32), ("max_levels", C.c_uint32), ("degree_max", C.c_uint32),
        ("order", C.c_int), ("use_tails", C.c_int),
        ("nsig", C.c_uint32), ("sigma", f64p),
        ("nch", C.c_uint32), ("ncheb", u32p),
        ("neps", C.c_uint32), ("level_eps", f64p),
    ]


class Level(C.Structure):
    _fields_ = [
        ("N", C.c_uint32), ("nnz", C.c_uint32), ("M", C.c_uint32), ("Md", C.c_uint32),
        ("niter", C.c_uint32), ("q", C.c_double), ("eps", C.c_double),
        ("A", CSR), ("L", CSR), ("U", CSR),
        ("map", u32p), ("rmap", u32p), ("dval", f64p),
        ("alpha", C.c_double), ("beta", C.c_double), ("lmin", C.c_double), ("lmax", C.c_double),
        ("ncheb", C.c_uint32), ("lu", f64p),
    ]


ORDERS = {"none": 0, "original": 1, "block": 2, "simple_1": 3}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = C.CDLL(LIB_PATH)
        L.or_assemble.argtypes = [C.c_uint32] * 3 + [f64p] * 3 + [C.c_double, C.c_int, C.POINTER(CSR), f64p]
        L.or_spmv.argtypes = [C.POINTER(CSR), f64p, f64p]
        L.or_generate_x0.argtypes = [f64p, C.c_uint32]
        L.or_prec_build.argtypes = [C.POINTER(CSR), C.POINTER(PrecCfg), C.c_char_p, C.c_int]
        L.or_prec_build.restype = C.c_void_p
        L.or_prec_apply.argtypes = [C.c_void_p, f64p, f64p]
        L.or_prec_free.argtypes = [C.c_void_p]
        L.or_prec_nlevels.argtypes = [C.c_void_p]
        L.or_prec_nlevels.restype = C.c_uint32
        L.or_prec_level.argtypes = [C.c_void_p, C.c_uint32]
        L.or_prec_level.restype = C.POINTER(Level)
        L.or_pcg.argtypes = [C.POINTER(CSR), f64p, C.c_void_p, f64p, C.c_double,
                             C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.c_uint32]
        L.or_csr_free.argtypes = [C.POINTER(CSR)]
        L.or_pcg_ex.argtypes = [C.POINTER(CSR), f64p, C.c_void_p, f64p, C.c_double,
                                C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.c_uint32, C.c_int]
        L.or_grad_logk.argtypes = [C.c_uint32] * 3 + [f64p] * 3 + [C.c_int, f64p, f64p, f64p]
        L.or_cheb_solve.argtypes = [C.POINTER(CSR), f64p, C.c_void_p, C.c_double, C.c_double, f64p, C.c_double,
                                    C.POINTER(C.c_uint32), C.POINTER(C.c_double), C.c_uint32]
        L.or_cheb.argtypes = [C.c_double, C.c_uint32]
        L.or_cheb.restype = C.c_double
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


class Matrix:
    """numpy-backed CSR (diagonal-first rows) with a ctypes view."""

    def __init__(self, ia, ja, a, ncol=None):
        self.ia = np.ascontiguousarray(ia, np.uint32)
        self.ja = np.ascontiguousarray(ja, np.uint32)
        self.a = np.ascontiguousarray(a, np.float64)
        self.n = len(self.ia) - 1
        self.ncol = self.n if ncol is None else ncol
        self._c = CSR(self.n, self.ncol, _p(self.ia, u32p), _p(self.ja, u32p), _p(self.a, f64p))

    @property
    def c(self):
        return C.byref(self._c)

    @property
    def nnz(self):
        return int(self.ia[-1])


def _csr_to_numpy(c: CSR):
    nr = c.nrow
    if not c.ia:
        return np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0)
    ia = np.ctypeslib.as_array(c.ia, shape=(nr + 1,)).copy()
    nnz = int(ia[-1])
    if nnz == 0:
        return ia, np.zeros(0, np.uint32), np.zeros(0)
    ja = np.ctypeslib.as_array(c.ja, shape=(nnz,)).copy()
    a = np.ctypeslib.as_array(c.a, shape=(nnz,)).copy()
    return ia, ja, a


def assemble(nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True):
    L = lib()
    kx = np.ascontiguousarray(kx, np.float64)
    ky = np.ascontiguousarray(ky, np.float64)
    kz = np.ascontiguousarray(kz, np.float64)
    N = nx * ny * nz
    b = np.zeros(N)
    cs = CSR()
    L.or_assemble(nx, ny, nz, _p(kx, f64p), _p(ky, f64p), _p(kz, f64p), c, int(dirichlet), C.byref(cs), _p(b, f64p))
    ia, ja, a = _csr_to_numpy(cs)
    L.or_csr_free(C.byref(cs))
    return Matrix(ia, ja, a), b


def generate_x0(n):
    x = np.empty(n)
    lib().or_generate_x0(_p(x, f64p), n)
    return x


def spmv(A: Matrix, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(A.n)
    lib().or_spmv(A.c, _p(x, f64p), _p(y, f64p))
    return y


def cheb(x, k):
    return lib().or_cheb(x, k)


class Prec:
    """Oracle preconditioner (multi-split or uh_cheb)."""

    def __init__(self, A: Matrix, kind="msplit", q=(0.8,), niter=(5,), coarse_n=0, max_levels=15,
                 degree_max=2, order="simple_1", use_tails=True, sigma=(3.0,), ncheb=(2,), level_eps=None):
        """level_eps: per-level eps of msplit.cfg inner_iter = dynamic (index 0
        ignored, the last repeats); None keeps the fixed niter."""
        self._keep = []
        qa = np.asarray(q, np.float64); na = np.asarray(niter, np.uint32)
        sa = np.asarray(sigma, np.float64); ca = np.asarray(ncheb, np.uint32)
        ea = np.asarray(level_eps if level_eps is not None else [], np.float64)
        self._keep += [qa, na, sa, ca, ea, A]
        cfg = PrecCfg({"msplit": 0, "cheb": 1, "sym": 2}[kind], len(qa), _p(qa, f64p), len(na), _p(na, u32p),
                      coarse_n, max_levels, degree_max, ORDERS[order], int(use_tails),
                      len(sa), _p(sa, f64p), len(ca), _p(ca, u32p), len(ea), _p(ea, f64p) if len(ea) else None)
        err = C.create_string_buffer(256)
        self.h = lib().or_prec_build(A.c, C.byref(cfg), err, 256)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.kind = kind
        self.n = A.n

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_prec_free(self.h)
            self.h = None

    @property
    def nlevels(self):
        return lib().or_prec_nlevels(self.h)

    def level(self, l):
        lv = lib().or_prec_level(self.h, l).contents
        d = dict(N=lv.N, nnz=lv.nnz, M=lv.M, Md=lv.Md, niter=lv.niter, q=lv.q, eps=lv.eps,
                 alpha=lv.alpha, beta=lv.beta, lmin=lv.lmin, lmax=lv.lmax, ncheb=lv.ncheb)
        d["A"] = _csr_to_numpy(lv.A)
        if l < self.nlevels and lv.map:
            d["L"] = _csr_to_numpy(lv.L)
            d["U"] = _csr_to_numpy(lv.U)
            d["map"] = np.ctypeslib.as_array(lv.map, shape=(lv.N,)).copy() if lv.N else np.zeros(0, np.uint32)
            d["dval"] = np.ctypeslib.as_array(lv.dval, shape=(lv.Md,)).copy() if lv.Md else np.zeros(0)
        return d

    def apply(self, f):
        f = np.ascontiguousarray(f, np.float64)
        x = np.zeros(self.n)
        lib().or_prec_apply(self.h, _p(f, f64p), _p(x, f64p))
        return x


def pcg(A: Matrix, b, P: Prec, eps=1e-8, maxit=0, x0_zero=False):
    """PCGSolver restated; returns (x, niter, final_rel, rc). rc -3: cap reached."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    it = C.c_uint32(0)
    rel = C.c_double(0)
    rc = lib().or_pcg_ex(A.c, _p(b, f64p), P.h, _p(x, f64p), eps, C.byref(it), C.byref(rel), maxit,
                         1 if x0_zero else 0)
    return x, it.value, rel.value, rc


def cheb_solve(A: Matrix, b, P: Prec, lmin, lmax, eps=1e-8, maxit=0):
    """ChebSolver restated; returns (x, niter, final_rel, rc). rc -3: cap reached."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    it = C.c_uint32(0)
    rel = C.c_double(0)
    rc = lib().or_cheb_solve(A.c, _p(b, f64p), P.h, lmin, lmax, _p(x, f64p), eps, C.byref(it), C.byref(rel), maxit)
    return x, it.value, rel.value, rc


def grad_logk(nx, ny, nz, kx, ky, kz, p, lam, dirichlet=True):
    """CPU FP64 dJ/d(ln K) per cell (differentiation form)."""
    kx, ky, kz, p, lam = (np.ascontiguousarray(v, np.float64) for v in (kx, ky, kz, p, lam))
    g = np.empty(nx * ny * nz)
    lib().or_grad_logk(nx, ny, nz, _p(kx, f64p), _p(ky, f64p), _p(kz, f64p), int(dirichlet), _p(p, f64p),
                       _p(lam, f64p), _p(g, f64p))
    return g


# ---- reference driver -------------------------------------------------------

def read_csr(fn):
    """Reference BINARY CSR (csrmatrix.cc:174-190)."""
    b = open(fn, "rb").read()
    nr, nc = np.frombuffer(b[:8], np.uint32)
    ia = np.frombuffer(b[8:8 + 4 * (nr + 1)], np.uint32).copy()
    nnz = int(ia[-1])
    o = 8 + 4 * (nr + 1)
    ja = np.frombuffer(b[o:o + 4 * nnz], np.uint32).copy()
    a = np.frombuffer(b[o + 4 * nnz:o + 12 * nnz], np.float64).copy()
    return int(nr), int(nc), ia, ja, a


def write_csr(fn, ia, ja, a, ncol=None):
    nr = len(ia) - 1
    with open(fn, "wb") as f:
        f.write(np.array([nr, nr if ncol is None else ncol], np.uint32).tobytes())
        f.write(np.asarray(ia, np.uint32).tobytes())
        f.write(np.asarray(ja, np.uint32).tobytes())
        f.write(np.asarray(a, np.float64).tobytes())


def ref_available():
    return os.path.exists(REF_DRIVER)


def run_ref(outdir, *, perm=None, csr=None, rhs=None, nx=60, ny=220, nz=85, c=1.0, prec="msplit",
            cfg=None, eps=1e-8, dump=False, no_solve=False, sigmas=None, niters=None, apply=None,
            reps=1, dirichlet=True, timeout=None, ms_use_tails=None, solver=None, dump_formats=False):
    """Runs oracle/_ref/ref_driver; returns the parsed result.json."""
    args = [REF_DRIVER, "--out", outdir, "--nx", str(nx), "--ny", str(ny), "--nz", str(nz),
            "--c", repr(float(c)), "--prec", prec, "--eps", repr(float(eps)), "--reps", str(reps)]
    if perm is not None:
        args += ["--perm", perm]
    if csr is not None:
        args += ["--csr", csr]
    if rhs is not None:
        args += ["--rhs", rhs]
    if cfg is not None:
        args += ["--cfg", cfg]
    if dump:
        args += ["--dump"]
    if no_solve:
        args += ["--no-solve"]
    if not dirichlet:
        args += ["--no-dirichlet"]
    if sigmas is not None:
        args += ["--sigmas", ",".join(repr(float(s)) for s in sigmas)]
    if niters is not None:
        args += ["--niters", ",".join(str(int(s)) for s in niters)]
    if apply is not None:
        args += ["--apply", apply]
    if ms_use_tails is not None:
        args += ["--ms-use-tails", str(int(ms_use_tails))]
    if solver is not None:
        args += ["--solver", solver]
    if dump_formats:
        args += ["--dump-formats"]
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "log.txt"), "w") as log:
        subprocess.run(args, check=True, stdout=log, timeout=timeout)
    with open(os.path.join(outdir, "result.json")) as f:
        res = json.load(f)
    if solver == "cheb":
        # ChebSolver's last log line: "#<steps>: relative -> ..." (cheb.cc:86-93)
        import re
        steps = re.findall(r"#(\d+): relative", open(os.path.join(outdir, "log.txt")).read())
        res["niter"] = int(steps[-1])
    return res


def msplit_cfg_text(q="0.8", level_niter="5", elim_order="simple_1", degree_max=2, coarse_n=0,
                    max_levels=15, level_eps=None):
    """An msplit.cfg in the reference's key = value format (project/msplit.cfg);
    level_eps (a string of per-level values) selects inner_iter = dynamic."""
    inner = (f"inner_iter = dynamic\nlevel_eps = {level_eps}\n" if level_eps is not None
             else f"inner_iter = fixed\nlevel_niter = {level_niter}\n")
    return (f"q = {q}\n{inner}lu_method = exact\n"
            f"elim_order = {elim_order}\nelim_stop = degree\ndegree_max = {degree_max}\n"
            f"coarse_n = {coarse_n}\nmax_levels = {max_levels}\n")
