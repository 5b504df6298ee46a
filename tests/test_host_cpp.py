"""The C++ host interface (ml_prec_b200/host/ml_prec.h) and its command-line
driver: the reference's types and calls (CSRMatrix, SkylineMatrix, Vector,
ConfigFile, Config, MultiSplitPrec(A, cfg), PCGSolver(A, b, B, x, stats, eps))
compiled into a C++ program.

CPU: host logic (config and command-line parsing, file formats, errors raised
before the device is used). GPU: a solve through the C++ interface and through
the driver, checked against the oracle (iterations within 1, solution within
1e-10 relative)."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ml_prec_b200", "lib")
BIN = os.path.join(ROOT, "tests", "host", "_bin", "host_api_test")
DRIVER = os.path.join(LIBDIR, "ml_prec_b200")
TOL = 1e-10


def _build():
    from ml_prec_b200 import build as B
    if not os.path.exists(B.LIB):
        pytest.skip("CUDA library not built")
    B.build_host()
    src = os.path.join(ROOT, "tests", "host", "host_api_test.cc")
    if not os.path.exists(BIN) or os.path.getmtime(BIN) < max(os.path.getmtime(src), os.path.getmtime(B.HOST_LIB)):
        os.makedirs(os.path.dirname(BIN), exist_ok=True)
        subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I" + B.HOST, "-I" + B.INCLUDE, src, "-o", BIN,
                        "-L" + LIBDIR, "-lml_prec_host", "-lmlp_b200", "-Wl,-rpath," + LIBDIR], check=True)
    return BIN


def test_host_logic(tmp_path):
    exe = _build()
    r = subprocess.run([exe, "cpu", str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


def test_reference_written_files_load(tmp_path):
    """The reference's own writers (csrmatrix.cc:302-355, vector.cc:18-49), run
    by the compiled reference driver, produce BINARY / ASCII / MatrixMarket
    matrix files and ASCII / BINARY vector files of a 16x22x8 problem; the C++
    host interface loads the matrices and the ASCII vector back to the
    reference's own raw arrays, reads the MatrixMarket file the reference itself
    cannot (it skips the size line as a comment, csrmatrix.cc:221-224), and
    refuses the reference's BINARY vector file, which holds only n * 4 of its
    n * 8 value bytes (vector.cc:42-46), with a message."""
    from ml_prec_b200 import fields
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference driver not built")
    exe = _build()
    kx, ky, kz = fields.field("iid", 1)
    perm = str(tmp_path / "perm.bin")
    fields.write_perm_bin(perm, kx, ky, kz)
    cfg = str(tmp_path / "msplit.cfg")
    with open(cfg, "w") as f:
        f.write(O.msplit_cfg_text())
    out = str(tmp_path / "ref")
    O.run_ref(out, perm=perm, nx=16, ny=22, nz=8, c=1.0, cfg=cfg, no_solve=True, dump=True, dump_formats=True,
              timeout=300)
    r = subprocess.run([exe, "ref-files", out], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


def test_driver_help():
    _build()
    r = subprocess.run([DRIVER, "-h"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "--prec-config-file" in r.stdout and "multi_split" in r.stdout


def _case(tmp_path, nx=30, ny=44, nz=12):
    from ml_prec_b200 import fields
    from oracle import oracle as O
    kx, ky, kz = fields.field("iid", 1)
    perm = str(tmp_path / "perm.bin")
    fields.write_perm_bin(perm, kx, ky, kz)
    cfg = str(tmp_path / "msplit.cfg")
    with open(cfg, "w") as f:
        f.write(O.msplit_cfg_text())
    return (nx, ny, nz), (kx, ky, kz), perm, cfg


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [0, 1])
def test_cpp_interface_solve_matches_oracle(tmp_path, fp32):
    from oracle import oracle as O
    exe = _build()
    (nx, ny, nz), (kx, ky, kz), perm, cfg = _case(tmp_path)
    out = str(tmp_path / "x.bin")
    r = subprocess.run([exe, "solve", str(nx), str(ny), str(nz), perm, cfg, "1e-8", str(fp32), out],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"niter (\d+) rel (\S+)", r.stdout)
    niter, rel = int(m.group(1)), float(m.group(2))
    raw = open(out, "rb").read()
    n = np.frombuffer(raw[:4], np.uint32)[0]
    x = np.frombuffer(raw[4:], np.float64)
    assert n == nx * ny * nz and x.size == n
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True)
    P = O.Prec(A, "msplit", q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="simple_1")
    xo, it, rel_o, rc = O.pcg(A, b, P, eps=1e-8)
    assert rc == 0 and rel <= 1e-8
    if fp32:
        # FP32-stored hierarchy: the same residual tolerance; two solutions with
        # relative residual 1e-8 differ by up to cond(A) * 1e-8 (about 1e-5 here)
        assert np.linalg.norm(x - xo) <= 1e-4 * np.linalg.norm(xo)
    else:
        assert abs(niter - it) <= 1
        assert np.linalg.norm(x - xo) <= TOL * np.linalg.norm(xo)


@pytest.mark.gpu
def test_driver_runs_config_file(tmp_path):
    from oracle import oracle as O
    _build()
    (nx, ny, nz), (kx, ky, kz), perm, cfg = _case(tmp_path)
    with open(tmp_path / "default.properties", "w") as f:
        f.write("log4j.rootLogger=all, R\nlog4j.appender.R.File=trace.log\n")
    r = subprocess.run([DRIVER, "-p", "multi_split", "-C", cfg, "-x", str(nx), "-y", str(ny), "-z", str(nz),
                        "--perm", perm, "--dirichlet", "--eps", "1e-8", "-a", "2", "--dir", str(tmp_path / "res")],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    it = int(re.search(r"Number of iterations : (\d+)", r.stdout).group(1))
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True)
    P = O.Prec(A, "msplit", q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="simple_1")
    _, it_o, _, _ = O.pcg(A, b, P, eps=1e-8)
    assert abs(it - it_o) <= 1
    log = open(tmp_path / "res" / "trace.log").read()
    assert "Number of iterations" in log and "Level 0:" in log


@pytest.mark.gpu
def test_driver_runs_uh_cheb(tmp_path):
    """The driver's -p uh_cheb path (Prec(A, cfg) from the command line: sigma
    3, Chebyshev degree 4) reaches the oracle's iteration count within 1."""
    from oracle import oracle as O
    _build()
    (nx, ny, nz), (kx, ky, kz), perm, _ = _case(tmp_path, 20, 22, 8)
    r = subprocess.run([DRIVER, "-p", "uh_cheb", "-s", "3", "-b", "4", "-x", str(nx), "-y", str(ny), "-z", str(nz),
                        "--perm", perm, "--dirichlet", "--eps", "1e-8"],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    it = int(re.search(r"Number of iterations : (\d+)", r.stdout).group(1))
    A, b = O.assemble(nx, ny, nz, kx, ky, kz, c=1.0, dirichlet=True)
    P = O.Prec(A, "cheb", sigma=(3.0,), ncheb=(4,), use_tails=True)
    _, it_o, _, rc = O.pcg(A, b, P, eps=1e-8)
    assert rc == 0 and abs(it - it_o) <= 1
