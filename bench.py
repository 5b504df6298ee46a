"""Benchmark: seconds to relative residual 1e-8 on the 60x220x85 (1,122,000-cell)
reservoir-pressure problem, multi-split preconditioned CG on B200.

Workload (one "step"): build the multi-split hierarchy on the device from the
matrix already resident in HBM (marking, ordering, Schur elimination, solve
operators, apply graph), then PCG from generate_x0's start vector to
||r||/||r0|| <= 1e-8 (one graph launch). Problem: seeded synthetic layered
permeability field (smooth layers 1-35, channelised layers 36-85, ky = kx,
kz = 0.1 kx) standing in for SPE10, the reference stencil with c = 1 and
Dirichlet x-faces; msplit.cfg parameters (q = 0.8, simple_1, degree_max = 2,
level_niter = 5, max_levels = 15).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line. `value`: device-timed seconds per step of the
FP64 path, max over ranks (every rank solves its own replica; no data-path
collective; "weak" scaling). `e2e`: the same step through the C ABI with host
buffers (matrix and right-hand side uploaded, solution downloaded), host-timed.
`forms`: the FP64 step with launch shapes from the build-time autotuner, the
c = 0.1 problem, the uh_cheb preconditioner (sigma 3, degree 4) on the same
matrix, the FP32-stored hierarchy inside flexible FP64 PCG (time with fixed and tuned
shapes, accuracy against a tight FP64 solve), the adjoint gradient (time
against one forward solve), and the 64-realization ensemble solved in one
graph launch per rank (sharded over ranks). `roofline`: the level-0 CSR SpMV
(pipelined tile kernel), 50 graph-recorded launches over two alternating
matrix copies, with the DRAM traffic of an ncu capture. `cpu_baseline`: the
reference itself (oracle/_ref, single-threaded) on the same problem (and on
the c = 0.1 and uh_cheb forms).
`--no-forms` and `--no-cpu-baseline` leave out those extra measurements (the
profiling runs use them); the timed steps are the same.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

_T0 = time.perf_counter()


def progress(msg):
    """One line per finished phase on stderr (the JSON line stays on stdout)."""
    print(f"[bench +{time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to rel-res 1e-8 @1.1M cells (multi-split PCG, 60x220x85)"
UNIT = "s"
NX, NY, NZ, C_REACT, SEED = 60, 220, 85, 1.0, 2
EPS = 1e-8
MSPLIT = dict(q=(0.8,), niter=(5,), max_levels=15, degree_max=2, order="simple_1")
# uh_cheb as `ml_prec -p uh_cheb -s 3 -b 4` runs it: sigma 3, Chebyshev degree 4
UH_CHEB = dict(sigma=(3.0,), ncheb=(4,), use_tails=True)
# DRAM bytes of one level-0 SpMV launch on this matrix from an ncu capture
# (106.84 MB read + 4.79 MB written): the matrix and x stream once; part of y
# is still in L2 when the kernel ends.
SPMV_DRAM_TRAFFIC = 111.63e6
# DRAM bytes (read + write) of one launch of the folded level-2 phase 2
# (k_phase2_fold) on this matrix, from the ncu capture summarised in
# profiles/phase2_fold_level2_60x220x85.md (cold caches: in the graph its
# operators stay in L2). Not measured in the run.
FOLD_DRAM_TRAFFIC = {"phase2_fold L2": 4.42e6}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """Samples SM clocks and throttle reasons (nvidia-smi, every 200 ms)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.proc = None

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        try:
            for line in open(self.path):
                f = [t.strip() for t in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
            os.unlink(self.path)
        except (OSError, TypeError):
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(values):
    """Every rank's timings, reduced with MAX over the ranks (each reported
    time is the slowest rank's); the identity on one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def flush_l2(buf):
    buf.fill_(1.0)  # 256 MB write, larger than the 126 MB L2


def run_ours(args, ws, rank, local):
    import torch
    import ml_prec_b200 as M
    from ml_prec_b200 import adjoint, ensemble, fields
    from ml_prec_b200._capi import Stats, check, lib

    torch.cuda.set_device(local)
    check(lib().mlp_set_device(local))
    kx, ky, kz = fields.field("layered", SEED)
    A, b = M.CSRMatrix.spe(NX, NY, NZ, kx, ky, kz, c=C_REACT, dirichlet=True)
    N = A.n
    dev = torch.device("cuda", local)
    b_d = torch.from_numpy(b).to(dev)
    x_d = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    barrier = (lambda: torch.distributed.barrier()) if ws > 1 else (lambda: None)

    def solve(P, fp32, eps=EPS, maxit=0):
        st = Stats()
        rc = lib().mlp_pcg_device(A.h, C.c_void_p(b_d.data_ptr()), P.h, C.c_void_p(x_d.data_ptr()), eps, maxit,
                                  int(fp32), C.byref(st), C.c_void_p(stream.cuda_stream))
        if rc != 0 and not (maxit and rc == 6):  # 6: the cap a caller asked for
            check(rc)
        return st

    def timed(fp32, K, tag=None, autotune=False):
        """K steps (setup + solve), each timed with events on the solve stream;
        the handle is released after the step's end event."""
        times, last = [], None
        for k in range(K):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if tag and k == 0:
                torch.cuda.nvtx.range_push(tag)
            e0.record(stream)
            P = M.MultiSplitPrec(A, fp32=fp32, autotune=autotune, **MSPLIT)
            st = solve(P, fp32)
            e1.record(stream)
            if tag and k == 0:
                torch.cuda.nvtx.range_pop()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            last = (st, P.bytes_per_apply)
            del P
        return times, last

    def launches():
        c = C.c_uint64()
        check(lib().mlp_launch_count(C.byref(c)))
        return c.value

    # the clock sampler starts before the warm-up so that its start-up is over
    # when the timed region begins
    clk = Clocks(local)
    clk.start()
    time.sleep(3.0)
    timed(False, args.warmup)
    barrier()
    torch.cuda.synchronize()
    l0 = launches()
    t64, (st64, nb64) = timed(False, args.steps, tag="bench_step")
    torch.cuda.synchronize()
    nlaunch = launches() - l0
    barrier()
    clk.stop()
    clocks = clk.summary()
    progress("timed FP64 steps")

    out = dict(t64=t64, st64=st64, nb64=nb64, nlaunch=nlaunch, clocks=clocks, N=N, nnz=A.nnz())
    if not args.no_forms:
        # the same step with launch shapes from the build-time autotuner (its
        # first build tunes and caches; the timed steps reuse the cache)
        MSPLIT_T = dict(MSPLIT, autotune=True)
        P = M.MultiSplitPrec(A, **MSPLIT_T)
        del P
        ta = []
        for _ in range(max(3, args.steps // 2)):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            P = M.MultiSplitPrec(A, **MSPLIT_T)
            st_t = solve(P, False)
            e1.record(stream)
            e1.synchronize()
            ta.append(e0.elapsed_time(e1) / 1e3)
            del P
        out["autotuned"] = dict(s_per_step=float(np.mean(ta)), iters=st_t.niter, solve_ms=st_t.t_solve_ms,
                                setup_ms=st_t.t_setup_ms)

        progress("autotuned FP64 steps")
    if not args.no_forms:
        # ---- FP32-stored hierarchy (flexible FP64 PCG) ----
        timed(True, 2)  # warm-up of the FP32 kernels and graphs
        t32, (st32, nb32) = timed(True, max(3, args.steps // 2))
        timed(True, 1, autotune=True)  # tunes and caches the FP32 launch shapes
        t32a, (st32a, _) = timed(True, max(3, args.steps // 2), autotune=True)
        def host_solve(P, eps, flexible, maxit=0):
            x = np.empty(N)
            st = Stats()
            rc = lib().mlp_pcg(A.h, b.ctypes.data_as(C.POINTER(C.c_double)), P.h,
                               x.ctypes.data_as(C.POINTER(C.c_double)), eps, maxit, int(flexible), C.byref(st))
            if rc not in (0, 6):  # 6: the cap, when eps is below what rounding lets the residual reach
                check(rc)
            return x, st
        Pref = M.MultiSplitPrec(A, **MSPLIT)
        # tight FP64 reference: flexible iteration (the multi-split operator is not symmetric)
        x_true, st_true = host_solve(Pref, 1e-12, True, 1000)
        x64, _ = host_solve(Pref, EPS, False)
        del Pref
        P32 = M.MultiSplitPrec(A, fp32=True, **MSPLIT)
        x32, _ = host_solve(P32, EPS, True)
        x32b, st10 = host_solve(P32, 1e-10, True)
        nrm = np.linalg.norm(x_true)
        # the loosest tolerance at which the FP32-form solution is within 1e-8 of
        # the tight FP64 solution, with the device time of both forms there
        Pm = M.MultiSplitPrec(A, **MSPLIT)
        matched, sweep = None, []
        for e_m in (1e-8, 1e-9, 1e-10, 1e-11, 1e-12):
            xm, stm = host_solve(P32, e_m, True, 1000)
            sweep.append(dict(eps=e_m, x_err=float(np.linalg.norm(xm - x_true) / nrm), iters=stm.niter,
                              rel_res=stm.final_rel))
            if np.linalg.norm(xm - x_true) / nrm <= 1e-8:
                t32m = min(solve(P32, True, e_m, 1000).t_solve_ms for _ in range(3))
                s64m = [solve(Pm, False, e_m, 1000) for _ in range(3)]
                t64m = min(t.t_solve_ms for t in s64m)
                matched = dict(eps=e_m, x_err=float(np.linalg.norm(xm - x_true) / nrm), iters=stm.niter,
                               solve_ms=t32m, fp64_iters=s64m[0].niter, fp64_solve_ms=t64m,
                               solve_speedup_vs_fp64=t64m / t32m)
                break
        del P32, Pm
        out["fp32"] = dict(s_per_step=float(np.mean(t32)), iters=st32.niter, setup_ms=st32.t_setup_ms,
                           solve_ms=st32.t_solve_ms, bytes_per_apply=nb32,
                           solve_speedup_vs_fp64=st64.t_solve_ms / st32.t_solve_ms,
                           autotuned=dict(s_per_step=float(np.mean(t32a)), iters=st32a.niter,
                                          solve_ms=st32a.t_solve_ms,
                                          solve_speedup_vs_fp64=st64.t_solve_ms / st32a.t_solve_ms),
                           reference_rel_res=st_true.final_rel, reference_iters=st_true.niter,
                           x_err_fp32_1e8=float(np.linalg.norm(x32 - x_true) / nrm),
                           x_err_fp64_1e8=float(np.linalg.norm(x64 - x_true) / nrm),
                           x_err_fp32_1e10=float(np.linalg.norm(x32b - x_true) / nrm),
                           iters_1e10=st10.niter, rel_res_1e10=st10.final_rel,
                           x_diff_fp32_vs_fp64_1e8=float(np.linalg.norm(x32 - x64) / nrm),
                           within_1e8_of_fp64=matched, x_err_sweep=sweep)

        progress("FP32 form")
        # ---- adjoint gradient on the same mesh ----
        rng = np.random.default_rng(2)
        obs = np.sort(rng.choice(N, 25, replace=False))
        prob = adjoint.MisfitProblem(NX, NY, NZ, obs, np.zeros(25), eps=EPS, fp32=True)
        theta = np.log(kx)[adjoint.field_index(NX, NY, NZ)]
        prob.objective(theta)  # warm-up
        fw, gr = [], []
        for _ in range(3):
            torch.cuda.synchronize(); t0 = time.perf_counter()
            prob.objective(theta)
            torch.cuda.synchronize(); t1 = time.perf_counter()
            prob.gradient(theta)
            torch.cuda.synchronize(); t2 = time.perf_counter()
            fw.append(t1 - t0); gr.append(t2 - t1)
        out["adjoint"] = dict(grad_s=float(np.median(gr)), forward_s=float(np.median(fw)),
                              ratio=float(np.median(gr) / np.median(fw)), cells=N,
                              forward_solve_ms=prob.stats["forward"]["t_solve_ms"],
                              adjoint_solve_ms=prob.stats["adjoint"]["t_solve_ms"],
                              setup_ms=prob.stats["forward"]["t_setup_ms"],
                              adjoint_iters=prob.stats["adjoint"]["niter"])

        progress("adjoint")
        # ---- ensemble of 64 uneven realizations, sharded over the ranks ----
        dims = ensemble.realization_dims(64)
        mine = ensemble.shard(dims, rank, ws)
        E = ensemble.Ensemble([dims[i] for i in mine], field_seed0=1000, fp32=True)
        _, fwd_its = E.forward()
        fwd = [E.forward()[0] for _ in range(3)]
        adj = [E.adjoint([np.zeros(len(o)) for o in E.obs])[0] for _ in range(3)]
        pz = [np.zeros(len(o)) for o in E.obs]
        E.gradient(pz)
        grad1 = [E.gradient(pz)[0] for _ in range(3)]  # forward + adjoint + dJ/dlnK in one launch
        loop = [E.looped_forward()[0] for _ in range(2)]
        E.close()
        out["ensemble"] = dict(fwd_ms=float(np.median(fwd)), adj_ms=float(np.median(adj)),
                               grad_one_launch_ms=float(np.median(grad1)),
                               looped_ms=float(np.median(loop)), members=len(mine),
                               fwd_iters=[int(t) for t in fwd_its],
                               cells=int(sum(np.prod(dims[i]) for i in mine)))

        progress("ensemble")
    # ---- per-launch time of one apply inside its graph (the roofline's kernel) ----
    # mlp_prec_timeline: 10 back-to-back replays of the apply graph, each
    # kernel stamping %globaltimer as it passes its dependent-launch wait; per
    # launch group its in-graph time and algorithmic bytes. The levels below
    # the finest one are L2-resident (126 MB L2), so their traffic is mostly
    # not DRAM traffic. The launch-by-launch replay with events between the
    # launches (mlp_prec_profile) is kept beside it: it adds an event and a
    # launch gap to every launch, so it overstates the small launches.
    Pp = M.MultiSplitPrec(A, **MSPLIT)
    Pp.solve(np.random.default_rng(3).standard_normal(N))

    def grouped(rows, scale):
        groups = {}
        for nm, t_, by in rows:
            g = groups.setdefault(nm, [0, 0.0, 0])
            g[0] += 1
            g[1] += t_ * scale
            g[2] += by
        return sorted(([nm, c, t_, by] for nm, (c, t_, by) in groups.items()), key=lambda t: -t[2])

    prof = Pp.profile(5)
    out["apply_profile"] = grouped(prof, 1.0)  # ms
    out["apply_profile_ms"] = float(sum(t[1] for t in prof))
    tl = Pp.timeline(10)
    out["apply_timeline"] = grouped(tl, 1e-3)  # ms
    out["apply_timeline_ms"] = float(sum(t[1] for t in tl)) / 1e3
    # the whole apply (gather, graph, scatter) 20 times, events around them on
    # a stream of its own (a null stream handle would select the handle's
    # stream, which the events on torch's default stream do not wait for)
    fa = torch.randn(N, dtype=torch.float64, device=dev)
    za = torch.empty_like(fa)
    sa = torch.cuda.Stream(dev)
    sa.wait_stream(stream)
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record(sa)
    for _ in range(20):
        check(lib().mlp_prec_apply(Pp.h, C.c_void_p(fa.data_ptr()), C.c_void_p(za.data_ptr()),
                                   C.c_void_p(sa.cuda_stream)))
    g1.record(sa)
    g1.synchronize()
    out["apply_graph_ms"] = g0.elapsed_time(g1) / 20
    del fa, za
    # the PCG's own launches inside the solve graph (mlp_pcg_timeline, one
    # iteration near the end), with their algorithmic bytes
    nnz = A.nnz()
    pcg_bytes = {"pcg spmv_dot": 12 * nnz + 4 * (N + 1) + 16 * N, "pcg update": 48 * N, "pcg dot_rz": 16 * N,
                 "pcg p": 24 * N}
    out["pcg_timeline"] = [[nm, us_, pcg_bytes[nm]] for nm, us_ in Pp.pcg_timeline(A, b_d, x_d, EPS)
                           if nm in pcg_bytes]
    progress("apply timeline")
    del Pp

    if not args.no_forms:
        # ---- the harder c = 0.1 problem (6 levels on this field) ----
        A01, b01 = M.CSRMatrix.spe(NX, NY, NZ, kx, ky, kz, c=0.1, dirichlet=True)
        b01_d = torch.from_numpy(b01).to(dev)
        x01_d = torch.empty_like(b01_d)
        t01, st01, nl01 = [], None, 0
        for k in range(3 + max(3, args.steps // 2)):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            P01 = M.MultiSplitPrec(A01, **MSPLIT)
            st01 = Stats()
            check(lib().mlp_pcg_device(A01.h, C.c_void_p(b01_d.data_ptr()), P01.h, C.c_void_p(x01_d.data_ptr()),
                                       EPS, 0, 0, C.byref(st01), C.c_void_p(stream.cuda_stream)))
            e1.record(stream)
            e1.synchronize()
            nl01 = P01.nlevels
            if k >= 3:
                t01.append(e0.elapsed_time(e1) / 1e3)
            del P01
        out["c01"] = dict(s_per_step=float(np.mean(t01)), iters=st01.niter, levels=nl01,
                          setup_ms=st01.t_setup_ms, solve_ms=st01.t_solve_ms, steps=len(t01))
        del A01
        progress("c=0.1 steps")

        # ---- uh_cheb (sigma 3, Chebyshev degree 4 on every level, tails) ----
        # the same matrix and PCG; one warm-up step, then three timed ones
        tch, stch, nlch = [], None, 0
        for k in range(4):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            Pc = M.Prec(A, **UH_CHEB)
            stch = Stats()
            check(lib().mlp_pcg_device(A.h, C.c_void_p(b_d.data_ptr()), Pc.h, C.c_void_p(x_d.data_ptr()),
                                       EPS, 0, 0, C.byref(stch), C.c_void_p(stream.cuda_stream)))
            e1.record(stream)
            e1.synchronize()
            nlch = Pc.nlevels
            if k >= 1:
                tch.append(e0.elapsed_time(e1) / 1e3)
            del Pc
        out["uh_cheb"] = dict(s_per_step=float(np.mean(tch)), iters=stch.niter, levels=nlch,
                              setup_ms=stch.t_setup_ms, solve_ms=stch.t_solve_ms, steps=len(tch),
                              params="sigma 3, degree 4 per level, tails (-p uh_cheb -s 3 -b 4)")
        progress("uh_cheb steps")

    # ---- roofline: level-0 SpMV (staged kernel), events on its stream ----
    # 50 launches back to back between two events, alternating between two
    # copies of the matrix and vectors (2 x 116 MB > the 126 MB L2), so every
    # launch streams its matrix from HBM and the launch latency is amortised.
    ia, ja, a = A.arrays()
    A2 = M.CSRMatrix.from_arrays(ia, ja, a)
    mats = [A, A2]
    xs = [torch.randn(N, dtype=torch.float64, device=dev) for _ in range(2)]
    ys = [torch.empty_like(xs[0]) for _ in range(2)]

    def spmv(k):
        check(lib().mlp_spmv(mats[k & 1].h, C.c_void_p(xs[k & 1].data_ptr()), C.c_void_p(ys[k & 1].data_ptr()),
                             C.c_void_p(stream.cuda_stream)))

    for k in range(6):
        spmv(k)
    torch.cuda.synchronize()
    # the launches are recorded into a CUDA graph so that the host's call
    # overhead does not pace them
    reps = 50
    graph = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream(dev)
    with torch.cuda.stream(cap):
        cs = cap.cuda_stream
        graph.capture_begin()
        for k in range(reps):
            check(lib().mlp_spmv(mats[k & 1].h, C.c_void_p(xs[k & 1].data_ptr()), C.c_void_p(ys[k & 1].data_ptr()),
                                 C.c_void_p(cs)))
        graph.capture_end()
    graph.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    flush_l2(flush)
    gs = torch.cuda.current_stream(dev)
    e0.record(gs)
    graph.replay()
    e1.record(gs)
    e1.synchronize()
    out["spmv_ms"] = e0.elapsed_time(e1) / reps
    progress("level-0 SpMV")
    del graph
    out["spmv_bytes"] = 12 * A.nnz() + 4 * (N + 1) + 8 * N + 8 * N
    del A2

    if not args.no_forms:
        # ---- e2e through the C ABI with host buffers ----

        def e2e_step():
            A2 = M.CSRMatrix.from_arrays(ia, ja, a)
            P2 = M.MultiSplitPrec(A2, **MSPLIT)
            x = M.PCGSolver(A2, b, P2, eps=EPS)
            del P2, A2
            return x

        e2e_step()
        ke = max(3, min(args.steps, 5))
        tt = []
        for _ in range(ke):
            t0 = time.perf_counter()
            e2e_step()
            tt.append(time.perf_counter() - t0)
        out["e2e"] = {"value": float(np.mean(tt)), "unit": UNIT,
                      "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + a.nbytes + b.nbytes),
                      "d2h_bytes_per_step": int(8 * N)}
        progress("e2e")
    return out


def cpu_info():
    """Host CPU model and the cores the process may use."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    return model, cores


def reference_cpu(steps, warmup, timeout=1800, c=C_REACT, prec="msplit"):
    """The reference's own CPU build (oracle/_ref/ref_driver) on the same problem
    (prec "cheb": uh_cheb with the UH_CHEB parameters)."""
    from oracle import oracle as O
    from ml_prec_b200 import fields
    if not O.ref_available():
        return None
    kx, ky, kz = fields.field("layered", SEED)
    with tempfile.TemporaryDirectory() as td:
        perm = os.path.join(td, "perm.bin")
        fields.write_perm_bin(perm, kx, ky, kz)
        cfg = os.path.join(td, "msplit.cfg")
        with open(cfg, "w") as f:
            f.write(O.msplit_cfg_text())
        if prec == "cheb":
            r = O.run_ref(os.path.join(td, "out"), perm=perm, nx=NX, ny=NY, nz=NZ, c=c, prec="cheb",
                          sigmas=UH_CHEB["sigma"], niters=UH_CHEB["ncheb"], eps=EPS, reps=warmup + steps,
                          timeout=timeout)
        else:
            r = O.run_ref(os.path.join(td, "out"), perm=perm, nx=NX, ny=NY, nz=NZ, c=c, prec="msplit",
                          cfg=cfg, eps=EPS, reps=warmup + steps, timeout=timeout)
    su = r["t_setup_all"][warmup:]
    so = r["t_solve_all"][warmup:]
    per = [x + y for x, y in zip(su, so)]
    return dict(value=float(np.mean(per)), setup=float(np.mean(su)), solve=float(np.mean(so)),
                niter=r["niter"], steps=len(per))


def reference_ensemble(count, timeout=30):
    """min(count, cores) concurrent single-threaded reference processes, one
    ensemble realization each (the ensemble form's meshes and fields, matrices
    written in the reference's BINARY CSR format and loaded by its own reader):
    aggregate solves per second over the wall time of the batch. The
    reference's PCG has no iteration cap, and some realizations converge very
    slowly in FP64 (realization 4, 44x213x73, is still at 8.5e-8 after 200
    iterations), so a process still running after `timeout` seconds is
    stopped and counted in `timed_out`; the rate counts finished solves over
    the wall time up to the last one that finished."""
    from oracle import oracle as O
    from ml_prec_b200 import ensemble, fields
    if not O.ref_available():
        return None
    model, cores = cpu_info()
    k = min(count, cores)
    dims = ensemble.realization_dims(64)[:k]
    with tempfile.TemporaryDirectory() as td:
        cfg = os.path.join(td, "msplit.cfg")
        with open(cfg, "w") as f:
            f.write(O.msplit_cfg_text())
        jobs = []
        for i, d in enumerate(dims):
            kx, ky, kz = fields.field("iid", 1000 + i)
            A, b = O.assemble(*d, kx, ky, kz, 1.0, True)
            fa, fb = os.path.join(td, f"A{i}.csr"), os.path.join(td, f"b{i}.f64")
            O.write_csr(fa, A.ia, A.ja, A.a)
            b.tofile(fb)
            od = os.path.join(td, f"o{i}")
            os.makedirs(od)
            jobs.append([O.REF_DRIVER, "--out", od, "--csr", fa, "--rhs", fb, "--prec", "msplit", "--cfg", cfg,
                         "--eps", repr(EPS)])
        t0 = time.perf_counter()
        procs = [subprocess.Popen(j, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for j in jobs]
        rcs, ends = [None] * k, [None] * k
        while any(r is None for r in rcs) and time.perf_counter() - t0 < timeout:
            for i, p in enumerate(procs):
                if rcs[i] is None and p.poll() is not None:
                    rcs[i], ends[i] = p.returncode, time.perf_counter() - t0
            time.sleep(0.05)
        timed_out = 0
        for i, p in enumerate(procs):
            if rcs[i] is None:
                p.kill()  # this process was started above (its own PID)
                p.wait()
                timed_out += 1
        per, wall = [], max([e for e in ends if e is not None], default=0.0)
        for i in range(k):
            if rcs[i] == 0:
                r = json.load(open(os.path.join(td, f"o{i}", "result.json")))
                per.append(r["t_setup"] + r["t_solve"])
    return dict(processes=k, cores=cores, cpu_model=model, wall_s=wall,
                solves_per_s=len(per) / wall if wall > 0 else None,
                mean_solve_s=float(np.mean(per)) if per else None, failed=k - len(per) - timed_out,
                timed_out=timed_out, timeout_s=timeout, cells=int(sum(np.prod(d) for d in dims)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32, adjoint, ensemble and e2e measurements (profiling runs)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(1, min(args.steps, 5))
        r = reference_cpu(steps, 1)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver was not built"}))
            return
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": r["steps"],
                "warmup": 1, "ms_per_step": r["value"] * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "60x220x85 layered field (seed 2), c=1, Dirichlet x-faces; msplit.cfg; "
                                       "setup+PCG to rel-res 1e-8",
                           "parallelism": "single-threaded reference (the reference has no threads)"},
                "impl": "reference",
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                 "sample": f"{r['steps']} full setup+solve steps after 1 warm-up"},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "setup_s": r["setup"], "solve_s": r["solve"], "iters": r["niter"]}
        print(json.dumps(line))
        return

    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
    res = run_ours(args, ws, rank, local)
    t_step = float(np.sum(res["t64"])) / args.steps
    ens = res.get("ensemble")
    if ws > 1:
        import torch
        import torch.distributed as dist
        e2e = res.get("e2e")
        t = max_over_ranks([t_step, ens["fwd_ms"] if ens else 0.0, ens["adj_ms"] if ens else 0.0,
                            e2e["value"] if e2e else 0.0, ens["grad_one_launch_ms"] if ens else 0.0])
        t_step = float(t[0])
        if ens:
            ens["fwd_ms"], ens["adj_ms"], ens["grad_one_launch_ms"] = float(t[1]), float(t[2]), float(t[4])
        if e2e:
            e2e["value"] = float(t[3])
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = res["spmv_bytes"] / (res["spmv_ms"] / 1e3) / 1e9
    prof = res["apply_timeline"]
    top = prof[0]  # [name, launches, ms, bytes] of the launch group with the most in-graph time per apply

    def group_rows(rows):
        return [{"launch": nm, "launches": c, "ms": round(ms_, 4), "MB": round(by / 1e6, 3),
                 "GBps": round(by / (ms_ / 1e3) / 1e9, 1) if ms_ > 0 else None,
                 "frac": round(by / (ms_ / 1e3) / 1e9 / hbm, 3) if ms_ > 0 else None}
                for nm, c, ms_, by in rows[:12]]

    apply_groups = group_rows(prof)
    pcg_kernels = [{"launch": nm, "us": round(us_, 2), "MB": round(by / 1e6, 2),
                    "GBps": round(by / (us_ / 1e6) / 1e9, 1) if us_ > 0 else None,
                    "frac": round(by / (us_ / 1e6) / 1e9 / hbm, 3) if us_ > 0 else None}
                   for nm, us_, by in res["pcg_timeline"]]
    st64 = res["st64"]
    cpu = None
    if not args.no_cpu_baseline:
        r = reference_cpu(1, 0)
        progress("reference CPU step")
        if r:
            model, cores = cpu_info()
            cpu = {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "one full setup+PCG solve of the same 60x220x85 problem (single-threaded reference)",
                   "iters": r["niter"], "setup_s": r["setup"], "solve_s": r["solve"],
                   "host_cpu": model, "host_cores": cores}
            if not args.no_forms:
                r01 = reference_cpu(1, 0, c=0.1)
                progress("reference CPU step, c=0.1")
                if r01:
                    cpu["c01"] = {"value": r01["value"], "iters": r01["niter"], "setup_s": r01["setup"],
                                  "solve_s": r01["solve"]}
                rch = reference_cpu(1, 0, prec="cheb")
                progress("reference CPU step, uh_cheb")
                if rch:
                    cpu["uh_cheb"] = {"value": rch["value"], "iters": rch["niter"], "setup_s": rch["setup"],
                                      "solve_s": rch["solve"]}
                cpu["ensemble_concurrent"] = reference_ensemble(64)
                progress("reference ensemble")
    line = {
        "metric": METRIC, "value": t_step, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "60x220x85 layered field (seed 2), c=1, Dirichlet x-faces; multi-split "
                               "q=0.8 simple_1 degree_max=2 level_niter=5; setup+PCG to rel-res 1e-8",
                   "cells": res["N"], "nnz": res["nnz"], "l2": "flushed (256 MB write) between steps",
                   "parallelism": f"replicas x{ws}"},
        "step_s": [round(t, 5) for t in res["t64"]],
        "iters": st64.niter, "setup_ms": st64.t_setup_ms, "solve_ms": st64.t_solve_ms,
        "forms": None if ens is None else {
            "autotuned_fp64": res.get("autotuned"),
            "c01": res.get("c01"),
            "uh_cheb": res.get("uh_cheb"),
            "fp32_prec": res["fp32"],
            "adjoint": res["adjoint"],
            "ensemble": dict(ens, realizations=64, solves_per_s=64 / (ens["fwd_ms"] / 1e3),
                             gradients_per_s=64 / (ens["grad_one_launch_ms"] / 1e3),
                             scaling="strong (64 realizations sharded over the ranks)"),
        },
        "e2e": res.get("e2e"),
        "gpu_launches": res["nlaunch"],
        "roofline": {"bound": "hbm", "kernel": f"{top[0]} (the apply's launch group with the most in-graph time)",
                     "achieved": top[3] / (top[2] / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": top[3] / (top[2] / 1e3) / 1e9 / hbm,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s",
                     "bytes_per_launch": top[3] / top[1], "ms_per_launch": top[2] / top[1],
                     "timing": "in-graph time per launch (mlp_prec_timeline: %globaltimer stamped by each kernel "
                               "as it passes its dependent-launch wait, 10 back-to-back replays of the apply graph)",
                     "traffic": FOLD_DRAM_TRAFFIC.get(top[0]),
                     "traffic_source": ("taken from profiles/phase2_fold_level2_60x220x85.md (ncu, one launch, cold "
                                        "caches), not measured in this run" if top[0] in FOLD_DRAM_TRAFFIC
                                        else "no ncu capture of this launch group on this matrix"),
                     "apply_groups": apply_groups,
                     "pcg_kernels": pcg_kernels,
                     "apply_ms_in_graph": res["apply_timeline_ms"],
                     "apply_graph_ms_events": res["apply_graph_ms"],
                     "apply_groups_launch_by_launch": group_rows(res["apply_profile"]),
                     "apply_ms_launch_by_launch": res["apply_profile_ms"],
                     "spmv_level0": {"kernel": "level-0 CSR SpMV y = A x (k_spmv_staged, pipelined tiles)",
                                     "achieved": achieved, "frac": achieved / hbm,
                                     "bytes_per_launch": res["spmv_bytes"], "ms_per_launch": res["spmv_ms"],
                                     "timing": "50 launches back to back in one CUDA graph, two matrix copies "
                                               "alternated (232 MB > L2)",
                                     "traffic": SPMV_DRAM_TRAFFIC,
                                     "traffic_source": "taken from profiles/spmv_level0_60x220x85.md (an ncu capture "
                                                       "of one launch on this matrix), not measured in this run"}},
        "prec_bytes_per_apply": res["nb64"],
        "cpu_baseline": cpu,
        "clocks": res["clocks"],
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
