#!/usr/bin/env python
"""Benchmark: multigrid-preconditioned CG time to 1e-8 relative residual on the
128^3-element hexahedral elasticity cantilever, mixed precision vs FP64, plus
SpMV HBM throughput of the CSR and DuVi formats on the same operator.

Workload (all synthetic, seeded): unit-cube 8-node hexahedra, E = 1, nu = 0.3,
3 dofs/node, all nodes of face x = 0 clamped, uniform unit traction (-z) on
face x = 128 (6,390,144 free dofs, 509,597,550 stored entries).  Hierarchy:
factor-2 re-discretised levels 128 -> 64 -> 32 -> 16 -> 8 with trilinear
prolongation and restriction = its transpose, V(2,2) weighted Jacobi with the
weight 2/3 of the spectrally normalised operator, dense coarse solve.

  value       device time of one solve (b resident in HBM -> x in HBM), mixed
              precision: FP32 DuVi V-cycle inside the FP64 flexible CG, max over ranks
  e2e         the same solve through the host API (pinned host b in, host x out)
  fp64        the plain FP64 path (CSR FP64 operators everywhere) for comparison
  spmv        isolated SpMV of the finest operator per format/precision (uniform E and
              per-element E = 10^U(-2,0), both at the full size), each launch timed
              alone with CUDA events after an L2 flush, GB/s of the algorithmic bytes
              and the fraction of the measured HBM peak
  roofline    the dominant kernel of the solve (the fine-level residual / Jacobi sweep
              body on the FP32 DuVi operator's derived layout) against the bytes it must
              move, plus every isolated SpMV in roofline.kernels
  gauss_seidel  the same solve with V(2,2) forward Gauss-Seidel (multicolor; the
              reference's row order), mixed precision
  batched     64 load cases on 64^3 in one multi-right-hand-side solve, and 32
              uneven cantilevers in one batched solve, each against the same
              work done one solve at a time
  adjoint     96x48x48, E = rho^3: forward solve, adjoint solve + dJ/drho kernel
The comparison sections (fp64, gauss_seidel, batched, adjoint) run at N = 1 only.

--impl reference times the CPU restatement of the reference's algorithm
(oracle/, FP64, all host threads) on the same workload: every step is one
whole FP64 MG-FCG solve of the 128^3 problem to the tolerance.
Multi-GPU (--gpus N under torchrun): independent replicas, one 128^3 solve per
rank, no collective on the data path; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MG-PCG time to 1e-8 rel. residual (mixed FP32/FP64, 128^3 hex elasticity)"

# dv_matrix_info.kernel_variant -> kernel (DuVi: 100 + g lane layout, 200 + g node patterns,
# 300 + g grid stencil; CSR: threads per row; DuVi 4 / 9: staged row bundles)
KERNEL_NAMES = {101: "k_duvi_lanes", 102: "k_duvi_lanes", 103: "k_duvi_lanes", 201: "k_duvi_pattern",
                202: "k_duvi_pattern", 203: "k_duvi_pattern", 303: "k_duvi_grid", 400: "k_hex_elem", 4: "k_duvi",
                9: "k_duvi"}
# derived layouts whose matrix costs ~2 bytes per node group: their algorithmic bytes are the vectors
DERIVED_SHAPES = {201, 202, 203, 303}
OMEGA_EFF = (2.0 / 3.0) * 2.0 / (1.1 * 3.09)   # 2/3 of the spectrally normalised Jacobi weight (lambda ~ 3.09)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=128)
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--iterations-per-sync", type=int, default=4,
                   help="most outer iterations between host reads of the stop flag (MG-PCG solvers)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-spmv", action="store_true")
    p.add_argument("--no-batched", action="store_true", help="skip the multi-load-case section")
    p.add_argument("--batched-only", action="store_true",
                   help="only the multi-load-case MG-PCG (64 load cases on the 64^3 mesh)")
    p.add_argument("--adjoint-only", action="store_true", help="only the adjoint section (96x48x48)")
    p.add_argument("--no-gs", action="store_true", help="skip the Gauss-Seidel-smoothed MG-PCG lines")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint section")
    p.add_argument("--no-pcg", action="store_true", help="skip the Jacobi-PCG section (16^3, CSR and DuVi)")
    p.add_argument("--batch-size", type=int, default=64, help="mesh edge of the multi-load-case section")
    p.add_argument("--batch-k", type=int, default=64, help="load cases of the multi-load-case section")
    p.add_argument("--batch-meshes", type=int, default=32, help="meshes of the batched-mesh section")
    p.add_argument("--resid", action="store_true", help="with --spmv-only: time r = b - A x instead of y = A x")
    p.add_argument("--host-setup", action="store_true",
                   help="build the DuVi solvers from the host-assembled hierarchy instead of on the device")
    p.add_argument("--spmv-only", default=None, metavar="FMT_PREC",
                   help="only time the SpMV of the finest operator (duvi_f32, duvi_f64, csr_f32, csr_f64, or the "
                        "matrix-free hex_f32, hex_f64 with E = 10^U(-2,0)): the case used for ncu captures")
    return p.parse_args()


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def max_over_ranks(v, ws):
    from compressiontests_b200.replicas import max_over_ranks as mor
    return mor(v, ws, device="cuda")


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi samples (every 50 ms) of SM clock, power and throttle reasons.

    start() launches the sampler before the warm-up so it is running when the timed region
    begins; mark() / unmark() bracket the timed region; stop() keeps the samples whose
    timestamps fall inside it (with 60 ms of slack either side)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"bench_clocks_{os.getpid()}.csv")
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.5)   # let the sampler come up before the timed region
        except Exception:
            self.proc = None

    def mark(self):
        import datetime
        self.t0 = datetime.datetime.now()

    def unmark(self):
        import datetime
        self.t1 = datetime.datetime.now()

    def stop(self):
        import datetime
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        slack = datetime.timedelta(milliseconds=60)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
                clk, cmax = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            if self.t0 is not None and self.t1 is not None and not (self.t0 - slack <= ts <= self.t1 + slack):
                continue
            sm.append(clk)
            smax = cmax
            for n, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "interval_ms": 50}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(key):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch of a kernel from the committed
    single-pass ncu summary (profiles/dram_traffic_128.json), or None."""
    p = os.path.join(ROOT, "profiles", "dram_traffic_128.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)).get(key, {}).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


def roofline_entry(name, ms, alg, peak, peak_kind, traffic_key, bound="hbm"):
    achieved = alg / ms / 1e6
    e = {"kernel": name, "bound": bound, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
         "frac": round(achieved / peak, 3), "traffic": ncu_traffic(traffic_key), "peak_kind": peak_kind,
         "algorithmic_bytes_per_launch": int(alg), "avg_launch_ms": round(ms, 4)}
    return e


def build_problem(n):
    import compressiontests_b200 as cb
    t = time.time()
    A, P = cb.hex_hierarchy((n, n, n), coarse_ne=8)
    b = cb.traction_rhs((n, n, n))
    return A, P, b, time.time() - t


def time_events(stream, fn, reps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


_FLUSH = {}


def l2_flush(stream):
    """Writes 256 MB (twice the 126 MB L2) on `stream`, evicting what the previous launch left in L2."""
    import torch
    buf = _FLUSH.get("buf")
    if buf is None:
        buf = _FLUSH["buf"] = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        buf.fill_(1.0)


def time_launches(stream, fn, reps):
    """Mean device time of fn() over reps launches, each bracketed alone by CUDA events on `stream`
    after an L2 flush, so every launch reads its inputs from HBM."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for a, b in ev:
        l2_flush(stream)
        a.record(stream)
        fn()
        b.record(stream)
    ev[-1][1].synchronize()
    return sum(a.elapsed_time(b) for a, b in ev) / reps


def spmv_table(cb, ctx, A0, reps, peak, cases=(("duvi", "f32"), ("duvi", "f64"), ("csr", "f32"), ("csr", "f64"))):
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    n = A0.shape[0]
    dom = None
    for fmt, prec in cases:
        M = cb.SparseMatrix(ctx, A0, fmt, prec)
        info = M.info()
        dt = torch.float32 if prec == "f32" else torch.float64
        g = torch.Generator(device="cuda").manual_seed(20261203)
        x = torch.randn(n, dtype=dt, device="cuda", generator=g)
        y = torch.zeros_like(x)
        torch.cuda.synchronize()
        fn = lambda: M.multiply_device(x.data_ptr(), y.data_ptr(), prec)
        for _ in range(3):
            fn()
        ctx.synchronize()
        ms = time_launches(stream, fn, reps)
        vs = 4 if prec == "f32" else 8
        fmt_bytes = info["device_bytes"] + 2 * vs * n      # the caller's format: matrix arrays + x + y
        derived = info["kernel_variant"] in DERIVED_SHAPES  # node patterns / grid stencil: x + y + 2 B per node
        alg = (2 * vs * n + 2 * (n // 3)) if derived else fmt_bytes
        gbs = alg / ms / 1e6
        out[f"{fmt}_{prec}"] = {"ms": round(ms, 4), "algorithmic_bytes": int(alg), "GBps": round(gbs, 1),
                                "frac_of_peak": round(gbs / peak, 3), "value_index_bits": info["value_index_bits"],
                                "nblocks": info["nblocks"], "nuniq": info["nuniq"],
                                "launch_shape": info["kernel_variant"],
                                "kernel": KERNEL_NAMES.get(info["kernel_variant"], "k_csr" if fmt == "csr" else "k_duvi"),
                                "format_bytes": int(fmt_bytes),
                                "format_GBps": round(fmt_bytes / ms / 1e6, 1)}
        if fmt == "duvi" and prec == "f32":
            dom = (M, x, y, info)
        else:
            M.release()
        del x, y
        torch.cuda.empty_cache()
    return out, dom


def spmv_log_uniform(cb, ctx, n, reps, peak):
    """SpMV of the n^3 operator with per-element E = 10^U(-2, 0) (seeded): nearly every stored
    value is distinct, so DuVi needs 32-bit value indices and a table as long as nnz."""
    rng = np.random.default_rng(20261203)
    E = 10.0 ** rng.uniform(-2.0, 0.0, n ** 3)
    t = time.time()
    A0 = cb.hex_stiffness((n, n, n), E)
    t_asm = time.time() - t
    out, _ = spmv_table(cb, ctx, A0, reps, peak, (("csr", "f64"), ("duvi", "f64")))
    del A0
    out.update(hex_operator_spmv(cb, ctx, (n, n, n), E, reps, peak))
    return {"size": f"{n}^3", "elem_E": "10^U(-2,0) per element, seed 20261203", "assembly_s": round(t_asm, 1),
            **out}


def hex_operator_spmv(cb, ctx, ne, E, reps, peak):
    """The same operator applied matrix-free (element kernel): one factor per element, x and y."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    for prec in ("f64", "f32"):
        H = cb.SparseMatrix.hex_operator(ctx, ne, E, precision=prec)
        n = H.shape[0]
        dt = torch.float32 if prec == "f32" else torch.float64
        x = torch.randn(n, dtype=dt, device="cuda", generator=torch.Generator(device="cuda").manual_seed(20261203))
        y = torch.zeros_like(x)
        torch.cuda.synchronize()
        fn = lambda: H.multiply_device(x.data_ptr(), y.data_ptr(), prec)
        for _ in range(3):
            fn()
        ctx.synchronize()
        ms = time_launches(stream, fn, reps)
        vs = 4 if prec == "f32" else 8
        alg = H.info()["device_bytes"] + 2 * vs * n
        out[f"hex_{prec}"] = {"ms": round(ms, 4), "algorithmic_bytes": int(alg), "GBps": round(alg / ms / 1e6, 1),
                              "frac_of_peak": round(alg / ms / 1e6 / peak, 3), "launch_shape": 400,
                              "kernel": "k_hex_elem", "format_bytes": int(alg),
                              "format_GBps": round(alg / ms / 1e6, 1)}
        H.release()
        del x, y
        torch.cuda.empty_cache()
    return out


def cpu_solve(A, P, b, threads, tol):
    """One whole FP64 MG-FCG solve of the oracle (the CPU restatement of the reference's V-cycle
    algorithm) to tol on `threads` host threads: (iteration-phase seconds, iterations, rel. residual)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.build()
    O.lib().or_set_threads(threads)
    Ao = [a if isinstance(a, O.Csr) else O.Csr.from_scipy(a) for a in A]
    Po = [p if isinstance(p, O.Csr) else O.Csr.from_scipy(p) for p in P]
    _, its, rel = O.mg_fcg(Ao, Po, b, OMEGA_EFF, 2, 500, tol)
    return O.lib().or_last_solve_seconds(), its, rel


def oracle_problem(O, n):
    """The same workload built by the oracle's own structured restatement (no product code)."""
    A, P = [], []
    ne, scale = n, 1.0
    while True:
        A.append(O.hex_stiffness((ne, ne, ne), scale=scale))
        if ne <= 8 or ne % 2:
            break
        P.append(O.hex_trilinear((ne, ne, ne)))
        ne //= 2
        scale *= 2.0
    b = O.traction_rhs((n, n, n), (n, n, n), (0.0, 0.0, -1.0))
    return A, P, b


def run_reference(args):
    ws, rank, _ = dist_init(args)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.build()
    threads = O.lib().or_omp_threads()
    O.lib().or_set_threads(threads)
    n = args.size
    A, P, b = oracle_problem(O, n)
    times, its, rels = [], [], []
    for k in range(args.warmup + args.steps):
        sec, it, rel = cpu_solve(A, P, b, threads, args.tol)   # one whole solve to the tolerance
        assert it > 0, "the CPU restatement did not converge"
        if k >= args.warmup:
            times.append(sec * 1e3)
            its.append(it)
            rels.append(rel)
    v = float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 1), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"mg-pcg hex elasticity {n}^3 (unit traction, x=0 clamped), V(2,2) Jacobi, "
                                   "FP64 flexible CG, CPU restatement of the reference's algorithm",
                       "n_dofs": int(A[0].shape[0]), "nnz": int(A[0].nnz), "tol": args.tol,
                       "iterations": int(its[-1]), "relative_residual_fp64": float(rels[-1]),
                       "step_ms_min_max": [round(min(times), 1), round(max(times), 1)]},
            "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": threads, "kind": "port",
                             "sample": f"every step one whole FP64 MG-FCG solve of the {n}^3 problem to {args.tol:g} "
                                       f"({its[-1]} iterations), iteration phase timed (set-up excluded)"},
            "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    ws, rank, local = dist_init(args)
    torch.cuda.set_device(local)
    import compressiontests_b200 as cb
    peak, peak_kind = measured_peaks()
    n = args.size
    A, P, b, t_build = build_problem(n)
    ctx = cb.CudaContext(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    nf = A[0].shape[0]

    def make(precision, fmt, tol=None):
        tol = args.tol if tol is None else tol
        if fmt == "duvi" and not args.host_setup:   # hierarchy assembled and encoded on the device
            return cb.MultigridPcgSolver.from_hex(ctx, (n, n, n), coarse_ne=8, precision=precision, nu=2,
                                                  omega=2 / 3, omega_mode="spectral", tol=tol, max_iterations=500,
                                                  iterations_per_sync=args.iterations_per_sync)
        return cb.MultigridPcgSolver(ctx, A, P, precision=precision, fmt=fmt, outer_fmt=fmt, nu=2, omega=2 / 3,
                                     omega_mode="spectral", tol=tol, max_iterations=500,
                                     iterations_per_sync=args.iterations_per_sync)

    db = torch.from_numpy(b).to(f"cuda:{local}")
    dx = torch.zeros_like(db)
    torch.cuda.synchronize()

    def timed(solver, steps, warmup):
        st = None
        sampler = ClockSampler(local)
        sampler.start()
        try:
            for _ in range(warmup):
                st = solver.solve_device(db.data_ptr(), dx.data_ptr())
            barrier(ws)
            torch.cuda.synchronize()
            ctx.synchronize()
            l0 = ctx.launch_count()
            sampler.mark()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            its, rel = [], []
            for _ in range(steps):
                st = solver.solve_device(db.data_ptr(), dx.data_ptr())
                its.append(st.NumIterationsRequired)
                rel.append(st.RelativeResidual)
                assert st.HasConverged, st
            e1.record(stream)
            e1.synchronize()
            sampler.unmark()
        finally:
            clocks = sampler.stop()
        launches = ctx.launch_count() - l0
        ms = e0.elapsed_time(e1) / steps
        barrier(ws)
        return max_over_ranks(ms, ws), its, rel, launches, clocks

    t = time.time()
    mixed = make("mixed", "duvi")
    t_setup = time.time() - t
    ms_mixed, its_mixed, rel_mixed, launches, clocks = timed(mixed, args.steps, args.warmup)
    x_mixed = dx.cpu().numpy()
    true_rel = float(np.linalg.norm(b - A[0] @ x_mixed) / np.linalg.norm(b))

    # e2e through the host API: pinned host b -> device, solve, device x -> pinned host
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty_like(hb).pin_memory()
    bp, xp = hb.numpy(), hx.numpy()
    for _ in range(1):
        mixed.Solve(bp)
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        import ctypes as C
        st = cb._native.Stats()
        cb._native.check(cb._native.lib().dv_mgpcg_solve(mixed.h, C.c_void_p(hb.data_ptr()), C.c_void_p(hx.data_ptr()),
                                                         C.byref(st)))
        assert st.converged
    e1.record(stream)
    e1.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
    mixed.release()

    fp64 = {}
    extras = ws == 1   # the comparison sections run at N = 1 only (replicas would repeat them per rank)
    if not args.no_fp64 and extras:
        for fmt in ("csr", "duvi"):
            s = make("f64", fmt)
            ms, its, rel, _, _ = timed(s, max(2, min(5, args.steps // 2)), 1)
            fp64[fmt] = {"ms": round(ms, 2), "iterations": its[-1], "rel_residual": rel[-1],
                         "mixed_speedup": round(ms / ms_mixed, 2)}
            s.release()

    # The multigrid configuration also states its FP64 and mixed runs to 1e-10: the same solvers
    # to the tighter tolerance.
    tight = {}
    if not args.no_fp64 and extras:
        for prec in ("mixed", "f64"):
            s = make(prec, "duvi", tol=1e-10)
            try:
                ms, its, rel, _, _ = timed(s, max(2, min(5, args.steps // 2)), 1)
                tight[prec] = {"ms": round(ms, 2), "iterations": its[-1], "rel_residual": rel[-1]}
            except AssertionError as e:   # not converged: recorded, the other sections still run
                tight[prec] = {"error": f"not converged: {e}"}
            finally:
                s.release()
        if "ms" in tight["mixed"] and "ms" in tight["f64"]:
            tight["mixed_speedup_vs_fp64_duvi"] = round(tight["f64"]["ms"] / tight["mixed"]["ms"], 2)

    gauss_seidel = {}
    if not args.no_gs and extras:
        for smoother, prec in (("gs_color", "mixed"), ("gs_lex", "mixed")):
            t = time.time()
            s = cb.MultigridPcgSolver(ctx, A, P, precision=prec, fmt="duvi", outer_fmt="duvi", nu=2, tol=args.tol,
                                      max_iterations=500, smoother=smoother)
            t_gs = time.time() - t
            ms, its, rel, _, _ = timed(s, 1, 1)
            gauss_seidel[f"{smoother}_{prec}"] = {"ms": round(ms, 2), "iterations": its[-1], "rel_residual": rel[-1],
                                                  "setup_s": round(t_gs, 1)}
            s.release()

    spmv, dom = ({}, None) if args.no_spmv else spmv_table(cb, ctx, A[0], 20, peak)
    roof = None
    if dom is not None:
        # The dominant kernel of the solve: the fine-level FP32 operator pass of the V-cycle (residual and
        # Jacobi sweeps, about half of the device time) on the derived layout the autotuner picked.  Its
        # algorithmic bytes are the vectors it must stream: x (gathered once), b and r, 4 bytes per row each.
        M0, _, _, info0 = dom
        vb = [torch.randn(nf, dtype=torch.float32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(s))
              for s in (1, 2)]
        rv = torch.empty_like(vb[0])
        torch.cuda.synchronize()
        fn = lambda: M0.residual_device(vb[0].data_ptr(), vb[1].data_ptr(), rv.data_ptr(), "f32")
        for _ in range(3):
            fn()
        ctx.synchronize()
        ms_res = time_launches(stream, fn, 20)
        kname = KERNEL_NAMES.get(info0["kernel_variant"], "k_duvi")
        roof = roofline_entry(f"{kname}<float> r = b - A x, DuVi FP32 {n}^3 operator (fine-level V-cycle pass)",
                              ms_res, 12 * nf, peak, peak_kind, f"{kname}_f32_resid")
        roof["bytes_note"] = ("x, b, r: 4 bytes per row each, every launch after an L2 flush; the derived layout's "
                              "2-byte node ids are not counted")
        M0.release()
        del vb, rv
        kernels = []
        for key, v in spmv.items():
            kernels.append({**roofline_entry(f"{v['kernel']} y = A x, {key}, {n}^3 uniform E", v["ms"],
                                             v["algorithmic_bytes"], peak, peak_kind, f"{v['kernel']}_{key}_spmv"),
                            "format_GBps": v["format_GBps"]})
        if extras:
            spmv["log_uniform_E"] = spmv_log_uniform(cb, ctx, n, 10, peak)
            for key, v in spmv["log_uniform_E"].items():
                if isinstance(v, dict):
                    kernels.append(roofline_entry(f"{v['kernel']} y = A x, {key}, {n}^3 E = 10^U(-2,0)", v["ms"],
                                                  v["algorithmic_bytes"], peak, peak_kind,
                                                  f"{v['kernel']}_{key}_spmv_logE"))
        roof["kernels"] = kernels

    batched = None
    if not args.no_batched and extras:
        batched = {"load_cases": batched_multi_rhs(cb, ctx, stream, args.batch_size, args.batch_k,
                                                   max(1, min(5, args.steps // 2)), args.tol),
                   "meshes": batched_meshes(cb, ctx, stream, args.batch_meshes, max(1, min(5, args.steps // 2)), args.tol)}

    adjoint = None
    if not args.no_adjoint and extras:
        adjoint = adjoint_section(cb, ctx, stream, max(1, min(5, args.steps // 2)), 1e-10)

    jacobi_pcg = None
    if not args.no_pcg and extras:
        try:   # a reported extra: a failure here is recorded, not fatal to the headline line
            jacobi_pcg = jacobi_pcg_section(cb, ctx, 16, max(1, min(5, args.steps // 2)))
        except Exception as e:
            jacobi_pcg = {"error": f"{type(e).__name__}: {e}"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            sec, its_cpu, rel_cpu = cpu_solve(A, P, b, 1, args.tol)
            cpu = {"value": round(sec * 1e3, 1), "unit": "ms", "cores": 1, "kind": "port",
                   "sample": f"one whole FP64 MG-FCG solve of the oracle (single thread, the reference's CPU code is "
                             f"single-threaded) on the same {n}^3 problem to {args.tol:g}: {its_cpu} iterations, "
                             f"relative residual {rel_cpu:.2e}, iteration phase timed"}
        except Exception as e:  # the baseline must not hide the GPU result
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "port", "sample": f"failed: {e}"}

    summary = {}
    for fmt in ("duvi", "csr"):
        if fmt in fp64:
            summary[f"fp64_{fmt}_ms"] = fp64[fmt]["ms"]
            summary[f"mixed_speedup_vs_fp64_{fmt}"] = fp64[fmt]["mixed_speedup"]
    for prec in ("mixed", "f64"):
        if "ms" in tight.get(prec, {}):
            summary[f"tol_1e-10_{prec}_ms"] = tight[prec]["ms"]
            summary[f"tol_1e-10_{prec}_iterations"] = tight[prec]["iterations"]
    for key, v in gauss_seidel.items():
        summary[f"{key}_ms"] = v["ms"]
        summary[f"{key}_iterations"] = v["iterations"]
    if jacobi_pcg and "csr" in jacobi_pcg:
        for fmt in ("csr", "duvi"):
            summary[f"jacobi_pcg_16cube_{fmt}_ms"] = jacobi_pcg[fmt]["device_ms"]
            summary[f"jacobi_pcg_16cube_{fmt}_iterations"] = jacobi_pcg[fmt]["iterations"]
    if batched:
        summary["load_cases_64x64cube_ms"] = batched["load_cases"]["ms"]
        summary["meshes_32_ms"] = batched["meshes"]["ms"]
    if adjoint:
        summary["adjoint_mixed_forward_ms"] = adjoint["mixed"]["forward_ms"]
        summary["adjoint_mixed_backward_ms"] = adjoint["mixed"]["backward_ms"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms_mixed, 3), "unit": "ms", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_mixed, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"mg-pcg hex elasticity {n}^3 (unit traction, x=0 clamped), V(2,2) Jacobi, "
                                   f"FP32 DuVi V-cycle in FP64 flexible CG, {len(A)} levels to {A[-1].shape[0]} dofs",
                       "n_dofs": int(nf), "nnz": int(A[0].nnz), "tol": args.tol, "levels": len(A),
                       "l2_flush": f"working set larger than L2: five FP64 vectors and five FP32 finest-level "
                                   f"vectors per iteration, {60 * nf / 1e6:.0f} MB against 126 MB; isolated kernel "
                                   "timings flush L2 (256 MB write) before every launch",
                       "parallelism": f"replicas x{ws}",
                       "summary": summary},
            "iterations": its_mixed[-1], "relative_residual_fp64": true_rel,
            "e2e": {"value": round(ms_e2e, 3), "unit": "ms", "h2d_bytes_per_step": int(8 * nf),
                    "d2h_bytes_per_step": int(8 * nf)},
            "gpu_launches": int(launches), "fp64": fp64, "tol_1e-10": tight, "spmv": spmv, "gauss_seidel": gauss_seidel, "batched": batched, "adjoint": adjoint, "jacobi_pcg": jacobi_pcg, "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks, "setup_s": {"hierarchy_host": round(t_build, 1), "solver": round(t_setup, 1),
                                          "solver_built_on": "host" if args.host_setup else "device"},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batched_multi_rhs(cb, ctx, stream, size, k, steps, tol):
    """k load cases (N(0,1) nodal forces on the free face) on the size^3 mesh: one
    multi-right-hand-side solve against k single solves of the same load cases."""
    import torch
    ne = (size, size, size)
    A, P = cb.hex_hierarchy(ne, coarse_ne=8)
    B = cb.random_face_loads(ne, k, seed=20261203)
    s = cb.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", nu=2, omega=2 / 3, omega_mode="spectral",
                              tol=tol, max_iterations=500)
    dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    dX = torch.zeros_like(dB)
    torch.cuda.synchronize()
    st, conv = s.solve_many_device(k, dB.data_ptr(), dX.data_ptr())   # eager warm-up, then graph replays
    l0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        st, conv = s.solve_many_device(k, dB.data_ptr(), dX.data_ptr())
        assert conv.all(), st
    e1.record(stream)
    e1.synchronize()
    ms_multi = e0.elapsed_time(e1) / steps
    launches = (ctx.launch_count() - l0) // steps
    X = dX.cpu().numpy()
    rel = float(np.max(np.linalg.norm(B - A[0] @ X, axis=0) / np.linalg.norm(B, axis=0)))
    # the same load cases one after another (PcgSolver2.InverseSystemMatrixTimesOtherMatrix order)
    cols = [torch.from_numpy(np.ascontiguousarray(B[:, j])).cuda() for j in range(k)]
    dx = torch.zeros_like(cols[0])
    torch.cuda.synchronize()
    s.solve_device(cols[0].data_ptr(), dx.data_ptr())
    its1 = []
    e0.record(stream)
    for j in range(k):
        st1 = s.solve_device(cols[j].data_ptr(), dx.data_ptr())
        its1.append(st1.NumIterationsRequired)
    e1.record(stream)
    e1.synchronize()
    ms_seq = e0.elapsed_time(e1)
    s.release()
    return {"workload": f"{k} load cases, N(0,1) nodal forces on the free face, {size}^3 hex mesh, "
                        "mixed MG-PCG (FP32 DuVi V(2,2) in FP64 FCG), tol {tol:g} per load case".format(tol=tol),
            "n_dofs": int(A[0].shape[0]), "k": k, "ms": round(ms_multi, 3), "ms_per_load_case": round(ms_multi / k, 4),
            "iterations": int(st.NumIterationsRequired), "worst_relative_residual_fp64": rel,
            "sequential_ms": round(ms_seq, 3), "sequential_iterations_max": int(max(its1)),
            "speedup_vs_sequential": round(ms_seq / ms_multi, 2), "gpu_launches_per_solve": int(launches)}


def batched_meshes(cb, ctx, stream, n_meshes, steps, tol):
    """n_meshes cantilevers with edge lengths U{8..48} (seeded), Galerkin hierarchies, unit
    traction on each free face: one batched solve (block-diagonal levels, graph-captured)
    against the same meshes solved one after another with one solver each."""
    import torch
    t = time.time()
    dims, meshes, rhs = cb.cantilever_batch(n_meshes, 8, 48, seed=20261203)
    t_build = time.time() - t
    t = time.time()   # hierarchies built in the library, finest operators matrix-free (one launch for all meshes)
    s = cb.BatchedMultigridSolver.from_hex(ctx, dims, max_coarse_dofs=1000, precision="mixed", nu=2, omega=2 / 3,
                                           omega_mode="spectral", tol=tol, max_iterations=500)
    t_setup = time.time() - t
    b = torch.from_numpy(np.concatenate(rhs)).cuda()
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    st, conv, its = s.solve_device(b.data_ptr(), x.data_ptr())
    l0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        st, conv, its = s.solve_device(b.data_ptr(), x.data_ptr())
        assert conv.all(), st
    e1.record(stream)
    e1.synchronize()
    ms_batch = e0.elapsed_time(e1) / steps
    launches = (ctx.launch_count() - l0) // steps
    xs = np.split(x.cpu().numpy(), s.offsets[1:-1])
    worst = max(float(np.linalg.norm(r - A[0] @ xm) / np.linalg.norm(r)) for (A, _), r, xm in zip(meshes, rhs, xs))
    info = s.info()
    s.release()
    # the same meshes one after another, one solver per mesh (the reference's one-model-per-solver shape)
    ms_seq, its_seq = 0.0, []
    for (A, P), r in zip(meshes, rhs):
        one = cb.MultigridPcgSolver(ctx, A, P, precision="mixed", fmt="duvi", nu=2, omega=2 / 3,
                                    omega_mode="spectral", tol=tol, max_iterations=500)
        db = torch.from_numpy(r).cuda()
        dx = torch.zeros_like(db)
        torch.cuda.synchronize()
        one.solve_device(db.data_ptr(), dx.data_ptr())
        e0.record(stream)
        st1 = one.solve_device(db.data_ptr(), dx.data_ptr())
        e1.record(stream)
        e1.synchronize()
        ms_seq += e0.elapsed_time(e1)
        its_seq.append(st1.NumIterationsRequired)
        one.release()
    return {"workload": f"{n_meshes} cantilevers, edge lengths U{{8..48}} per axis (seeded), unit traction, "
                        "Galerkin hierarchies to <= 1000 coarse dofs, mixed MG-PCG per mesh to "
                        f"{tol:g}, one batched graph-captured solve, finest operators matrix-free",
            "n_dofs": int(s.n), "levels_max": info["n_levels_max"], "ms": round(ms_batch, 3),
            "iterations_max": int(its.max()), "worst_relative_residual_fp64": worst,
            "sequential_ms": round(ms_seq, 3), "sequential_iterations_max": int(max(its_seq)),
            "speedup_vs_sequential": round(ms_seq / ms_batch, 2), "gpu_launches_per_solve": int(launches),
            "launches_per_graph_chunk": info["launches_per_chunk"],
            "setup_s": {"hierarchies": round(t_build, 1), "solver": round(t_setup, 1)}}


def jacobi_pcg_section(cb, ctx, n, reps, tol=1e-8):
    """Jacobi-PCG (OpenCLCsrPcgSolver's algorithm) on the n^3 cantilever, unit traction, FP64, from
    zero to the relative residual ||r||_2 <= tol ||b||_2, CSR then DuVi (and once more with the
    reference's own stop test max |r_i| <= tol): the solver's device time per solve, the time through
    the host API (b in, x out) and the FP64 relative residual of the result."""
    ne = (n, n, n)
    A = cb.hex_stiffness(ne)
    b = cb.traction_rhs(ne)
    out = {"workload": f"Jacobi-PCG, {n}^3 cantilever, unit traction, FP64, stop ||r||_2 <= {tol:g} ||b||_2 "
                       f"(abs_max rows: the reference's max|r_i| <= {tol:g})",
           "n_dofs": int(A.shape[0])}
    for fmt, kind in (("csr", "rel_l2"), ("duvi", "rel_l2"), ("csr", "abs_max"), ("duvi", "abs_max")):
        s = cb.CudaCsrPcgSolver(ctx, 20000, tol, fmt=fmt, tol_kind=kind).Initialize(A=A, b=b)
        try:
            s.Solve()   # warm-up (the first call captures the iteration graph)
            dev, host = [], []
            for _ in range(reps):
                t0 = time.perf_counter()
                x, st = s.Solve()
                host.append((time.perf_counter() - t0) * 1e3)
                dev.append(st.SolveMilliseconds)
        finally:
            s.release()
        rel = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
        out[fmt if kind == "rel_l2" else f"{fmt}_abs_max"] = {
            "device_ms": round(min(dev), 3) if np.isfinite(min(dev)) else None,
            "host_api_ms": round(min(host), 3), "iterations": st.NumIterationsRequired,
            "converged": st.HasConverged, "relative_residual_fp64": rel if np.isfinite(rel) else None}
    return out


def adjoint_section(cb, ctx, stream, steps, tol):
    """96 x 48 x 48 cantilever, rho ~ U[0.01, 1] (seeded), E = rho^3, unit traction, J = c^T u
    with c ~ N(0, 1): forward solve, adjoint solve + element gradient kernel, FP64 and mixed."""
    import torch
    ne = (96, 48, 48)
    rng = np.random.default_rng(20261203)
    rho = rng.uniform(0.01, 1.0, int(np.prod(ne)))
    f = cb.traction_rhs(ne)
    c = rng.standard_normal(f.shape[0])
    out = {"workload": "adjoint dJ/drho, 96x48x48 hex cantilever, rho~U[0.01,1] seeded, E=rho^3, unit traction, "
                       f"J=c^T u (c~N(0,1)), Galerkin hierarchy to <= 2000 dofs, tol {tol:g}",
           "n_elements": int(rho.size), "n_dofs": int(f.shape[0])}
    grads = {}
    for prec in ("mixed", "f64"):
        t = time.time()
        prob = cb.AdjointCantilever(ctx, ne, rho, max_coarse_dofs=2000, precision=prec, tol=tol, max_iterations=2000)
        t_setup = time.time() - t
        prob.forward(f)
        prob.backward(c)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        fw = bw = 0.0
        for _ in range(steps):
            e0.record(stream)
            u, st_f = prob.forward(f)
            e1.record(stream)
            g, st_b = prob.backward(c)
            e2.record(stream)
            e2.synchronize()
            fw += e0.elapsed_time(e1)
            bw += e1.elapsed_time(e2)
        grads[prec] = g
        out[prec] = {"forward_ms": round(fw / steps, 3), "backward_ms": round(bw / steps, 3),
                     "forward_iterations": int(st_f.NumIterationsRequired),
                     "adjoint_iterations": int(st_b.NumIterationsRequired),
                     "forward_rel_residual": float(st_f.RelativeResidual),
                     "adjoint_rel_residual": float(st_b.RelativeResidual), "setup_s": round(t_setup, 1)}
        prob.release()
    out["mixed_vs_f64_gradient_max_rel"] = float(np.max(np.abs(grads["mixed"] - grads["f64"])) /
                                                 np.max(np.abs(grads["f64"])))
    # the element kernel alone
    d = [torch.from_numpy(v).cuda() for v in (rho, u, u)]
    gd = torch.zeros(rho.size, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fn = lambda: cb.element_gradient_device(ctx, ne, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), gd.data_ptr())
    fn()
    out["element_kernel_ms_incl_sync"] = round(time_events(stream, fn, 10), 4)
    return out


def run_adjoint_only(args):
    import torch
    import compressiontests_b200 as cb
    ctx = cb.CudaContext(0)
    r = adjoint_section(cb, ctx, torch.cuda.ExternalStream(ctx.stream), args.steps, 1e-10)
    print(json.dumps({"adjoint": r}), flush=True)
    ctx.close()


def run_batched_only(args):
    import torch
    import compressiontests_b200 as cb
    ctx = cb.CudaContext(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    r = {"load_cases": batched_multi_rhs(cb, ctx, stream, args.batch_size, args.batch_k, args.steps, args.tol),
         "meshes": batched_meshes(cb, ctx, stream, args.batch_meshes, args.steps, args.tol)}
    print(json.dumps({"batched": r}), flush=True)
    ctx.close()


def run_spmv_only(args):
    import torch
    import compressiontests_b200 as cb
    fmt, prec = args.spmv_only.split("_")
    n = args.size
    ctx = cb.CudaContext(0)
    if fmt == "hex":   # matrix-free operator, per-element E = 10^U(-2,0)
        E = 10.0 ** np.random.default_rng(20261203).uniform(-2.0, 0.0, n ** 3)
        M = cb.SparseMatrix.hex_operator(ctx, (n, n, n), E, precision=prec)
    else:
        M = cb.SparseMatrix(ctx, cb.hex_stiffness((n, n, n)), fmt, prec)
    info = M.info()
    dt = torch.float32 if prec == "f32" else torch.float64
    g = torch.Generator(device="cuda").manual_seed(20261203)
    x = torch.randn(M.shape[0], dtype=dt, device="cuda", generator=g)
    y = torch.zeros_like(x)
    b = torch.randn(M.shape[0], dtype=dt, device="cuda", generator=g)
    torch.cuda.synchronize()
    if args.resid:
        fn = lambda: M.residual_device(b.data_ptr(), x.data_ptr(), y.data_ptr(), prec)
    else:
        fn = lambda: M.multiply_device(x.data_ptr(), y.data_ptr(), prec)
    for _ in range(args.warmup):
        fn()
    ctx.synchronize()
    ms = time_events(torch.cuda.ExternalStream(ctx.stream), fn, args.steps)
    alg = info["device_bytes"] + (3 if args.resid else 2) * (4 if prec == "f32" else 8) * M.shape[0]
    print(json.dumps({"spmv": args.spmv_only, "resid": args.resid, "size": n, "ms": ms, "algorithmic_bytes": int(alg),
                      "GBps": alg / ms / 1e6, "launch_shape": info["kernel_variant"]}), flush=True)
    M.release()
    ctx.close()


if __name__ == "__main__":
    a = parse()
    if a.spmv_only:
        run_spmv_only(a)
    elif a.batched_only:
        run_batched_only(a)
    elif a.adjoint_only:
        run_adjoint_only(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
