#!/usr/bin/env python3
"""CPR-GMRES time-to-1e-8 on the 8M-row two-phase system, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl deco|reference]

Workload: the 200x200x100 two-phase grid (bs = 2: 8,000,000 rows, 111,360,000
nonzeros; lognormal permeability sigma 2.5 with 1e4-contrast channels; seeded
synthetic data in the reference's CSR layout), preconditioned by
CPR(FSAI global p1 + FSAI pressure p1; seq 3, quasiimpes_GE, CPD) and solved
with right-preconditioned GMRES(50) to a float64 true relative residual of 1e-8.

A step is one complete solve of a freshly assembled system: the matrix and
right-hand side are copied from pristine HBM copies (CPR decouples them in
place), then the CPR setup (decoupling, A_pp, two FSAI setups) and the GMRES
solve run.  `value` is the mixed-precision path (float32 CPR and Krylov basis,
float64 refinement); the plain float64 path is timed the same way and reported
beside it (`fp64`).  Times are CUDA events on the library's stream, max over
ranks.  Every input (1.3 GB of matrix) is larger than L2.

`e2e` repeats the mixed step through the C ABI from pinned host buffers: the
host-to-device copy of the CSR arrays and b and the device-to-host copy of x are
inside the timed region.  `roofline` is the dominant kernel of the mixed solve
(the float32 CSR SpMV of A) timed alone with CUDA events, L2 flushed between
launches.  `cpu_baseline` / `--impl reference` run the reference's own CPU code
(compiled from its sources into oracle/_ref) on the host cores.

With --gpus N > 1 (torchrun) every rank solves its own copy of the system
(replicas: the single-system path is not sharded).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the reference's OpenMP pool uses every host core; its LAPACK runs single-threaded inside it
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

METRIC = "CPR-GMRES time-to-1e-8 (mixed vs FP64, same B200); SpMV/FSAI HBM GB/s"
CONFIG = 3
SEED = 1234
WORKLOAD = ("200x200x100 two-phase grid, bs=2, 8,000,000 rows, 111,360,000 nnz, lognormal k sigma 2.5 "
            "+ 1e4-contrast channels; CPR(FSAI global p1 + FSAI pressure p1, seq 3, quasiimpes_GE, CPD) "
            "+ right GMRES(50), true relative residual 1e-8")
PREC = {"type": "CPR", "block_size": "2", "pressure_id": "0", "seq": "3", "weights": "quasiimpes_GE",
        "use_drs": "0", "drs": {"e_dd": "0.2", "e_ps": "0.0"}, "CPD": "1", "tol_zero": "0.0",
        "prec_glo": {"type": "FSAI", "tol_rel": "0.0", "tol_abs": "1e-16", "power": "1"},
        "prec_loc": {"type": "FSAI", "tol_rel": "1e-4", "tol_abs": "1e-16", "power": "1"}}
SOL = {"type": "rgmres", "reltol": "1e-8", "restart": "50", "itmax": "6000", "verbosity": "0"}
# Iterations the float64 path needs for this system and seed (the reference's MGS
# variant needs the same number within 10%, as the parity tests check at smaller
# sizes); the reference arm extrapolates its measured per-iteration time to it.
ITERS_TO_TOL = 1046
REF_SAMPLE_ITERS = 10


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        rows = [[x.strip() for x in line.split(",")] for line in self.f.read().splitlines() if line.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        load = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_system():
    from deco_b200 import gen
    return gen.generate(gen.preset(CONFIG, SEED))


def reference_sample(s, iters_to_tol):
    """Reference CPU code on the host: full CPR setup + REF_SAMPLE_ITERS GMRES
    iterations, extrapolated to `iters_to_tol` iterations."""
    from oracle import ref
    sol = dict(SOL, itmax=str(REF_SAMPLE_ITERS))
    t0 = time.perf_counter()
    R = ref.Cpr({"prec": PREC}, s.r, s.c, s.v, s.b)
    t_setup = time.perf_counter() - t0
    res = R.solve(sol)
    per_it = res["time"] / max(1, res["iter"])
    total = t_setup + per_it * iters_to_tol
    del R
    return total, t_setup, per_it, ref.num_threads()


def run_reference(args, rank, world):
    unit = "s"
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdeco_ref.so was not built"}))
        return
    s = make_system()
    times = []
    for k in range(args.warmup + args.steps):
        total, t_setup, per_it, threads = reference_sample(s, ITERS_TO_TOL)
        if k >= args.warmup:
            times.append(total)
    v = statistics.mean(times)
    sample = (f"reference CPR setup on the full system + {REF_SAMPLE_ITERS} GMRES iterations per step, "
              f"extrapolated to {ITERS_TO_TOL} iterations to 1e-8")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "seed": SEED, "parallelism": "openmp"},
        "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def bench_batch(args):
    """64 independent two-phase systems (cells log-uniform in 10k-500k), 8
    right-hand sides each, one lockstep CPR-GMRES solve per precision.  Under
    torchrun the systems are dealt round-robin to the ranks (independent systems:
    no collective on the data path); the time is the max over ranks."""
    import datetime
    import torch
    import deco_b200 as d
    from deco_b200 import gen, replicas
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = d.Context(int(os.environ.get("LOCAL_RANK", 0)))
    st = ctx.torch_stream
    torch.cuda.set_stream(st)
    r, c, v, ro, B, shapes = gen.batch(64, SEED, 10_000, 500_000, 2, 8)
    n_all, nnz_all = int(ro[-1]), len(c)
    if world > 1:
        r, c, v, ro, B = gen.batch_subset(r, c, v, ro, B, 8, list(range(rank, 64, world)))
    n, nnz = int(ro[-1]), len(c)
    dev = lambda a: torch.from_numpy(a).cuda()
    r_d, c_d, v_d, B_d = dev(r), dev(c), dev(v), dev(B)
    out = {}
    for bits in (32, 64):
        rows = []
        for k in range(args.warmup + args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            A = d.CSR(n, n, r_d, c_d, v_d, ctx)
            Bt = d.Batch(PREC, A, ro, 8, precision=bits)
            X = Bt.solve(SOL, B_d)
            e1.record(st)
            e1.synchronize()
            if k >= args.warmup:
                rows.append((e0.elapsed_time(e1), Bt.result, Bt.iters.copy(), Bt.res_rel.copy(), Bt.widths.copy()))
            del Bt, A, X
        ms = replicas.max_over_ranks(statistics.mean(t[0] for t in rows), device="cuda")
        res, it, rr, w = rows[-1][1], rows[-1][2], rows[-1][3], rows[-1][4]
        inst = int(replicas.sum_over_ranks(it.size, device="cuda"))
        out["mixed" if bits == 32 else "fp64"] = {
            "time_s": ms / 1e3, "solve_ms": res["t_solve_ms"], "cycles": res["cycles"], "graph": res["graph"],
            "converged": int(replicas.sum_over_ranks(res["converged"], device="cuda")), "instances": inst,
            "iterations_max": int(replicas.max_over_ranks(int(it.max()), device="cuda")),
            "iterations_median_rank0": float(statistics.median(it.ravel().tolist())),
            "max_true_rel_residual": replicas.max_over_ranks(float(rr.max()), device="cuda"),
            "widths": sorted(set(int(x) for x in w)), "instances_per_s": inst / (ms / 1e3)}
    line = {"metric": "batched CPR-GMRES time-to-1e-8 (64 systems x 8 right-hand sides)",
            "value": out["mixed"]["time_s"], "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "scaling": "strong", "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"64 two-phase systems, cells log-uniform 10k-500k ({n_all // 2} cells, "
                                   f"{n_all} rows, {nnz_all} nnz), 8 uniform right-hand sides each; CPR seq 3 + "
                                   f"GMRES(50)", "seed": SEED,
                       "parallelism": f"systems dealt round-robin to {world} GPU(s), no collective"}, **out,
            "speedup_mixed_vs_fp64": out["fp64"]["time_s"] / out["mixed"]["time_s"]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def bench_spmv(args):
    """The SpMV of the 8M-row system alone (a few GB on the device): CSR and cell-block
    storage, float64 and float32 values, all rows and the restricted row-0 product;
    sized for profiler captures (`ncu -k regex:bsr2_pair`)."""
    import torch
    import deco_b200 as d
    ctx = d.Context(0)
    st = ctx.torch_stream
    torch.cuda.set_stream(st)
    s = make_system()
    n, nnz = s.n, s.nnz
    A = d.CSR.from_system(s, ctx)
    del s
    x64 = torch.randn(n, dtype=torch.float64, device="cuda")
    x32 = x64.float()
    y64 = torch.empty(n, dtype=torch.float64, device="cuda")
    y32 = torch.empty(n, dtype=torch.float32, device="cuda")
    yr = torch.empty(n // 2, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    reps = max(1, args.steps)

    def ms(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    peak, _ = peaks()
    out = {}
    A.apply_f32(x32, y32)
    for fmt in ("csr", "blocks"):
        if fmt == "blocks":
            A.set_blocks(2)
        bsz, nblk = A.blocks
        if bsz:
            mat = lambda vb: nblk * 4 + nblk * 4 * vb + 4 * (n // 2 + 1)
            row0 = nblk * 4 + nblk * 2 * 8 + 4 * (n // 2 + 1)
        else:
            mat = lambda vb: nnz * (4 + vb) + 4 * (n + 1)
            row0 = nnz // 2 * 12 + 4 * (n // 2 + 1)
        for name, fn, byt in (("f64", lambda: A.apply(x64, y64), mat(8) + 16 * n),
                              ("f32", lambda: A.apply_f32(x32, y32), mat(4) + 8 * n),
                              ("f64_row0", lambda: A.apply(x64, yr, bs=2), row0 + 8 * n + 4 * n)):
            t = ms(fn)
            out[f"{fmt}_{name}"] = {"ms": t, "gbs": byt / t / 1e6, "frac_of_peak": byt / t / 1e6 / peak, "bytes": byt}
    print(json.dumps({"metric": "SpMV HBM GB/s on the 8M-row system", "unit": "GB/s", "n_gpus": 1, "steps": reps,
                      "warmup": args.warmup, "data": "synthetic", "peak_gbs": peak,
                      "config": {"workload": WORKLOAD.split(";")[0], "seed": SEED}, "kernels": out}))


def bench_adjoint(args):
    """64x64x32 log-permeability system: forward CPR-GMRES, adjoint CPR-GMRES on A^T
    and the on-pattern gradient, float64 and mixed."""
    import numpy as np
    import torch
    import deco_b200 as d
    from deco_b200 import gen
    ctx = d.Context(0)
    st = ctx.torch_stream
    torch.cuda.set_stream(st)
    p = gen.preset(5, SEED)
    s = gen.generate(p, with_logk=True)
    rng = np.random.default_rng(2024)
    obs = rng.choice(s.n // 2, 20, replace=False)
    g = np.zeros(s.n)
    g[2 * obs] = rng.random(20)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    r_d, c_d, v_d, b_d, g_d = dev(s.r), dev(s.c), dev(s.v), dev(s.b), dev(g)
    out = {}
    for bits in (64, 32):
        rows = []
        for k in range(args.warmup + args.steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(st)
            A = d.CSR(s.n, s.n, r_d, c_d, v_d, ctx)
            b = b_d.clone()
            P = d.CPR(PREC, A, b, bits)
            S = d.SOL(SOL, A, P, b, precision=bits)
            ev[1].record(st)
            A0 = d.CSR(s.n, s.n, r_d, c_d, v_d, ctx)
            J = d.ADJ(PREC, A0, bits)
            lam = J.solve(SOL, g_d)
            ev[2].record(st)
            grad = A0.grad_pattern(lam, S.x)
            ev[3].record(st)
            ev[3].synchronize()
            if k >= args.warmup:
                rows.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3]),
                             S.iter, J.iter))
            del S, P, A, J, A0, lam, grad
        f = statistics.mean(t[0] for t in rows)
        a = statistics.mean(t[1] for t in rows)
        gk = statistics.mean(t[2] for t in rows)
        alg = 12 * s.nnz + 8 * (s.n + 1) + 8 * s.n
        out["fp64" if bits == 64 else "mixed"] = {
            "forward_ms": f, "adjoint_ms": a, "adjoint_over_forward": a / f, "grad_kernel_ms": gk,
            "grad_kernel_gbs": alg / gk / 1e6, "forward_iterations": rows[-1][3], "adjoint_iterations": rows[-1][4]}
    print(json.dumps({"metric": "adjoint gradient time (forward + transpose CPR-GMRES + dL/dA on pattern)",
                      "value": (out["fp64"]["forward_ms"] + out["fp64"]["adjoint_ms"] + out["fp64"]["grad_kernel_ms"])
                      / 1e3, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "higher_is_better": False, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": "64x64x32 two-phase grid from a seeded log-permeability "
                                             "field, bs 2, 262,144 rows; L = weighted pressures at 20 seeded cells; "
                                             "CPR seq 3 + GMRES(50) to 1e-8 forward and adjoint", "seed": SEED},
                      **out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="deco", choices=["deco", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the per-kernel timings (for profiler captures on a smaller --config)")
    ap.add_argument("--config", type=int, default=3, help="system preset (3 = the 200x200x100 benchmark workload)")
    ap.add_argument("--workload", default="solve", choices=["solve", "batch", "adjoint", "spmv"],
                    help="solve: the headline single-system solve; batch: 64 systems x 8 right-hand sides; "
                         "adjoint: the 64x64x32 log-permeability gradient; "
                         "spmv: the SpMV kernels alone")
    args = ap.parse_args()
    if args.workload == "batch":
        return bench_batch(args)
    if args.workload == "adjoint":
        return bench_adjoint(args)
    if args.workload == "spmv":
        return bench_spmv(args)
    global CONFIG
    CONFIG = args.config
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import datetime

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import deco_b200 as d
    from deco_b200 import replicas
    from deco_b200._lib import lib

    ctx = d.Context(local)
    st = ctx.torch_stream
    torch.cuda.set_stream(st)
    s = make_system()
    n, nnz = s.n, s.nnz
    PREC["block_size"] = str(s.bs)
    dev = lambda a: torch.from_numpy(a).cuda()
    r_d, c_d, v_d, b_d = dev(s.r), dev(s.c), dev(s.v), dev(s.b)
    pin = lambda a: torch.from_numpy(a).pin_memory()
    r_h, c_h, v_h, b_h = pin(s.r), pin(s.c), pin(s.v), pin(s.b)
    x_h = torch.empty(n, dtype=torch.float64).pin_memory()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step(bits, host=False):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        if host:
            A = d.CSR(n, n, r_h, c_h, v_h, ctx)
            b = b_h.to("cuda", non_blocking=True)
        else:
            A = d.CSR(n, n, r_d, c_d, v_d, ctx)
            b = b_d.clone()
        P = d.CPR(PREC, A, b, precision=bits)
        S = d.SOL(SOL, A, P, b, precision=bits)
        if host:
            x_h.copy_(S.x, non_blocking=True)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        true_rel = (A.residual(b, S.x).norm() / b.norm()).item()
        ph = P.timings()
        info = dict(ms=ms, iter=S.iter, flag=S.flag, res_rel=S.res_rel, true_rel=true_rel, orig_rel=S.res_rel_orig,
                    setup_ms=ph["Prec"], solve_ms=S.time_ms, setup_phases_ms={k: round(v, 2) for k, v in ph.items()})
        del S, P, A, b
        return info

    def timed(bits, k, host=False):
        if k == 0:
            return 0.0, [dict(ms=0, iter=0, flag=-1, res_rel=0, true_rel=0, orig_rel=0, setup_ms=0, solve_ms=0)], 0.0, 0
        # no Python garbage-collection pause inside the timed steps (timeit's practice)
        gc.collect()
        gc.disable()
        barrier()
        l0 = lib().deco_launch_count()
        t0 = time.perf_counter()
        try:
            infos = [step(bits, host) for _ in range(k)]
        finally:
            gc.enable()
        barrier()
        wall = time.perf_counter() - t0
        launches = lib().deco_launch_count() - l0
        ms = replicas.max_over_ranks(sum(i["ms"] for i in infos) / k, device="cuda")
        return ms, infos, wall, launches

    if args.kernels_only:
        args.warmup, args.steps, args.no_fp64, args.no_e2e, args.no_cpu_baseline = 0, 0, True, True, True
    for _ in range(args.warmup):
        step(32)
    clk = Clocks(local)
    ms_mixed, info_mixed, wall_mixed, launches = timed(32, args.steps)
    clocks = clk.stop()
    fp64 = None
    if not args.no_fp64:
        step(64)  # warm the float64 kernels
        ms64, info64, _, _ = timed(64, args.steps)
        fp64 = {"time_s": ms64 / 1e3, "iterations": info64[-1]["iter"], "true_rel_residual": info64[-1]["true_rel"],
                "original_system_rel_residual": info64[-1]["orig_rel"],
                "setup_ms": info64[-1]["setup_ms"], "solve_ms": info64[-1]["solve_ms"],
                "ms_per_iteration": info64[-1]["solve_ms"] / max(1, info64[-1]["iter"]),
                "step_ms": [round(i["ms"], 1) for i in info64], "setup_phases_ms": info64[-1]["setup_phases_ms"]}
    e2e = None
    if not args.no_e2e:
        step(32, host=True)
        ms_e2e, _, _, _ = timed(32, args.steps, host=True)
        h2d = (n + 1) * 4 + nnz * 4 + nnz * 8 + n * 8
        e2e = {"value": ms_e2e / 1e3, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * 8}

    # ---- roofline of the dominant kernel (float32 CSR SpMV of A) and the other hot kernels
    peak, peak_kind = peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def kernel_ms(fn, reps=20):
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    A = d.CSR(n, n, r_d, c_d, v_d, ctx)
    b = b_d.clone()
    P64 = d.CPR(PREC, A, b, precision=64)
    x64 = torch.randn(n, dtype=torch.float64, device="cuda")
    y64 = torch.empty_like(x64)
    x32, y32 = x64.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    A.apply_f32(x32, y32)  # creates the float32 value copy
    Fg = P64.fsai(0)
    nzF = Fg.nz
    kernels = {}

    def matrix_bytes(nz, blocks, vb):
        """Bytes of one pass over a matrix in the layout the product reads: the
        cell-block copy (one 4-byte index per bs x bs block, block-row pointers)
        when there is one, else CSR (4-byte index + value per entry)."""
        bsz, nblk = blocks
        if bsz:
            return nblk * 4 + nblk * bsz * bsz * vb + 4 * (n // bsz + 1)
        return nz * (4 + vb) + 4 * (n + 1)

    fmt = ("cell-block (bs %d)" % A.blocks[0] if A.blocks[0] else "CSR") + \
        (", %d padded slots per cell" % A.padded if A.padded else "")
    ms = kernel_ms(lambda: A.apply_f32(x32, y32))
    alg32 = matrix_bytes(nnz, A.blocks, 4) + 4 * n + 4 * n
    kernels["spmv_A_f32"] = {"ms": ms, "gbs": alg32 / ms / 1e6, "alg_bytes": alg32, "format": fmt,
                             "subwarp": A.subwarp}
    ms = kernel_ms(lambda: A.apply(x64, y64))
    alg64 = matrix_bytes(nnz, A.blocks, 8) + 8 * n + 8 * n
    kernels["spmv_A_f64"] = {"ms": ms, "gbs": alg64 / ms / 1e6, "alg_bytes": alg64, "format": fmt}
    fb, kl, ku = Fg.blocks
    ms = kernel_ms(lambda: Fg.apply(x64, y64))
    algF = matrix_bytes(nzF, (fb, kl), 8) + matrix_bytes(nzF, (fb, ku), 8) + 8 * n + 2 * 8 * n + 8 * n
    kernels["fsai_apply_global_f64"] = {"ms": ms, "gbs": algF / ms / 1e6, "alg_bytes": algF, "nnz_factor": nzF,
                                        "format": ("cell-block (bs %d)" % fb if fb else "CSR")
                                        + (", %d/%d padded slots" % Fg.padded if Fg.padded[0] else ""),
                                        "note": "the intermediate FL x (64 MB) stays in L2 between the two products"}
    del P64
    P32 = d.CPR(PREC, d.CSR(n, n, r_d, c_d, v_d, ctx), b_d.clone(), precision=32)
    Fg32 = P32.fsai(0)
    fb, kl, ku = Fg32.blocks
    # as the mixed-precision CPR applies it: float32 x, intermediate and y
    ms = kernel_ms(lambda: Fg32.apply_f32(x32, y32))
    algF32 = matrix_bytes(nzF, (fb, kl), 4) + matrix_bytes(nzF, (fb, ku), 4) + 4 * n + 2 * 4 * n + 4 * n
    kernels["fsai_apply_global_f32"] = {"ms": ms, "gbs": algF32 / ms / 1e6, "alg_bytes": algF32,
                                        "format": "cell-block (bs %d)" % fb if fb else "CSR",
                                        "vectors": "float32 (deco_fsai_apply_f32)"}
    # through the reference-shaped interface: float64 x and y around the float32 factor
    ms = kernel_ms(lambda: Fg32.apply(x64, y64))
    algF32d = matrix_bytes(nzF, (fb, kl), 4) + matrix_bytes(nzF, (fb, ku), 4) + 8 * n + 2 * 4 * n + 8 * n
    kernels["fsai_apply_global_f32_f64io"] = {"ms": ms, "gbs": algF32d / ms / 1e6, "alg_bytes": algF32d,
                                              "format": "cell-block (bs %d)" % fb if fb else "CSR",
                                              "vectors": "float64 (deco_fsai_apply)"}
    del P32
    for k in kernels.values():
        k["frac_of_peak"] = k["gbs"] / peak
    dom = kernels["spmv_A_f32"]
    roofline = {"bound": "hbm", "achieved": dom["gbs"], "peak": peak, "unit": "GB/s", "frac": dom["gbs"] / peak,
                # DRAM read + write bytes per launch of this kernel from one ncu capture of this
                # workload: the padded kernel with 7 slots 592.0 MB read + 7.2 MB written
                # (profiles/ell2_f32_config3_full.md; with 8 slots 672.0 + 8.9 MB); the pair kernel 604.8 + 11.5 MB
                # (profiles/bsr2_pair_f32_config3_full.md)
                "traffic": ({7: 599.2e6, 8: 680.9e6}.get(A.padded) if A.padded else 616.3e6 if A.blocks[0] == 2 else None),
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/"
                                   + ("ell2_f32_config3_full.md" if A.padded else "bsr2_pair_f32_config3_full.md"))
                if A.blocks[0] == 2 else None,
                "kernel": ("deco::ell2_kernel<%d, float> (2x2 cell blocks, %d padded slots per cell)" % (A.padded, A.padded)
                           if A.padded else
                           {2: "deco::bsr2_pair_kernel<float> (2x2 cell blocks)",
                            3: "deco::bsr_kernel<float> (3x3 cell blocks)"}.get(A.blocks[0], "deco::spmv_kernel<float> (CSR)"))
                + " on A (8M rows, 111.36M nnz, float32 values)",
                "algorithmic_bytes": "the unpadded cell-block layout's bytes (padding slots count against the kernel)",
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                iters = fp64["iterations"] if fp64 else ITERS_TO_TOL
                total, t_setup, per_it, threads = reference_sample(s, iters)
                cpu = {"value": total, "unit": "s", "cores": threads, "kind": "reference",
                       "sample": f"reference CPR setup on the full system ({t_setup:.1f} s) + {REF_SAMPLE_ITERS} "
                                 f"GMRES iterations ({per_it:.3f} s each), extrapolated to {iters} iterations",
                       "setup_s": t_setup, "s_per_iteration": per_it}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    last = info_mixed[-1]
    out = {
        "metric": METRIC, "value": ms_mixed / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "seed": SEED, "precision": "mixed: float32 CPR + float32 Krylov basis, "
                   "float64 dots/Hessenberg/true residual/solution", "l2": "inputs larger than L2 (1.3 GB matrix)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "mixed": {"iterations": last["iter"], "true_rel_residual": last["true_rel"], "flag": last["flag"],
                  "original_system_rel_residual": last["orig_rel"],
                  "setup_ms": last["setup_ms"], "solve_ms": last["solve_ms"],
                  "ms_per_iteration": last["solve_ms"] / max(1, last["iter"]),
                  "step_ms": [round(i["ms"], 1) for i in info_mixed], "setup_phases_ms": last.get("setup_phases_ms")},
        "fp64": fp64,
        "speedup_mixed_vs_fp64": (fp64["time_s"] / (ms_mixed / 1e3)) if fp64 else None,
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": kernels,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
