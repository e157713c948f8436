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
(the float32 product of A) timed alone with CUDA events, L2 flushed between
launches; `kernels` adds the other hot kernels, the orthogonalisation among them
(timed by events around every Arnoldi step of one solve).  The line also carries
the other benchmark systems, each with its own stated step count: `config2`
(100x100x50 three-phase with faults, float64 and mixed), `adjoint` (64x64x32
log-permeability gradient) and `batch` (64 systems x 8 right-hand sides).

`cpu_baseline` runs the reference's own CPU code (compiled from its sources into
oracle/_ref) on the host cores: its CPR setup plus one whole restart cycle,
scaled by the reference's measured iteration count to 1e-8 (recorded by
tests/golden/make_reference_runs.py).  `--impl reference` measures the
reference's full solve to 1e-8 once, live, then samples one restart cycle per
remaining step.

With --gpus N > 1 (torchrun) every rank solves its own copy of the system
(replicas: the single-system path is not sharded); the batch's 64 independent
systems are dealt round-robin to the ranks.
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
REF_RUNS = os.path.join(ROOT, "tests", "golden", "reference_runs.json")


def reference_record(config):
    """The reference build's own run on a benchmark system (iterations, residual,
    threads), as tests/golden/make_reference_runs.py recorded it; None if absent."""
    try:
        with open(REF_RUNS) as f:
            return json.load(f).get(f"config{config}")
    except (OSError, ValueError):
        return None


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


GRID = None  # (nx, ny, nz) overriding the preset's grid (smaller cases for profiler captures)


def make_system():
    from deco_b200 import gen
    p = gen.preset(CONFIG, SEED)
    if GRID is not None:
        p.nx, p.ny, p.nz = GRID
    return gen.generate(p)


def reference_cycle(R):
    """One whole restart cycle of the reference's rgmres (50 iterations: every
    Gram-Schmidt length j = 0..49 of its MGS, then the cycle's solution update and
    true residual) on an existing CPR object; returns its seconds."""
    res = R.solve(dict(SOL, itmax=SOL["restart"]))
    return res["time"], res["iter"]


def reference_sample(s, iters):
    """Reference CPU code on the host: the full CPR setup plus one whole restart
    cycle, the cycle time scaled to `iters` iterations."""
    from oracle import ref
    t0 = time.perf_counter()
    R = ref.Cpr({"prec": PREC}, s.r, s.c, s.v, s.b)
    t_setup = time.perf_counter() - t0
    t_cyc, it = reference_cycle(R)
    del R
    per_it = t_cyc / max(1, it)
    return t_setup + per_it * iters, t_setup, t_cyc, it, ref.num_threads()


def run_reference(args, rank, world):
    """The reference's own CPU implementation (oracle/_ref) on the host cores.  The
    first timed step is the full solve to 1e-8, measured: CPR setup + rgmres(50)
    until its own convergence test passes (rgmres.tpp:58-66 inner |g_j|, :118-123
    outer true residual).  Its iteration count then scales the remaining steps,
    which each time one whole restart cycle on the same setup (so that the run
    ends within minutes); warm-up steps run one cycle each.  `value` is the
    measured full solve; `sample_estimates_s` lists the per-step estimates."""
    unit = "s"
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdeco_ref.so was not built"}))
        return
    s = make_system()
    PREC["block_size"] = str(s.bs)
    t0 = time.perf_counter()
    R = ref.Cpr({"prec": PREC}, s.r, s.c, s.v, s.b)
    t_setup = time.perf_counter() - t0
    for _ in range(args.warmup):
        reference_cycle(R)
    t_region = time.perf_counter()
    full = R.solve(SOL)
    t_full = t_setup + full["time"]
    iters = full["iter"]
    Dr, Dc, Dv, Db = R.decoupled()
    import numpy as np
    true_rel = float(np.linalg.norm(Db - ref.spmv(Dr, Dc, Dv, full["x"])) / np.linalg.norm(Db))
    del Dr, Dc, Dv, Db
    estimates, cycles = [t_full], []
    for _ in range(max(0, args.steps - 1)):
        t_cyc, it = reference_cycle(R)
        cycles.append(t_cyc)
        estimates.append(t_setup + t_cyc / max(1, it) * iters)
    wall = time.perf_counter() - t_region
    threads = ref.num_threads()
    sample = (f"step 1: the reference's full solve, measured (CPR setup {t_setup:.1f} s + rgmres(50) to 1e-8 in "
              f"{iters} iterations, {full['time']:.1f} s); steps 2..{args.steps}: one whole restart cycle (50 "
              f"iterations) on the same setup, scaled to {iters} iterations")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": t_full, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / max(1, args.steps) * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "seed": SEED, "parallelism": "openmp"},
        "reference": {"iterations": iters, "res_rel": full["res_rel"], "true_rel_residual": true_rel,
                      "flag": full["flag"], "setup_s": t_setup, "solve_s": full["time"],
                      "cycle_s": cycles, "sample_estimates_s": estimates,
                      "timing": "value = the measured full solve (setup + rgmres to 1e-8); ms_per_step = wall time of "
                                "the timed steps / steps"},
        "cpu_baseline": {"value": t_full, "unit": unit, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": t_full, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# the batched workload: 64 systems of 10k-500k cells (--batch-systems / --batch-cells
# shrink it for profiler captures)
BATCH_NSYS, BATCH_LO, BATCH_HI = 64, 10_000, 500_000


def batch_workload():
    return (f"{BATCH_NSYS} two-phase systems, cells log-uniform {BATCH_LO // 1000}k-{BATCH_HI // 1000}k, "
            "8 uniform right-hand sides each; CPR seq 3 + GMRES(50)")


def batch_result(steps, warmup, ctx, rank, world, precisions=(32, 64)):
    """64 independent two-phase systems (cells log-uniform in 10k-500k), 8
    right-hand sides each, one lockstep CPR-GMRES solve per precision.  Under
    torchrun the systems are dealt round-robin to the ranks (replicas.deal:
    independent systems, no collective on the data path); the time is the max
    over ranks."""
    import torch
    import deco_b200 as d
    from deco_b200 import gen, replicas
    st = ctx.torch_stream
    r, c, v, ro, B, shapes = gen.batch(BATCH_NSYS, SEED, BATCH_LO, BATCH_HI, 2, 8)
    n_all, nnz_all = int(ro[-1]), len(c)
    if world > 1:
        r, c, v, ro, B = gen.batch_subset(r, c, v, ro, B, 8, replicas.deal(BATCH_NSYS, rank, world))
    n = int(ro[-1])
    dev = lambda a: torch.from_numpy(a).cuda()
    r_d, c_d, v_d, B_d = dev(r), dev(c), dev(v), dev(B)
    out = {}
    xs = {}
    for bits in precisions:
        rows = []
        for k in range(warmup + steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            A = d.CSR(n, n, r_d, c_d, v_d, ctx)
            Bt = d.Batch(PREC, A, ro, 8, precision=bits)
            X = Bt.solve(SOL, B_d)
            e1.record(st)
            e1.synchronize()
            if k >= warmup:
                rows.append((e0.elapsed_time(e1), Bt.result, Bt.iters.copy(), Bt.res_rel.copy(), Bt.widths.copy()))
            if k == warmup + steps - 1:
                xs[bits] = X
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
    if 64 not in xs or 32 not in xs:  # one precision only (--no-fp64 on the batched line)
        del xs, r_d, c_d, v_d, B_d
        return {"value_s": out["mixed"]["time_s"], "steps": steps, "warmup": warmup,
                "workload": f"{batch_workload()} ({n_all // 2} cells, {n_all} rows, {nnz_all} nnz)",
                "parallelism": f"systems dealt round-robin to {world} GPU(s), no collective", **out,
                "speedup_mixed_vs_fp64": None}
    # the mixed solutions' error against the float64 ones, per instance (columns of the multi-vector)
    X32, X64 = xs[32].view(-1, 8), xs[64].view(-1, 8)
    ro_t = torch.from_numpy(ro.astype("int64"))
    worst = 0.0
    for q in range(len(ro) - 1):
        a, e = int(ro_t[q]), int(ro_t[q + 1])
        num = (X32[a:e] - X64[a:e]).norm(dim=0)
        den = X64[a:e].norm(dim=0)
        worst = max(worst, float((num / den).max()))
    out["mixed"]["max_err_vs_fp64"] = replicas.max_over_ranks(worst, device="cuda")
    del xs, X32, X64, r_d, c_d, v_d, B_d
    return {"value_s": out["mixed"]["time_s"], "steps": steps, "warmup": warmup,
            "workload": f"{batch_workload()} ({n_all // 2} cells, {n_all} rows, {nnz_all} nnz)",
            "parallelism": f"systems dealt round-robin to {world} GPU(s), no collective", **out,
            "speedup_mixed_vs_fp64": out["fp64"]["time_s"] / out["mixed"]["time_s"]}


def bench_batch(args):
    """The batched workload alone, as its own JSON line."""
    import datetime
    import torch
    import deco_b200 as d
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = d.Context(int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_stream(ctx.torch_stream)
    b = batch_result(args.steps, args.warmup, ctx, rank, world, (32,) if args.no_fp64 else (32, 64))
    line = {"metric": f"batched CPR-GMRES time-to-1e-8 ({BATCH_NSYS} systems x 8 right-hand sides)",
            "value": b["value_s"], "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "scaling": "strong", "dtype": "f32+f64",
            "data": "synthetic", "config": {"workload": b["workload"], "seed": SEED, "parallelism": b["parallelism"]},
            **{k: b[k] for k in ("mixed", "fp64", "speedup_mixed_vs_fp64") if k in b}}
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


ADJOINT_WORKLOAD = ("64x64x32 two-phase grid from a seeded log-permeability field, bs 2, 262,144 rows; L = weighted "
                    "pressures at 20 seeded cells; CPR seq 3 + GMRES(50) to 1e-8 forward and adjoint")


def adjoint_result(steps, warmup, ctx):
    """64x64x32 log-permeability system: forward CPR-GMRES, adjoint CPR-GMRES on A^T
    and the on-pattern gradient dL/dA, float64 and mixed; plus the mixed gradient's
    error against the float64 one."""
    import numpy as np
    import torch
    import deco_b200 as d
    from deco_b200 import gen
    st = ctx.torch_stream
    p = gen.preset(5, SEED)
    s = gen.generate(p, with_logk=True)
    rng = np.random.default_rng(2024)
    obs = rng.choice(s.n // 2, 20, replace=False)
    g = np.zeros(s.n)
    g[2 * obs] = rng.random(20)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    r_d, c_d, v_d, b_d, g_d = dev(s.r), dev(s.c), dev(s.v), dev(s.b), dev(g)
    prec = dict(PREC, block_size="2")
    out = {}
    grads = {}
    for bits in (64, 32):
        rows = []
        for k in range(warmup + steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(st)
            A = d.CSR(s.n, s.n, r_d, c_d, v_d, ctx)
            b = b_d.clone()
            P = d.CPR(prec, A, b, bits)
            S = d.SOL(SOL, A, P, b, precision=bits)
            ev[1].record(st)
            A0 = d.CSR(s.n, s.n, r_d, c_d, v_d, ctx)
            J = d.ADJ(prec, A0, bits)
            lam = J.solve(SOL, g_d)
            ev[2].record(st)
            grad = A0.grad_pattern(lam, S.x)
            ev[3].record(st)
            ev[3].synchronize()
            if k >= warmup:
                rows.append((ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3]),
                             S.iter, J.iter))
            if k == warmup + steps - 1:
                grads[bits] = grad.clone()
            del S, P, A, J, A0, lam, grad
        f = statistics.mean(t[0] for t in rows)
        a = statistics.mean(t[1] for t in rows)
        gk = statistics.mean(t[2] for t in rows)
        alg = 12 * s.nnz + 8 * (s.n + 1) + 8 * s.n
        out["fp64" if bits == 64 else "mixed"] = {
            "time_s": (f + a + gk) / 1e3, "forward_ms": f, "adjoint_ms": a, "adjoint_over_forward": a / f,
            "grad_kernel_ms": gk, "grad_kernel_gbs": alg / gk / 1e6, "forward_iterations": rows[-1][3],
            "adjoint_iterations": rows[-1][4]}
    out["mixed"]["grad_err_vs_fp64"] = float((grads[32] - grads[64]).norm() / grads[64].norm())
    return {"value_s": out["fp64"]["time_s"], "steps": steps, "warmup": warmup, "workload": ADJOINT_WORKLOAD, **out}


def bench_adjoint(args):
    import torch
    import deco_b200 as d
    ctx = d.Context(0)
    torch.cuda.set_stream(ctx.torch_stream)
    a = adjoint_result(args.steps, args.warmup, ctx)
    print(json.dumps({"metric": "adjoint gradient time (forward + transpose CPR-GMRES + dL/dA on pattern)",
                      "value": a["value_s"], "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                      "higher_is_better": False, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": a["workload"], "seed": SEED}, "fp64": a["fp64"], "mixed": a["mixed"]}))


CONFIG2_WORKLOAD = ("100x100x50 three-phase grid, bs=3, 1,500,000 rows, layered lognormal k sigma 2 (kz/kx 0.1) + 1% "
                    "random long-range fault connections; CPR(FSAI + FSAI, seq 3, quasiimpes_GE, CPD) + right GMRES(50)"
                    ", true relative residual 1e-8")


def config2_result(steps, warmup, ctx):
    """The 1.5M-row three-phase system: float64 and mixed-precision time to 1e-8
    (setup + solve, from pristine HBM copies), iterations, float64 true residuals
    on the decoupled and on the original system, the mixed solution's error against
    the float64 one, and the reference build's iteration count."""
    import torch
    import deco_b200 as d
    from deco_b200 import gen
    st = ctx.torch_stream
    s = gen.generate(gen.preset(2, SEED))
    prec = dict(PREC, block_size=str(s.bs))
    dev = lambda a: torch.from_numpy(a).cuda()
    r_d, c_d, v_d, b_d = dev(s.r), dev(s.c), dev(s.v), dev(s.b)
    out, xs = {}, {}
    for bits in (64, 32):
        rows = []
        for k in range(warmup + steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            A = d.CSR(s.n, s.n, r_d, c_d, v_d, ctx)
            b = b_d.clone()
            P = d.CPR(prec, A, b, precision=bits)
            S = d.SOL(SOL, A, P, b, precision=bits)
            e1.record(st)
            e1.synchronize()
            if k >= warmup:
                true_rel = (A.residual(b, S.x).norm() / b.norm()).item()
                rows.append(dict(ms=e0.elapsed_time(e1), iter=S.iter, flag=S.flag, true_rel=true_rel,
                                 orig_rel=S.res_rel_orig, setup_ms=P.timings()["Prec"], solve_ms=S.time_ms))
            if k == warmup + steps - 1:
                xs[bits] = S.x.clone()
            del S, P, A, b
        last = rows[-1]
        out["fp64" if bits == 64 else "mixed"] = {
            "time_s": statistics.mean(r["ms"] for r in rows) / 1e3, "iterations": last["iter"], "flag": last["flag"],
            "true_rel_residual": last["true_rel"], "original_system_rel_residual": last["orig_rel"],
            "setup_ms": last["setup_ms"], "solve_ms": last["solve_ms"],
            "ms_per_iteration": last["solve_ms"] / max(1, last["iter"])}
    out["mixed"]["err_vs_fp64"] = float((xs[32] - xs[64]).norm() / xs[64].norm())
    rec = reference_record(2)
    return {"steps": steps, "warmup": warmup, "workload": CONFIG2_WORKLOAD, "rows": s.n, "nnz": s.nnz, **out,
            "speedup_mixed_vs_fp64": out["fp64"]["time_s"] / out["mixed"]["time_s"],
            "reference_iterations": rec["iterations"] if rec else None,
            "reference_source": ("tests/golden/reference_runs.json: the reference build's rgmres(50) on this system "
                                 f"({rec['omp_threads']} OpenMP threads)") if rec else None}


TRAFFIC = os.path.join(ROOT, "profiles", "dram_traffic.json")


def dram_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary profiles/dram_traffic.json, keyed by the kernel's name; None if that
    kernel has no capture.  Each entry names the capture and workload it came from."""
    try:
        with open(TRAFFIC) as f:
            e = json.load(f).get("kernels", {}).get(kernel)
    except (OSError, ValueError):
        return None, None
    if not e:
        return None, None
    return float(e["dram_bytes_per_launch"]), e.get("source")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="deco", choices=["deco", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-config2", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--sub-steps", type=int, default=2,
                    help="timed steps of the config2 / adjoint / batch objects (one warm-up each)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only the per-kernel timings (for profiler captures on a smaller --config)")
    ap.add_argument("--batch-systems", type=int, default=64, help="systems of the batched workload")
    ap.add_argument("--batch-cells", default="10000,500000", help="LO,HI: cell counts of the batched systems")
    ap.add_argument("--config", type=int, default=3, help="system preset (3 = the 200x200x100 benchmark workload)")
    ap.add_argument("--grid", default=None,
                    help="NX,NY,NZ: the preset's distributions on a smaller grid (profiler captures)")
    ap.add_argument("--workload", default="solve", choices=["solve", "batch", "adjoint", "spmv"],
                    help="solve: the headline single-system solve; batch: 64 systems x 8 right-hand sides; "
                         "adjoint: the 64x64x32 log-permeability gradient; "
                         "spmv: the SpMV kernels alone")
    args = ap.parse_args()
    global CONFIG, GRID, BATCH_NSYS, BATCH_LO, BATCH_HI
    BATCH_NSYS = args.batch_systems
    BATCH_LO, BATCH_HI = (int(t) for t in args.batch_cells.split(","))
    CONFIG = args.config
    GRID = tuple(int(t) for t in args.grid.split(",")) if args.grid else None
    if args.workload == "batch":
        return bench_batch(args)
    if args.workload == "adjoint":
        return bench_adjoint(args)
    if args.workload == "spmv":
        return bench_spmv(args)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import datetime

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
    keep = {}

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
                    setup_ms=ph["Prec"], solve_ms=S.time_ms, setup_phases_ms={k: round(v, 2) for k, v in ph.items()},
                    phases_ms=S.phases_ms)
        if not host:
            keep[bits] = S.x
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
        args.no_config2, args.no_batch, args.no_adjoint = True, True, True
    for _ in range(args.warmup):
        step(32)
    clk = Clocks(local)
    ms_mixed, info_mixed, wall_mixed, launches = timed(32, args.steps)
    clocks = clk.stop()
    fp64 = None
    err_vs_fp64 = None
    if not args.no_fp64:
        step(64)  # warm the float64 kernels
        ms64, info64, _, _ = timed(64, args.steps)
        fp64 = {"time_s": ms64 / 1e3, "iterations": info64[-1]["iter"], "true_rel_residual": info64[-1]["true_rel"],
                "original_system_rel_residual": info64[-1]["orig_rel"],
                "setup_ms": info64[-1]["setup_ms"], "solve_ms": info64[-1]["solve_ms"],
                "ms_per_iteration": info64[-1]["solve_ms"] / max(1, info64[-1]["iter"]),
                "step_ms": [round(i["ms"], 1) for i in info64], "setup_phases_ms": info64[-1]["setup_phases_ms"]}
        if 32 in keep and 64 in keep:
            err_vs_fp64 = float((keep[32] - keep[64]).norm() / keep[64].norm())
    keep.clear()
    e2e = None
    if not args.no_e2e:
        step(32, host=True)
        ms_e2e, _, _, _ = timed(32, args.steps, host=True)
        h2d = (n + 1) * 4 + nnz * 4 + nnz * 8 + n * 8
        e2e = {"value": ms_e2e / 1e3, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * 8}

    # ---- roofline of the dominant kernel (float32 product of A) and the other hot kernels
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

    def matrix_bytes(nz, blocks, vb, ib=4):
        """Bytes of one pass over a matrix in the layout the product reads: the
        cell-block copy (one column index of ib bytes per bs x bs block -- 4, or the
        1- or 2-byte offset code of the padded copy -- and block-row pointers) when
        there is one, else CSR (4-byte index + value per entry)."""
        bsz, nblk = blocks
        if bsz:
            return nblk * ib + nblk * bsz * bsz * vb + 4 * (n // bsz + 1)
        return nz * (4 + vb) + 4 * (n + 1)

    cb = A.slot_codes[0] if A.padded else 4  # bytes per block column the padded product reads
    fmt = ("cell-block (bs %d)" % A.blocks[0] if A.blocks[0] else "CSR") + \
        (", %d padded slots per cell" % A.padded if A.padded else "") + \
        (", %d-byte column offset codes" % cb if A.padded and cb < 4 else "")
    ms = kernel_ms(lambda: A.apply_f32(x32, y32))
    alg32 = matrix_bytes(nnz, A.blocks, 4, cb) + 4 * n + 4 * n
    kernels["spmv_A_f32"] = {"ms": ms, "gbs": alg32 / ms / 1e6, "alg_bytes": alg32, "format": fmt,
                             "subwarp": A.subwarp}
    ms = kernel_ms(lambda: A.apply(x64, y64))
    alg64 = matrix_bytes(nnz, A.blocks, 8, cb) + 8 * n + 8 * n
    kernels["spmv_A_f64"] = {"ms": ms, "gbs": alg64 / ms / 1e6, "alg_bytes": alg64, "format": fmt}
    fb, kl, ku = Fg.blocks
    ms = kernel_ms(lambda: Fg.apply(x64, y64))
    cl, cu = (b_ if b_ else 4 for b_ in Fg.slot_codes)
    algF = matrix_bytes(nzF, (fb, kl), 8, cl) + matrix_bytes(nzF, (fb, ku), 8, cu) + 8 * n + 2 * 8 * n + 8 * n
    kernels["fsai_apply_global_f64"] = {"ms": ms, "gbs": algF / ms / 1e6, "alg_bytes": algF, "nnz_factor": nzF,
                                        "format": ("cell-block (bs %d)" % fb if fb else "CSR")
                                        + (", %d/%d padded slots" % Fg.padded if Fg.padded[0] else ""),
                                        "note": "the intermediate FL x (64 MB) stays in L2 between the two products"}
    plans = {"A_f64": A.product_plan(64)}
    del P64
    A32 = d.CSR(n, n, r_d, c_d, v_d, ctx)
    P32 = d.CPR(PREC, A32, b_d.clone(), precision=32)
    plans["A_f32"] = A32.product_plan(32)
    Fg32 = P32.fsai(0)
    fb, kl, ku = Fg32.blocks
    # as the mixed-precision CPR applies it: float32 x, intermediate and y
    ms = kernel_ms(lambda: Fg32.apply_f32(x32, y32))
    cl, cu = (b_ if b_ else 4 for b_ in Fg32.slot_codes)
    algF32 = matrix_bytes(nzF, (fb, kl), 4, cl) + matrix_bytes(nzF, (fb, ku), 4, cu) + 4 * n + 2 * 4 * n + 4 * n
    kernels["fsai_apply_global_f32"] = {"ms": ms, "gbs": algF32 / ms / 1e6, "alg_bytes": algF32,
                                        "format": "cell-block (bs %d)" % fb if fb else "CSR",
                                        "vectors": "float32 (deco_fsai_apply_f32)"}
    # through the reference-shaped interface: float64 x and y around the float32 factor
    ms = kernel_ms(lambda: Fg32.apply(x64, y64))
    algF32d = matrix_bytes(nzF, (fb, kl), 4, cl) + matrix_bytes(nzF, (fb, ku), 4, cu) + 8 * n + 2 * 4 * n + 8 * n
    kernels["fsai_apply_global_f32_f64io"] = {"ms": ms, "gbs": algF32d / ms / 1e6, "alg_bytes": algF32d,
                                              "format": "cell-block (bs %d)" % fb if fb else "CSR",
                                              "vectors": "float64 (deco_fsai_apply)"}
    del P32, A32, A, b, x64, y64, x32, y32
    # the orthogonalisation (dot pass + update pass of every Arnoldi step), timed by CUDA
    # events around each step's phases inside one mixed solve (DECO_PROFILE=1).  Bytes of
    # step j with a float32 basis: 2 (j + 3) 4n (each pass reads the j + 1 columns and w;
    # the dot pass also u_j, the update pass writes u_{j+1}); a cycle of m steps
    # averages j over 0..m-1.
    if args.steps > 0:
        os.environ["DECO_PROFILE"] = "1"
        try:
            info = step(32)
        finally:
            os.environ.pop("DECO_PROFILE", None)
        keep.clear()
        m = int(SOL["restart"])
        it = info["iter"]
        full, rest = divmod(it, m)
        steps_j = [j for _ in range(full) for j in range(m)] + list(range(rest))
        alg_o = sum(2 * (j + 3) * 4 * n for j in steps_j) / max(1, len(steps_j))
        t_o = info["phases_ms"]["ortho"] / max(1, it)
        kernels["orthogonalisation_f32"] = {
            "ms": t_o, "gbs": alg_o / t_o / 1e6, "alg_bytes": alg_o,
            "what": "arnoldi_dots + arnoldi_update per Arnoldi step, float32 basis, mean over the solve's steps "
                    f"(restart {m}, {it} iterations)",
            "phase_ms_per_iteration": {k: v / max(1, it) for k, v in info["phases_ms"].items()}}
        # each pass alone: (j + 3) 4n bytes per step (the j + 1 columns, w, and u_j read or u_{j+1} written)
        t_d = info["phases_ms"]["dots"] / max(1, it)
        for name, t, what in (("arnoldi_dots_f32", t_d, "dot pass (arnoldi_dots / arnoldi_dots_bulk)"),
                              ("arnoldi_update_f32", t_o - t_d, "update pass (arnoldi_update)")):
            kernels[name] = {"ms": t, "gbs": (alg_o / 2) / t / 1e6, "alg_bytes": alg_o / 2,
                             "what": f"{what} per Arnoldi step, float32 basis, mean over the solve's steps"}
    for k in kernels.values():
        k["frac_of_peak"] = k["gbs"] / peak
    dom = kernels["spmv_A_f32"]
    padded = "padded slots per cell" in dom["format"]
    kname = ("ell2_kernel<%d, float>" % int(dom["format"].split(", ")[1].split()[0])) if padded else None
    traffic, tsrc = dram_traffic(kname) if kname else (None, None)
    roofline = {"bound": "hbm", "achieved": dom["gbs"], "peak": peak, "unit": "GB/s", "frac": dom["gbs"] / peak,
                "traffic": traffic, "traffic_source": tsrc,
                "kernel": ("deco::%s (2x2 cell blocks, padded slots per cell)" % kname if kname else
                           "deco::bsr2_pair_kernel / bsr_kernel / spmv_kernel (float32)")
                + " on A (%d rows, %d nnz, float32 values)" % (n, nnz),
                "algorithmic_bytes": "the unpadded cell-block layout's bytes, block columns in the padded copy's "
                                     "encoding (1-byte offset codes when it has them); padding slots count against "
                                     "the kernel",
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}

    rec3 = reference_record(CONFIG) if GRID is None else None
    ref_iters = rec3["iterations"] if rec3 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                iters = ref_iters or (fp64["iterations"] if fp64 else info_mixed[-1]["iter"])
                total, t_setup, t_cyc, cyc_it, threads = reference_sample(s, iters)
                cpu = {"value": total, "unit": "s", "cores": threads, "kind": "reference",
                       "sample": f"reference CPR setup on the full system ({t_setup:.1f} s) + one whole restart "
                                 f"cycle ({cyc_it} GMRES iterations, {t_cyc:.2f} s), the cycle scaled to the "
                                 f"reference's {iters} iterations to 1e-8",
                       "setup_s": t_setup, "cycle_s": t_cyc, "s_per_iteration": t_cyc / max(1, cyc_it)}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}
    del s

    sub = {}
    if not args.no_config2 and GRID is None:
        sub["config2"] = config2_result(args.sub_steps, 1, ctx)
    if not args.no_adjoint and GRID is None:
        sub["adjoint"] = adjoint_result(args.sub_steps, 1, ctx)
    if not args.no_batch and GRID is None:
        sub["batch"] = batch_result(args.sub_steps, 1, ctx, rank, world)

    last = info_mixed[-1]
    out = {
        "metric": METRIC, "value": ms_mixed / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if GRID is None else "grid %dx%dx%d of preset %d" % (GRID + (CONFIG,)),
                   "seed": SEED, "precision": "mixed: float32 CPR + float32 Krylov basis, "
                   "float64 dots/Hessenberg/true residual/solution", "l2": "inputs larger than L2 (1.3 GB matrix)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "mixed": {"iterations": last["iter"], "true_rel_residual": last["true_rel"], "flag": last["flag"],
                  "original_system_rel_residual": last["orig_rel"], "err_vs_fp64": err_vs_fp64,
                  "setup_ms": last["setup_ms"], "solve_ms": last["solve_ms"],
                  "ms_per_iteration": last["solve_ms"] / max(1, last["iter"]),
                  "step_ms": [round(i["ms"], 1) for i in info_mixed], "setup_phases_ms": last.get("setup_phases_ms")},
        "fp64": fp64,
        "reference_iterations": ref_iters,
        "reference_iterations_source": ("tests/golden/reference_runs.json: the reference build's rgmres(50) on this "
                                        f"system ({rec3['omp_threads']} OpenMP threads); --impl reference measures it "
                                        "live") if rec3 else None,
        "speedup_mixed_vs_fp64": (fp64["time_s"] / (ms_mixed / 1e3)) if fp64 else None,
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": kernels,
        # the product the CPR setup's autotuner chose for A: (padded | cells | csr, lanes per cell or row)
        "product_plans": plans,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        **sub,
    }
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
