#!/usr/bin/env python
"""Benchmark of the IPM hot path on the 2-D Euler workload (200,000 cells).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: 2-D Euler (gamma 1.4), seeded jittered triangle mesh of 400 x 250
rectangles x 2 = 200,000 cells on [0,1]^2, uncertain Sod-type interface
(x = 0.5 + 0.05 xi1, left density 1 + 0.1 xi2), total-degree-5 Legendre basis
(21 moments x 4 states = 84 duals per cell), 10 x 10 tensor Gauss nodes,
guarded Newton to |g| < 1e-10. Synthetic, seeded; no dataset is involved.

A step is one explicit time step of the hot path (closure for every cell,
nodal reconstruction, kinetic flux, update). `value` is cell-steps/s of the
chosen form with the state resident in HBM; `e2e` is the same metric through
the C ABI with the state uploaded from and downloaded to pinned host memory
every step (uqc_step_host: one call per step, the copies in chunks beside the
convergence check and the duals' download beside the update; every step starts
cold, with no held factors or lists, as after any state upload). The plain FP64 form is timed in the same run (`fp64`), from the same
state, and the chosen form's moments are compared with it after the K steps.

`serving`: p50/p99 request latency and aggregate cell-steps/s of the request
server (continuous batching) on the first requests of the seeded serving
stream, submitted at their Poisson arrival times.

N > 1 (torchrun): spatial sharding, weak scaling. The mesh grows with N (400 N x
250 rectangles x 2 = N x 200,000 cells) and is split into N blocks of about
200,000 cells (recursive coordinate bisection: stripes along x), a rank per GPU
(uqcreator_b200.shard.ShardedSolver). A step is the closure of the rank's
cells, an NCCL all-reduce MIN of the step size (8 bytes), the halo exchange of
the nodal states of the cells next to the stripe boundaries (NCCL send/recv on
the solver's stream) and the update; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-steps/s mixed vs FP64 GPU at ≤1e-6 moment err; p50/p99 request latency"
WORKLOAD = dict(nx=400, ny=250, degree=5, nquad=10, dim_xi=2)
SAMPLE_NY = 10           # CPU sample: a 400 x 10 strip of the same mesh construction (8,000 cells)
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def work_per_cell_step(n_states, n_total, n_quad, n_faces=3):
    """Algorithmic FP64-equivalent flops of the closure kernel, per unit:
    F_it per Newton iteration = 2 nQ n^2 (Hessian) + 4 nQ n (ansatz + gradient)
    + n^3/3 + 2 n^2 (Cholesky + solves); 4 nQ n per extra gradient evaluation
    (initial check, line-search trial); epilogue 4 nQ n (reconstruction +
    re-projection)."""
    n = n_states * n_total
    f_it = 2 * n_quad * n * n + 4 * n_quad * n + n ** 3 / 3 + 2 * n * n
    f_grad = 4 * n_quad * n
    f_epi = 4 * n_quad * n
    f_flux = n_faces * 2 * n_quad * n
    return f_it, f_grad, f_epi, f_flux


# Where each form computes the Newton system's parts: the Hessian assembly
# (2 nQ n^2 flops per iteration: FP64 form on FP64 units, the mixed form on the
# tensor cores when uqc_info.mixed_form == 2, else FP32 CUDA cores), the
# factorisation and solves (n^3/3 + 2 n^2: FP64, or FP32 in the mixed form) and
# everything else (ansatz, gradients, line search, epilogue: FP64 in both forms).
def hessian_unit(form, mixed_form):
    return "fp64" if form == "fp64" else ("tensor" if mixed_form == 2 else "fp32")


FACTOR_UNIT = {"fp64": "fp64", "mixed": "fp32"}
# DRAM bytes (read + write) of the closure phase per cell that takes Newton
# iterations, from ncu captures of the 5th step of a 60,000-cell case of the
# same workload (6,457 active cells; profiles/closure_rounds_euler2d.md):
# FP64 form k_closure 9.58 MB; mixed form (rounds) k_chord rounds 0-1, k_hess_tc
# and k_invert_sweep round 0: 358.9 MB, mostly each active cell's held FP32
# inverse (28 KB) read by the chord kernel.
CLOSURE_DRAM_BYTES_PER_ACTIVE_CELL = {"fp64": 9.576e6 / 6457, "mixed": 358.9e6 / 6457}


def closure_roofline(form, n_states, n_total, n_quad, cells, steps, ref_info, closure_ms, measured, active_cells, mixed_form=0):
    """T_bound of the closure phase: max over units of (work on that unit /
    its measured peak); achieved = algorithmic work / measured time, peak =
    work / T_bound, frac = T_bound / time. Work uses the FP64 form's Newton
    iteration and line-search counts (ref_info) for both forms, so the mixed
    form is not credited for the extra iterations of its inexact Newton."""
    n = n_states * n_total
    iters = ref_info["newton_iterations"]
    grads = iters + ref_info["line_search_trials"] + cells * steps    # + the initial test of every cell
    work = {"fp64": 0.0, "fp32": 0.0, "tensor": 0.0}
    work[hessian_unit(form, mixed_form)] += iters * 2.0 * n_quad * n * n
    work[FACTOR_UNIT[form]] += iters * (n ** 3 / 3.0 + 2.0 * n * n)
    work["fp64"] += grads * 4.0 * n_quad * n + cells * steps * 4.0 * n_quad * n
    hbm, bf16, src = peaks()
    peak = {"fp64": measured.get("fp64_tflops"), "fp32": measured.get("fp32_tflops"), "tensor": bf16}
    t_unit = {u: (w / steps) / (peak[u] * 1e12) * 1e3 for u, w in work.items() if w > 0 and peak[u]}
    total = sum(work.values()) / steps
    traffic = CLOSURE_DRAM_BYTES_PER_ACTIVE_CELL[form] * active_cells
    t_unit["hbm"] = traffic / (hbm * 1e9) * 1e3
    bound = max(t_unit, key=t_unit.get)
    t_bound = t_unit[bound]
    return {"bound": bound, "achieved": total / (closure_ms / 1e3) / 1e12, "peak": total / (t_bound / 1e3) / 1e12,
            "unit": "TFLOP/s", "frac": t_bound / closure_ms, "traffic": traffic,
            "traffic_unit": "bytes per closure phase (scaled from the form's ncu capture by its active cells)",
            "t_bound_ms": t_unit, "closure_ms_per_launch": closure_ms, "flops_per_launch": total,
            "peaks_tflops": {**peak, "tensor_source": f"bf16 {src} (MEASURED_PEAKS.json)"},
            "hbm_peak_gbs": hbm, "kernels": "closure phase: k_check + k_closure (FP64 form); k_check + k_chord / k_hess_tc / k_invert_sweep rounds + the FP64 fallback pass (mixed form)"}


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.p is None:
            return
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        # host scalars over gloo, device buffers (the step, the halos) over NCCL
        dist.init_process_group("cpu:gloo,cuda:nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_run(steps, warmup, min_seconds=None, ny=SAMPLE_NY):
    """UQCreator's own code (oracle/_ref, OpenMP build) on a strip of the workload."""
    from oracle import refharness
    from uqcreator_b200 import workloads as W
    toml = W.euler2d(nx=WORKLOAD["nx"], ny=ny)
    r = refharness.RefSolver(toml, "Euler2D", [0.5, 1.0, 1.0, 0.125, 0.1], bounds=(3, 12), mesh2d=W.mesh_for(toml),
                             variant="omp", newton="guarded")
    r.init_state()
    for _ in range(warmup):
        r.step(1)
    t0 = time.perf_counter()
    done = 0
    while True:
        r.step(1)
        done += 1
        el = time.perf_counter() - t0
        if (min_seconds is None and done >= steps) or (min_seconds is not None and el >= min_seconds and done >= 1):
            break
    cores = os.cpu_count()
    return dict(value=r.n_cells * done / el, unit="cell-steps/s", cores=cores, kind="reference",
                sample=f"UQCreator C++ (OpenMP, {cores} threads) on a {WORKLOAD['nx']}x{ny}x2 = {r.n_cells}-cell strip of the same "
                       f"workload after {warmup} warm-up steps, {done} steps in {el:.1f} s"), r.n_cells, done, el


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import refharness
    if not refharness.available("omp"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libuqcref_omp.so not built (make -C oracle/ref)"}))
        return
    cb, cells, done, el = cpu_reference_run(args.steps, args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": done,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / done, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "euler2d_sod_2u_deg5_q10x10", "cells": cells, "sample_of_cells": 200000},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def oracle_strip_errors(forms, steps=5):
    """Error of each GPU form against the FP64 oracle (oracle/uqc_oracle.c) on
    the 400 x 10 x 2 = 8,000-cell strip of the benchmark mesh construction (same
    x resolution), `steps` steps from the initial state; outside the timed
    region. Returns {form: {"moment_rel_l1", "mean_var_rel_l1_max"}}."""
    from oracle.oracle import Oracle
    from uqcreator_b200 import Solver, workloads as W, FP64, MIXED
    toml = W.euler2d(nx=WORKLOAD["nx"], ny=SAMPLE_NY)
    o = Oracle(toml, W.mesh_for(toml))
    o.init_state()
    o.step(steps)
    uo = o.get_state()[0]
    mvo = o.mean_var()
    area = o.geometry()["area"][:, None]
    out = {"sample": f"{WORKLOAD['nx']}x{SAMPLE_NY}x2 = {o.n_cells}-cell strip, {steps} steps from the initial state"}
    for form in forms:
        s = Solver(toml)
        s.set_precision(MIXED if form == "mixed" else FP64)
        s.init_state()
        s.step(steps)
        u = s.download_state()[0]
        mv = s.mean_var()
        s.close()
        mv_err = (np.abs(mv - mvo) * area).sum(0) / (np.abs(mvo) * area).sum(0)
        out[form] = {"moment_rel_l1": float(np.abs(u - uo).sum() / np.abs(uo).sum()),
                     "mean_var_rel_l1_max": float(mv_err.max())}
    return out


def measure_peaks(device_index=0):
    """FP64 and FP32 (no TF32) GEMM throughput of cuBLAS on this GPU (torch.matmul,
    8192^3, best of 5 after a warm-up, CUDA events): the CUDA-core ceilings of
    the FP64 and FP32 parts of the closure, measured in the same run."""
    import torch
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for name, dt, n in (("fp64_tflops", torch.float64, 8192), ("fp32_tflops", torch.float32, 8192)):
            a = torch.randn(n, n, dtype=dt, device=f"cuda:{device_index}")
            b = torch.randn(n, n, dtype=dt, device=f"cuda:{device_index}")
            torch.matmul(a, b)
            best = 1e30
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(); torch.matmul(a, b); e1.record(); torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            out[name] = 2.0 * n ** 3 / (best / 1e3) / 1e12
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    out["how"] = "cuBLAS GEMM 8192^3 via torch.matmul (TF32 off), best of 5, CUDA events"
    return out


def run_serving(args, precision):
    """p50/p99 request latency: the first `serve_requests` requests of the seeded
    serving stream (Poisson arrivals, Burgers 1-D 200-20k cells / Euler 2-D
    10k-200k cells, 5-40 steps each) submitted at their arrival times to the
    request server and driven to completion."""
    from uqcreator_b200 import workloads as W
    from uqcreator_b200.serve import Server, latency_percentiles
    stream = W.serving_stream(args.serve_requests, args.serve_rate, seed=11)
    srv = Server(budget_bytes=int(args.serve_budget_gb * (1 << 30)), max_active=16, steps_per_slice=4,
                 policy=args.serve_policy, max_stepping=args.serve_max_stepping)
    if args.serve_policy == 1:
        srv.set_option("aging", args.serve_aging)
    import threading
    ids, failures = [], []

    def front_end():
        # requests arrive on a thread of their own (their solvers are built
        # there), the main thread runs the scheduling passes
        try:
            for arr, kind, toml in stream:
                wait = arr - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                ids.append((srv.submit(toml, precision), kind))
        except Exception as e:    # reported after the loop
            failures.append(e)

    t0 = time.perf_counter()
    th = threading.Thread(target=front_end, daemon=True)
    th.start()
    while True:
        alive = th.is_alive()
        q, r, _ = srv.progress()
        if not alive and q == 0 and r == 0:
            break
    th.join()
    if failures:
        raise failures[0]
    el = time.perf_counter() - t0
    res = [srv.result(k, mean_var=False) for k, _ in ids]
    srv.close()
    ok = [x for x in res if x["state"] == "done"]
    lat = [x["latency_ms"] for x in ok]
    queue = [x["queue_ms"] for x in ok]
    service = [x["service_ms"] for x in ok]
    out = {"requests": len(res), "failed": len(res) - len(ok), "arrival_rate_per_s": args.serve_rate,
           "elapsed_s": el, "cell_steps_per_s": sum(x["n_cells"] * x["steps"] for x in ok) / el,
           "stream": "seeded serving stream (seed 11): Poisson arrivals, Burgers1D 200-20k cells deg 2-9, "
                     "Euler2D 10k-200k cells deg 2-5, offsets U[0.05,0.3], 5-40 steps per request",
           "budget_gb": args.serve_budget_gb, "max_active": 16, "steps_per_slice": 4,
           "policy": "shortest remaining time first" if args.serve_policy == 1 else "round robin",
           "max_stepping": args.serve_max_stepping, "aging": args.serve_aging if args.serve_policy == 1 else None}
    out.update(latency_percentiles(lat))
    out["queue"] = latency_percentiles(queue)
    out["service"] = latency_percentiles(service)
    for kind in ("burgers1d", "euler2d"):
        lk = [x["latency_ms"] for x, (_, k) in zip(res, ids) if k == kind and x["state"] == "done"]
        out[kind] = dict(n=len(lk), **latency_percentiles(lk))
    return out


def run_b200_sharded(args, rank, world, local):
    """The bench line at N > 1: the 2-D Euler workload on an N-times wider mesh,
    one stripe of cells per rank, halo exchange and step all-reduce over NCCL."""
    import torch
    import torch.distributed as dist
    from uqcreator_b200 import workloads as W, FP64, MIXED
    from uqcreator_b200.shard import ShardedSolver

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    toml = W.euler2d(**dict(WORKLOAD, nx=WORKLOAD["nx"] * world))
    ss = ShardedSolver(toml)
    ss.init_state()
    sh = ss.shard
    s = sh.solver
    forms = ["fp64"]
    try:
        s.set_precision(MIXED)
        s.set_precision(FP64)
        forms.append("mixed")
    except Exception:
        pass
    chosen = "mixed" if "mixed" in forms else "fp64"
    warm = ss.step(args.warmup, with_info=True)
    u0, l0, v0 = s.download_state()
    results = {}
    for form in forms:
        s.set_precision(MIXED if form == "mixed" else FP64)
        s.upload_state(u0, l0, v0, t=warm["t"])
        ss.step(args.warmup)
        torch.cuda.synchronize()
        barrier(world)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(dev) as ck:
            ev0.record(sh.stream)
            info = ss.step(args.steps, with_info=True)
            ev1.record(sh.stream)
            torch.cuda.synchronize()
        barrier(world)
        results[form] = dict(ms=max_over_ranks(ev0.elapsed_time(ev1), world), info=info, clocks=ck.summary(),
                             launches=s.last_launch_count() * args.steps, state=s.download_state())
    no = sh.n_owned
    err = None
    if chosen != "fp64":
        uf, ub = results["fp64"]["state"][0][:no], results[chosen]["state"][0][:no]
        area = s.geometry()["area"][:no, None, None]
        num = torch.tensor((np.abs(ub - uf) * area).sum(axis=(0, 2)))
        den = torch.tensor((np.abs(uf) * area).sum(axis=(0, 2)))
        dist.all_reduce(num)
        dist.all_reduce(den)
        err = float((num / den).max())
    # end to end through the public API: the rank's state from and to pinned host memory every step
    s.set_precision(MIXED if chosen == "mixed" else FP64)
    s.upload_state(u0, l0, v0, t=warm["t"])
    hu = torch.empty(u0.shape, dtype=torch.float64, pin_memory=True).numpy()
    hl = torch.empty(l0.shape, dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty(v0.shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    hu[...] = u0; hl[...] = l0; hv[...] = v0
    e2e_steps = max(1, min(args.steps, 10))
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    tcur = warm["t"]
    for _ in range(e2e_steps):
        s.upload_state(hu, hl, hv, t=tcur)
        tcur = ss.step(1, with_info=True)["t"]
        s.download_state(out=(hu, hl, hv))
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(1e3 * (time.perf_counter() - t0), world)
    cells = sh.plan["n_global"]
    r = results[chosen]
    value = cells * args.steps / (r["ms"] / 1e3)
    fp64_value = cells * args.steps / (results["fp64"]["ms"] / 1e3)
    local_bytes = s.n_cells * s.n_states * s.n_total * 8
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if chosen == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"euler2d_sod_2u_deg5_q10x10 on a {WORKLOAD['nx'] * world}x{WORKLOAD['ny']} mesh",
                   "cells": cells, "cells_per_rank": no, "halo_rows_per_step": sh.plan["n_send"],
                   "duals_per_cell": s.n_states * s.n_total, "nodes": s.n_quad, "form": chosen,
                   "parallelism": f"spatial{world} (stripes, NCCL halo exchange + all-reduce MIN)",
                   "l2": "inputs larger than L2"},
        "fp64": {"value": fp64_value, "ms_per_step": results["fp64"]["ms"] / args.steps},
        "chosen_over_fp64": value / fp64_value,
        "moment_rel_l1_vs_fp64": err,
        "roofline": None,
        "e2e": {"value": cells * e2e_steps / (e2e_ms / 1e3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": world * (2 * local_bytes + 4 * s.n_cells),
                "d2h_bytes_per_step": world * (2 * local_bytes + 4 * s.n_cells), "steps": e2e_steps},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(line))
    ss.close()


def run_b200(args, rank, world, local):
    if world > 1 or args.sharded:
        return run_b200_sharded(args, rank, world, local)
    import torch
    from uqcreator_b200 import Solver, workloads as W, FP64, MIXED

    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream(device=dev)
    toml = W.euler2d(**WORKLOAD)
    s = Solver(toml, stream=stream.cuda_stream)
    s.init_state()
    forms = ["fp64"]
    try:
        s.set_precision(MIXED)
        s.set_precision(FP64)
        forms.append("mixed")
    except Exception:
        pass
    chosen = "mixed" if "mixed" in forms else "fp64"
    # warm-up (FP64: the first step from the initial state is the expensive one)
    warm = s.step(args.warmup)
    u0, l0, v0 = s.download_state()
    results = {}
    tuned = {}
    for form in forms:
        s.set_precision(MIXED if form == "mixed" else FP64)
        if not args.no_autotune:
            # launch shapes and schedule of this form from the project's autotuner
            # (coordinate descent, timed on this state; untimed)
            from uqcreator_b200.autotune import autotune
            s.upload_state(u0, l0, v0, t=warm["t"])
            s.step(args.warmup)
            tuned[form] = autotune(s, steps=3, repeats=2, warmup=args.warmup, cache=None)["best"]
        s.upload_state(u0, l0, v0, t=warm["t"])
        # untimed warm-up in this form: an upload drops the mixed form's held
        # factors and the update kernel's next-step list, as a fresh run has none
        s.step(args.warmup)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(dev) as ck:
            ev0.record(stream)
            info = s.step(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier(world)
        ms = ev0.elapsed_time(ev1)
        phase = s.last_timing()
        results[form] = dict(ms=max_over_ranks(ms, world), info=info, phase=phase, clocks=ck.summary(),
                             launches=s.last_launch_count(), state=s.download_state())
    # accuracy of the chosen form vs the FP64 form after the same K steps
    err = None
    if chosen != "fp64":
        uf, ub = results["fp64"]["state"][0], results[chosen]["state"][0]
        area = s.geometry()["area"][:, None, None]
        err = float(((np.abs(ub - uf) * area).sum(axis=(0, 2)) / (np.abs(uf) * area).sum(axis=(0, 2))).max())
    # end to end through the C ABI with pinned host buffers, chosen form
    s.set_precision(MIXED if chosen == "mixed" else FP64)
    for k, v in tuned.get(chosen, {}).items():
        s.set_option(k, v)
    s.upload_state(u0, l0, v0, t=warm["t"])
    hu = torch.empty(u0.shape, dtype=torch.float64, pin_memory=True).numpy()
    hl = torch.empty(l0.shape, dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty(v0.shape, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    hu[...] = u0; hl[...] = l0; hv[...] = v0
    e2e_steps = max(1, min(args.steps, 10))
    # one untimed call first: its streams, events and buffers are made on first use
    tcur = s.step_host(hu, hl, hv, t=warm["t"], out=(hu, hl, hv))[3]["t"]
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e2e_steps):
        # one C-ABI call per step: host state in, host state out (uqc_step_host)
        inf = s.step_host(hu, hl, hv, t=tcur, out=(hu, hl, hv))[3]
        tcur = inf["t"]
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(ev0.elapsed_time(ev1), 1e3 * (time.perf_counter() - t0)), world)
    cells = s.n_cells
    r = results[chosen]
    value = cells * args.steps * world / (r["ms"] / 1e3)
    fp64_value = cells * args.steps * world / (results["fp64"]["ms"] / 1e3)
    # roofline of the closure phase (the dominant kernels): algorithmic work
    # of the timed steps, split by the unit it runs on, over the phase time
    inf = r["info"]
    ref_inf = results["fp64"]["info"]
    closure_ms = r["phase"][0] / args.steps
    measured = measure_peaks(dev)
    s.set_precision(MIXED if chosen == "mixed" else FP64)
    mixed_form = s.form()["mixed_form"]
    roof = closure_roofline(chosen, s.n_states, s.n_total, s.n_quad, cells, args.steps, ref_inf, closure_ms, measured,
                            inf["active_cells"], mixed_form)
    roof["mixed_form"] = mixed_form
    roof["update_ms_per_launch"] = r["phase"][1] / args.steps
    roof["fp64_form"] = closure_roofline("fp64", s.n_states, s.n_total, s.n_quad, cells, args.steps, ref_inf,
                                         results["fp64"]["phase"][0] / args.steps, measured, ref_inf["active_cells"])
    state_bytes = cells * s.n_states * s.n_total * 8
    h2d = 2 * state_bytes + 4 * cells
    d2h = 2 * state_bytes + 4 * cells
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if chosen == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": "euler2d_sod_2u_deg5_q10x10", "cells": cells, "duals_per_cell": s.n_states * s.n_total,
                   "nodes": s.n_quad, "form": chosen, "parallelism": "single GPU",
                   "l2": f"inputs larger than L2 (resident state {cells * (2 * s.n_states * s.n_total + s.n_states * s.n_quad) * 8 / 1e9:.2f} GB)"},
        "fp64": {"value": fp64_value, "ms_per_step": results["fp64"]["ms"] / args.steps},
        "chosen_over_fp64": value / fp64_value,
        "moment_rel_l1_vs_fp64": err,
        "newton": {"iterations_per_step": inf["newton_iterations"] / args.steps, "active_cells_last_step": inf["active_cells"],
                   "line_search_trials": inf["line_search_trials"]},
        "roofline": roof,
        "e2e": {"value": cells * e2e_steps * world / (e2e_ms / 1e3), "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
        "autotuned": tuned or None,
    }
    if rank == 0 and not args.no_oracle_strip:
        line["moment_rel_l1_vs_oracle_strip"] = oracle_strip_errors(forms)
    if args.serve_requests > 0:
        line["serving"] = run_serving(args, MIXED if chosen == "mixed" else FP64)
    if not args.no_other_configs:
        # the other configurations in the same run (GPU only; `--configs` adds the CPU samples)
        s.close()
        line["other_configs"] = {name: config_gpu(name, mk, st) for name, (mk, _p, _i, _b, _n, st, _s) in _configs().items()
                                 if not name.startswith("C2")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, *_ = cpu_reference_run(0, 2, min_seconds=args.cpu_seconds)
            line["cpu_baseline"] = cb
        except Exception as e:  # the reference build is optional on a box without it
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    s.close()


# The other configurations: (builder, reference problem, reference IC parameters,
# bounded-barrier bounds, Newton mode, GPU steps, CPU sample builder).
def _configs():
    from uqcreator_b200 import workloads as W
    return {
        "C1_burgers1d_500": (W.burgers1d, "Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5), "reference", 0,
                             lambda: W.burgers1d()),
        "C2_euler2d_200k": (W.euler2d, "Euler2D", [0.5, 1.0, 1.0, 0.125, 0.1], (3, 12), "guarded", 10,
                            lambda: W.euler2d(nx=400, ny=10)),
        "C3_sw1d_1M_adaptive": (W.shallow_water1d, "ShallowWater1D", [0.5, 1.0, 0.5], (3, 12), "reference", 10,
                                lambda: W.shallow_water1d(ncells=50_000)),
        "C5_euler2d_3u_262k": (W.euler2d_3u, "Euler2D", [0.5, 1.0, 1.0, 0.125, 0.1], (3, 12), "guarded", 3,
                               lambda: W.euler2d_3u(nx=512, ny=2)),
    }


def config_gpu(name, mk, steps):
    """GPU FP64 and mixed cell-steps/s of one configuration from the same state
    (steps 0: the whole solve, CUDA graphs; else 3 warm-up steps, then `steps`
    timed by CUDA events) and the mixed form's moment error against the FP64
    form after them."""
    import torch
    from uqcreator_b200 import Solver, MIXED
    toml = mk()
    out = {"config": name}
    states = {}
    for form in ("fp64", "mixed"):
        s = Solver(toml)
        s.init_state()
        if form == "mixed":
            s.set_precision(MIXED)
        if steps == 0:    # whole solve
            s.run(1e-3)
            torch.cuda.synchronize(); t0 = time.perf_counter()
            info = s.run(s.settings.GetTEnd())
            torch.cuda.synchronize(); el = time.perf_counter() - t0
            done = info["steps"]
        else:
            s.step(3)
            s.step(steps)
            el = sum(s.last_timing()[2:3]) / 1e3
            done = steps
        out[form] = {"cell_steps_per_s": s.n_cells * done / el, "ms_per_step": 1e3 * el / done, "steps": done}
        states[form] = s.download_state()[0]
        s.close()
    uf, um = states["fp64"], states["mixed"]
    out["mixed_over_fp64"] = out["mixed"]["cell_steps_per_s"] / out["fp64"]["cell_steps_per_s"]
    out["moment_rel_l1_mixed_vs_fp64"] = float(np.abs(um - uf).sum() / np.abs(uf).sum())
    return out


def run_configs(args):
    """One JSON line per configuration: config_gpu's figures and the
    reference's own C++ (OpenMP) on a sample of the configuration."""
    from oracle import refharness
    for name, (mk, problem, ic, bounds, newton, steps, sample) in _configs().items():
        out = config_gpu(name, mk, steps)
        if refharness.available("omp") and not args.no_cpu_baseline:
            st = sample()
            r = refharness.RefSolver(st, problem, ic, bounds=bounds, mesh2d=__import__("uqcreator_b200").workloads.mesh_for(st),
                                     variant="omp", newton=newton)
            r.init_state()
            r.step(1)
            t0 = time.perf_counter(); n = 0
            while time.perf_counter() - t0 < args.cpu_seconds / 3 or n == 0:
                r.step(1); n += 1
            el = time.perf_counter() - t0
            out["cpu_reference"] = {"cell_steps_per_s": r.n_cells * n / el, "cells": r.n_cells, "steps": n,
                                    "cores": os.cpu_count()}
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-strip", action="store_true", help="skip the error against the oracle on the 8,000-cell strip")
    ap.add_argument("--no-autotune", action="store_true", help="time both forms in their default launch shapes")
    ap.add_argument("--no-other-configs", action="store_true", help="skip the GPU lines of C1, C3 and C5 in the bench line")
    ap.add_argument("--sharded", action="store_true",
                    help="N = 1: run the sharded path (one shard, a one-rank NCCL group) that N > 1 runs")
    ap.add_argument("--serve-requests", type=int, default=120, help="requests of the serving stream (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=12.0, help="arrivals per second")
    ap.add_argument("--serve-budget-gb", type=float, default=100.0)
    ap.add_argument("--serve-policy", type=int, default=0, help="0 round robin, 1 shortest remaining time first")
    ap.add_argument("--serve-max-stepping", type=int, default=0, help="requests stepping at a time (policy 1; 0: no limit)")
    ap.add_argument("--serve-aging", type=float, default=1.0, help="policy 1: ms of remaining time one ms of waiting offsets")
    ap.add_argument("--serving-only", action="store_true",
                    help="only the serving section (e.g. the whole stream: --serve-requests 2000)")
    ap.add_argument("--configs", action="store_true", help="one line per configuration (C1, C2, C3, C5) instead of the bench line")
    args = ap.parse_args()
    rank, world, local = dist_init()
    one_rank_group = False
    if args.sharded and world == 1 and args.impl == "b200":
        import socket
        import torch.distributed as dist
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("cpu:gloo,cuda:nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
        one_rank_group = True
    if args.serving_only:
        if rank == 0:
            import torch
            from uqcreator_b200 import MIXED
            torch.cuda.set_device(local)
            print(json.dumps({"serving": run_serving(args, MIXED)}))
    elif args.configs:
        if rank == 0:
            run_configs(args)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local)
    if world > 1 or one_rank_group:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
