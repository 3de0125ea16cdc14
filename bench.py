#!/usr/bin/env python
"""Resolvent solves/sec at 1e-10 relative true residual on B200: FP32-multigrid-preconditioned
FP64 flexible GMRES (the served path) beside the plain FP64 GMRES + FP64 multigrid path.

Workload (default): two-particle annihilation A + B -> 0 on a 2-D 32 x 32 grid, h = 1/32,
D_A = D_B = 1, reaction 10 / voxel volume on a shared voxel, population_box(1024, {1, 1})
(N = 1,050,625 states), shift s = 1, Dirichlet(1) right-hand sides from a seeded counter
generator, GMRES(30) with sector_multigrid, tolerance 1e-10 * ||b||.

One step = one resolvent solve of a fresh right-hand side. `value` is whole-job solves/sec
with the right-hand sides already resident in HBM (device-timed with CUDA events, L2 flushed
between steps, max over ranks); `e2e` is the same through the C ABI with host buffers, the
host->device copy of b and device->host copy of x inside the timed region.

Beside it: `fp64_path` (the plain FP64 drop-in path, one request at a time), `served` (64
requests of the same workload through the request loop, FP32 path batched four wide against
the FP64 path; `fp32_over_plain_fp64_path` is the serving speed-up), `served_mix` (one GPU only:
the seeded serving workload of markovkit_b200.inputs.serving_requests, Poisson arrivals over
mixed models of up to 186,043,585 states), `roofline` (the generator SpMV on the 3-D 16^3 box of
cap 2) and `cpu_baseline`.

Multi-GPU: independent replicas (one resident solver per rank, each solving its own
right-hand sides; no collective on the data path), weak scaling.

--impl reference times the reference's own CPU implementation (MarkovKit's headers compiled
against the numerics shim, oracle/_ref/ref_driver) on this host's cores, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "annihilation_2d32": dict(
        workload="rdme_annihilation_2d_32x32_box_1_1",
        dim=2, cells=32, caps=[1, 1], model="annihilation", k=10.0, D=[1.0, 1.0], shift=1.0,
        rhs="dirichlet", seed=1,
    ),
    "birth_death_1d16": dict(
        workload="rdme_birth_death_1d_16_box_3",
        dim=1, cells=16, caps=[3], model="birth_death", birth=0.05, death=0.02, D=[1.0], shift=0.5,
        rhs="uniform", seed=0,
    ),
    "birth_death_3d16": dict(
        workload="rdme_birth_death_3d_16x16x16_box_2",
        dim=3, cells=16, caps=[2], model="birth_death", birth=0.05, death=0.02, D=[1.0], shift=0.5,
        rhs="uniform", seed=2,
    ),
}
DEFAULT_WORKLOAD = "annihilation_2d32"
REL_TOL = 1e-10
RESTART = 30
FP32_COARSEST = 256
L2_FLUSH_BYTES = 256 << 20


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def reactions_of(w: dict):
    if w["model"] == "birth_death":
        b, d = w["birth"], w["death"]
        return [([1], lambda n, vol: b * vol), ([-1], lambda n, vol: d * n[0])]
    if w["model"] == "annihilation":
        k = w["k"]
        return [([-1, -1], lambda n, vol: k * n[0] * n[1] / vol)]
    return []


def rhs_of(w: dict, seed: int, n: int) -> np.ndarray:
    from markovkit_b200.inputs import dirichlet_rhs, uniform_rhs

    return dirichlet_rhs(seed, n) if w["rhs"] == "dirichlet" else uniform_rhs(seed, n)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = "uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            if self.uuid and self.uuid not in parts[0]:
                continue
            rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, val in zip(names, r[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {
            "sm_mhz": sm[len(sm) // 2] if sm else None,
            "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
            "reasons": sorted(reasons),
            "samples": len(rows),
        }


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*); a short
    process-group timeout so that ranks waiting on a lost peer end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_teardown(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()


def replica_seeds(base: int, rank: int, count: int) -> list[int]:
    """The right-hand-side seeds of one replica: each rank solves its own, disjoint stream."""
    return [base + 1_000_003 * rank + s for s in range(count)]


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int, device) -> float:
    """The slowest rank's time: whole-job throughput is all ranks' work over this."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args) -> dict | None:
    import torch

    import markovkit_b200 as mk

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    dims = [w["cells"]] * w["dim"]
    h = 1.0 / w["cells"]
    dom = mk.voxel_domain(mk.grid(dims, [h] * w["dim"]), w["D"])
    model = mk.reaction_diffusion(dom, [mk.local_reaction(c, f) for c, f in reactions_of(w)])
    V = int(np.prod(dims))
    box = mk.population_box(V, w["caps"])
    Q = mk.generator(box, model, "absorbing")
    A = mk.shifted_generator(Q, w["shift"])
    N = box.size()

    # right-hand sides resident in HBM (each rank its own stream of seeds)
    K, W = args.steps, args.warmup
    seeds = replica_seeds(w["seed"], rank, W + K)
    host_b = [rhs_of(w, s, N) for s in seeds]
    dev_b = [torch.from_numpy(b).to(dev) for b in host_b]
    bnorm = [float(np.linalg.norm(b)) for b in host_b]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def make_solver(precision: str):
        # the FP32 path uses a dense solve for sectors of at most 256 states; the FP64 path
        # keeps the reference's multigrid_options (coarsest 4)
        mo = (mk.multigrid_options(precision="fp32", coarsest_size=FP32_COARSEST) if precision == "fp32"
              else mk.multigrid_options(precision="fp64"))
        M = mk.sector_multigrid(dom, box, w["shift"], mo)
        opts = mk.gmres_options(tolerance=REL_TOL * bnorm[0], max_iterations=2000, restart=RESTART,
                                flexible=(precision == "fp32"))
        return M, mk.solver(A, M, opts)

    def solve_all(solver, steps, host_side=False):
        lat, its, res = [], [], []
        xs = []
        stream = torch.cuda.current_stream()
        for s in steps:
            opts_tol = REL_TOL * bnorm[s]
            _set_tolerance(solver, opts_tol)
            flush.zero_()
            x = torch.zeros(N, dtype=torch.float64, device=dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if host_side:
                hb = pinned_b[s]
                hx = pinned_x
                hx.zero_()
                e0.record(stream)
                r = solver.solve_host(hb.numpy(), hx.numpy())
                e1.record(stream)
                x = hx.to(dev)
            else:
                e0.record(stream)
                r = solver.solve(dev_b[s], x)
                e1.record(stream)
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
            its.append(r.iterations)
            res.append(r.converged)
            xs.append(x)
        return lat, its, res, xs

    def true_rel(x, s):
        r = torch.empty_like(x)
        A.apply(x, r)
        return float(torch.linalg.norm(dev_b[s] - r)) / bnorm[s]

    pinned_b = [torch.from_numpy(b).pin_memory() for b in host_b]
    pinned_x = torch.zeros(N, dtype=torch.float64).pin_memory()

    results = {}
    for precision in ("fp32", "fp64"):
        M, solver = make_solver(precision)
        solve_all(solver, range(W))
        barrier(world)
        torch.cuda.synchronize()
        sampler = ClockSampler(_uuid(dev)) if precision == "fp32" else None
        if sampler:
            sampler.__enter__()
        launches0 = mk.api.kernel_launches()
        lat, its, conv, xs = solve_all(solver, range(W, W + K))
        torch.cuda.synchronize()
        launches = mk.api.kernel_launches() - launches0
        if sampler:
            sampler.__exit__(None, None, None)
        worst = max(true_rel(x, W + i) for i, x in enumerate(xs))
        total_ms = max_over_ranks(sum(lat), world, dev)
        results[precision] = dict(
            lat=lat, its=its, converged=all(conv), worst_true_rel=worst, total_ms=total_ms,
            clocks=sampler.summary() if sampler else None, M=M, solver=solver, xs=xs,
            launches=launches,
        )
        if precision == "fp32":
            # e2e through the C ABI with host buffers
            lat_h, its_h, conv_h, xs_h = solve_all(solver, range(W, W + K), host_side=True)
            total_h = max_over_ranks(sum(lat_h), world, dev)
            results["e2e"] = dict(lat=lat_h, total_ms=total_h, converged=all(conv_h),
                                  worst_true_rel=max(true_rel(x, W + i) for i, x in enumerate(xs_h)))
            # the same solution as the FP64 oracle path is checked below

    # error of each FP32-MG solution against the FP64 path's solution of the same right-hand side
    r32 = results["fp32"]
    r64 = results["fp64"]
    err_vs_fp64 = max(
        float(torch.linalg.norm(a - b64) / torch.linalg.norm(b64)) for a, b64 in zip(r32["xs"], r64["xs"])
    )

    roof = roofline(mk, Q, M=results["fp32"]["M"], dev=dev, N=N)
    launches = r32["launches"]
    served = serve_measure(mk, box, model, w, host_b, W, K)
    # the mixed serving workload runs on one GPU only (it is a per-device measurement)
    served_mix = serve_mix_measure() if world == 1 and not args.no_serve_mix else None

    dist_teardown(world)
    if rank != 0:
        return None
    solves = world * K
    value = solves / (r32["total_ms"] / 1e3)
    e2e_value = solves / (results["e2e"]["total_ms"] / 1e3)
    lat_sorted = sorted(r32["lat"])

    def pct(p):
        return lat_sorted[min(len(lat_sorted) - 1, int(round(p / 100 * (len(lat_sorted) - 1))))]

    line = {
        "metric": "resolvent solves/sec at 1e-10 relative true residual (FP32-MG / FP64-FGMRES)",
        "value": round(value, 3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(r32["total_ms"] / K, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (Krylov) + f32 (multigrid)",
        "data": "synthetic: seeded Dirichlet(1) right-hand sides; model built from its definition",
        "config": {
            "workload": w["workload"], "states": N, "voxels": V, "shift": w["shift"],
            "gmres_restart": RESTART, "tolerance": "1e-10 relative true residual",
            "parallelism": f"replicas x{world}", "l2": "flushed between steps (256 MiB write)",
        },
        "latency_ms": {"p50": round(pct(50), 4), "p99": round(pct(99), 4)},
        "iterations": {"median": int(np.median(r32["its"])), "max": int(max(r32["its"]))},
        "worst_true_rel_residual": r32["worst_true_rel"],
        "rel_error_vs_fp64_path": err_vs_fp64,
        "fp64_path": {
            "value": round(world * K / (r64["total_ms"] / 1e3), 3),
            "unit": "solves/s",
            "ms_per_step": round(r64["total_ms"] / K, 4),
            "iterations_median": int(np.median(r64["its"])),
            "worst_true_rel_residual": r64["worst_true_rel"],
        },
        "e2e": {
            "value": round(e2e_value, 3),
            "unit": "solves/s",
            "h2d_bytes_per_step": N * 8 * 2,
            "d2h_bytes_per_step": N * 8,
        },
        "served": served,
        "served_mix": served_mix,
        "roofline": roof,
        "gpu_launches": launches,
        "clocks": r32["clocks"],
    }
    # the served path against the plain FP64 drop-in path (one stream, one request at a time)
    served["fp32_over_plain_fp64_path"] = round(served["fp32"]["value"] / line["fp64_path"]["value"], 3)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w)
    print(json.dumps(line), flush=True)
    return line


SERVE_SLOTS = 4
SERVE_REQUESTS = 64
SERVE_RESTART = 15  # a batched step's Gram-Schmidt cost grows with the basis; 15 served best


def serve_measure(mk, box, model, w, host_b, W, K) -> dict:
    """SERVE_REQUESTS right-hand sides of the bench workload (the K timed ones, then more seeds)
    through the request loop (markovkit_b200.serve): all submitted at once to SERVE_SLOTS workers
    that overlap their solves on the device, host buffers in and out, after warm-up requests
    that make the resident solvers. Host wall clock from the first submit to the last
    completion. The count keeps every slot busy for several rounds, so the number is the
    loop's steady throughput rather than one round and its tail."""
    from markovkit_b200.serve import server

    n = box.size()
    extra = [rhs_of(w, w["seed"] + 7_000_001 + k, n) for k in range(max(0, SERVE_REQUESTS - K))]
    reqs = (host_b[W:W + K] + extra)[:SERVE_REQUESTS]
    out = {}
    # served path: FP32 multigrid, same-key requests batched four wide; the FP64 line is the
    # plain path through the same loop (no batching, the reference's multigrid options)
    variants = {"fp32": dict(precision="fp32", batch=4, coarsest_size=FP32_COARSEST, restart=SERVE_RESTART),
                "fp64": dict(precision="fp64", batch=1, coarsest_size=4, restart=RESTART)}
    for precision, kw in variants.items():
        with server(slots=SERVE_SLOTS, rel_tolerance=REL_TOL, **kw) as srv:
            pid = srv.register(box, model)
            warm = [srv.submit(pid, w["shift"], host_b[k % W]) for k in range(SERVE_SLOTS * kw["batch"])]
            for t in warm:
                srv.wait(t)
            t0 = time.perf_counter()
            tickets = [srv.submit(pid, w["shift"], b) for b in reqs]
            res = [srv.wait(t)[1] for t in tickets]
            wall = time.perf_counter() - t0
            lat = sorted(r.latency_ms for r in res)
            out[precision] = {
                "value": round(len(reqs) / wall, 3),
                "unit": "solves/s",
                "p50_ms": round(lat[len(lat) // 2], 3),
                "p99_ms": round(lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))], 3),
                "worst_rel_residual": max(r.residual for r in res),
                "all_converged": all(r.status == 0 for r in res),
            }
    out["slots"] = SERVE_SLOTS
    out["fp32_over_fp64"] = round(out["fp32"]["value"] / out["fp64"]["value"], 3)
    out["requests"] = len(reqs)
    out["note"] = ("requests submitted at once; host b and x; resident solver per slot; fp32: "
                   "batch 4, FGMRES(15), dense solve of sectors <= 256 states; fp64: batch 1, "
                   "GMRES(30), the reference's multigrid options")
    return out


MIX_COUNT = 24
MIX_RATE = 20.0    # requests per second
MIX_RESTART = 30   # the 1-D boxes of 10^7-10^8 states need ~75 FGMRES(15) steps, ~45 at 30


def serve_mix_measure() -> dict:
    """The serving workload: MIX_COUNT seeded requests (markovkit_b200.inputs.serving_requests)
    with Poisson arrivals at MIX_RATE per second, models uniform over configurations 0-2 and 1-D
    birth-death boxes of 64-256 voxels and cap 2-4 (969 to 186,043,585 states), shifts
    log-uniform in [0.1, 10], Dirichlet(1) right-hand sides. Each request is submitted at its
    arrival time (host b and x); latency runs from submit to x on the host; solves/s is the count
    over the wall time from the first arrival to the last completion. Shifts differ, so requests
    never share a resident solver and no batching happens; the served FP32 path gains only by
    overlapping SERVE_SLOTS solves and by its cheaper V-cycle."""
    from markovkit_b200.inputs import serving_requests
    from markovkit_b200.serve import server, serving_problem

    reqs = serving_requests(count=MIX_COUNT, rate=MIX_RATE)
    keys = sorted({(r["model"], r["voxels"], r["cap"]) for r in reqs})
    problems = {k: serving_problem(*k) for k in keys}
    sizes = {k: problems[k][0].size() for k in keys}
    bs = [rhs_of({"rhs": "dirichlet"}, r["rhs_seed"], sizes[(r["model"], r["voxels"], r["cap"])]) for r in reqs]
    out = {}
    variants = {"fp32": dict(precision="fp32", slots=SERVE_SLOTS, batch=4, coarsest_size=FP32_COARSEST,
                             restart=MIX_RESTART),
                "fp64": dict(precision="fp64", slots=1, batch=1, coarsest_size=4, restart=RESTART)}
    for precision, kw in variants.items():
        with server(rel_tolerance=REL_TOL, **kw) as srv:
            pids = {k: srv.register(*problems[k]) for k in keys}
            t0 = time.perf_counter()
            tickets = []
            for r, b in zip(reqs, bs):
                wait = r["arrival_s"] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
                tickets.append(srv.submit(pids[(r["model"], r["voxels"], r["cap"])], r["shift"], b))
            res = [srv.wait(t)[1] for t in tickets]
            wall = time.perf_counter() - t0 - reqs[0]["arrival_s"]
            st = srv.stats()
        lat = sorted(r.latency_ms for r in res)
        out[precision] = {
            "value": round(len(res) / wall, 3),
            "unit": "solves/s",
            "p50_ms": round(lat[len(lat) // 2], 3),
            "p99_ms": round(lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))], 3),
            "worst_rel_residual": max(r.residual for r in res),
            "all_converged": all(r.status == 0 for r in res),
            "evictions": st["evictions"],
            "memory_waits": st["memory_waits"],
        }
    out["fp32_over_fp64"] = round(out["fp32"]["value"] / out["fp64"]["value"], 3)
    out["requests"] = len(reqs)
    out["largest_states"] = max(sizes.values())
    out["note"] = (f"Poisson arrivals at {MIX_RATE}/s, seed 4; fp32: {SERVE_SLOTS} slots, FGMRES({MIX_RESTART}), "
                   "dense solve of sectors <= 256 states; fp64: 1 slot, GMRES(30), the reference's "
                   "multigrid options; 1-D boxes use configuration 0's voxel size 1/16")
    return out


def _set_tolerance(solver, tol):
    solver.set_tolerance(tol)


def _uuid(dev) -> str | None:
    import torch

    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def _time_apply(Q, N, dev, flush=None, reps=20) -> float:
    """Average ms of one FP64 apply_shifted, CUDA events on its launch stream, each launch timed
    on its own (L2 flushed before each when `flush` is given)."""
    import torch

    x = torch.rand(N, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    for _ in range(3):
        Q.apply_shifted(1.0, x, y)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Q.apply_shifted(1.0, x, y)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / reps


def ncu_traffic(name: str) -> float | None:
    """dram__bytes_read.sum + dram__bytes_write.sum per launch from a committed ncu summary
    (profiles/<name>.md, the row 'traffic (read + write) | X MB per launch')."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("| traffic (read + write)"):
            return float(line.split("|")[2].split()[0]) * 1e6
    return None


def roofline(mk, Q, M, dev, N) -> dict:
    """The generator SpMV, the kernel the north star's roofline target names, on the 3-D
    16^3-voxel box of cap 2 (8,394,753 states): FP64 apply_shifted, one compulsory read of x and
    write of y, 16 bytes per state (134 MB per launch, larger than L2), L2 flushed before each
    timed launch. The bench workload's own SpMV (16.8 MB, L2-resident) is reported beside it."""
    import torch

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    pk = peaks()
    w = WORKLOADS["birth_death_3d16"]
    dom = mk.voxel_domain(mk.grid([16] * 3, [1 / 16] * 3), w["D"])
    model = mk.reaction_diffusion(dom, [mk.local_reaction(c, f) for c, f in reactions_of(w)])
    box = mk.population_box(4096, w["caps"])
    Q3 = mk.generator(box, model, "absorbing")
    N3 = box.size()
    ms = _time_apply(Q3, N3, dev, flush)
    algo = N3 * 16
    achieved = algo / (ms * 1e-3) / 1e9
    ms_w = _time_apply(Q, N, dev, None)
    achieved_w = N * 16 / (ms_w * 1e-3) / 1e9
    return {
        "kernel": "generator apply_shifted, FP64 gather SpMV (row_kernel<double,1,2>), 3-D 16^3 box cap 2",
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": pk["hbm_gbs"],
        "peak_source": pk["source"],
        "unit": "GB/s",
        "frac": round(achieved / pk["hbm_gbs"], 4),
        "traffic": ncu_traffic("row_kernel_spmv_birth_death_3d16"),
        "traffic_source": "profiles/row_kernel_spmv_birth_death_3d16.md (ncu, bytes per launch)",
        "us_per_launch": round(ms * 1e3, 3),
        "algorithmic_bytes_per_launch": algo,
        "workload_spmv": {"kernel": "row_kernel<double,2,1>", "us_per_launch": round(ms_w * 1e3, 3),
                          "achieved_gbs": round(achieved_w, 1), "note": "16.8 MB per launch, L2-resident"},
    }


def _problem_args(w: dict) -> list[str]:
    keys = {"dim": w["dim"], "cells": w["cells"], "cap": ",".join(str(c) for c in w["caps"]), "model": w["model"],
            "shift": w["shift"], "D": w["D"][0]}
    if len(w["D"]) > 1:
        keys["D2"] = w["D"][1]
    for k in ("birth", "death", "k"):
        if k in w:
            keys[k] = w[k]
    return [f"{k}={v}" for k, v in keys.items()]


def cpu_baseline(w) -> dict:
    """The matrix-free CPU port (oracle/_ref/mf_port, a restatement of the reference's path
    validated against it) on this host's cores: full solves of the same workload, setup excluded."""
    port = ROOT / "oracle" / "_ref" / "mf_port"
    if not port.exists():
        return {"value": None, "unit": "solves/s", "cores": None, "kind": "port", "sample": "oracle/_ref/mf_port not built"}
    threads = os.cpu_count() or 1
    solves = 2
    args = [str(port), *_problem_args(w), f"rhs={w['rhs']}", f"seed={w['seed']}", "tol=1e-10",
            f"restart={RESTART}", f"threads={threads}", f"solves={solves}"]
    proc = subprocess.run(args, capture_output=True, text=True, timeout=1800)
    if proc.returncode != 0:
        return {"value": None, "unit": "solves/s", "cores": threads, "kind": "port", "sample": proc.stderr[-200:]}
    m = json.loads(proc.stdout.strip().splitlines()[-1])
    secs = sum(m["solve_ms"]) / 1e3
    return {
        "value": round(solves / secs, 5), "unit": "solves/s", "cores": m["threads"], "kind": "port",
        "sample": f"{solves} full solves ({m['iterations']} MG-GMRES iterations each, true rel. residual "
                  f"{m['true_rel_residual']:.2e}) after an untimed {m['setup_ms'] / 1e3:.1f} s set-up",
    }


def run_reference(args) -> None:
    """The reference's own CPU path (MarkovKit headers + numerics shim, oracle/_ref/ref_driver),
    single-threaded as the reference is. Its set-up (population_box, generator, sector_multigrid)
    runs untimed once; one full solve gives the iteration count; each step is a bounded sample of
    SAMPLE_ITERS Arnoldi iterations, and solves/sec = SAMPLE_ITERS / (iterations * step time)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    driver = ROOT / "oracle" / "_ref" / "ref_driver"
    if not driver.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver is not built"}))
        return
    sample_iters = 6
    K, W = args.steps, args.warmup
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [str(driver), *_problem_args(w), f"rhs={w['rhs']}", f"seed={w['seed']}", "tol=1e-10",
               f"restart={RESTART}", "do_apply=0", "do_plain=0", "warmup=1", f"solves={W + K}",
               f"sample_iters={sample_iters}", f"out={tmp}"]
        t0 = time.time()
        proc = subprocess.run(cmd, capture_output=True, text=True)
        wall = time.time() - t0
    if proc.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": "ref_driver failed: " + proc.stderr[-200:].replace("\n", " ")}))
        return
    m = json.loads(proc.stdout.strip().splitlines()[-1])
    its = m["full_solve_iterations"]
    steps_ms = m["gmres_mg"]["solve_ms"][W:]
    per_solve_s = (sum(steps_ms) / len(steps_ms)) / 1e3 * its / sample_iters
    value = 1.0 / per_solve_s
    sample = (f"each step: {sample_iters} of the {its} MG-GMRES iterations of a full solve, scaled; "
              f"untimed set-up {(m['box_ms'] + m['generator_ms'] + m['mg_setup_ms']) / 1e3:.0f} s")
    line = {
        "metric": "resolvent solves/sec at 1e-10 relative true residual (FP32-MG / FP64-FGMRES)",
        "impl": "reference", "value": round(value, 5), "unit": "solves/s", "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": round(per_solve_s * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded right-hand side",
        "config": {"workload": w["workload"], "states": m["N"], "parallelism": "1 host thread"},
        "cpu_baseline": {"value": round(value, 5), "unit": "solves/s", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 5), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1),
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve-mix", action="store_true", help="skip the mixed serving workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
