#!/usr/bin/env python
"""Resolvent solves/sec at 1e-10 relative true residual on B200: FP32-multigrid-preconditioned
FP64 flexible GMRES beside the plain FP64 GMRES + FP64 multigrid path.

Workload (default; the largest single-GPU configuration): single-species birth-death on the
3-D 16 x 16 x 16 grid, h = 1/16, D = 1, birth 0.05 * voxel volume, death 0.02 * n,
population_box(4096, {2}) (N = 8,394,753 states), shift s = 0.5, right-hand sides Uniform(0, 1)
normalised to sum 1 from a seeded counter generator, GMRES(30), tolerance 1e-10 * ||b||. The
FP32 path is flexible GMRES(30) around a sector multigrid whose smoothers, transfers and coarse
solves all run in FP32 (smoother FP32_SMOOTHER); the plain FP64 path is GMRES(30) around the
reference's default multigrid (weighted Jacobi 2/2, coarsest 4) in FP64.

One step = one resolvent solve of a fresh right-hand side. `value` is whole-job solves/sec with
the right-hand sides already resident in HBM (device-timed with CUDA events, inputs larger than
L2 and L2 flushed between steps, max over ranks); `e2e` is the same through the C ABI with host
buffers, the host->device copy of b and device->host copy of x inside the timed region.

Beside it: `fp64_path`; `rel_error_vs_oracle` (each path's solution against the FP64 solution of
the matrix-free CPU port of the reference's path, oracle/_ref/mf_port, for the first timed
right-hand side); `fp32_smoothers` (the FP32 path with each smoother); `secondary` (the 2-D 32 x 32
two-particle annihilation box of 1,050,625 states); `served` (requests of the workload through the
request loop, batched four wide); `served_mix` (the seeded serving workload of
markovkit_b200.inputs.serving_requests against the plain FP64 path on the same arrivals);
`fsp_batch` (512 Krylov-FSP propagations in one persistent launch, with its CPU baseline);
`ssa_batch` (2^20 Gillespie paths of a toggle switch in one launch, with the reference's own
gillespie on the host cores beside it); `roofline` (the generator SpMV of the workload) and `cpu_baseline`.

Multi-GPU: independent replicas (one resident solver per rank, each solving its own
right-hand sides; no collective on the data path), weak scaling. `--gpus N` outside torchrun
re-launches itself under torchrun with N ranks.

--impl reference times the reference's CPU path on this host's cores, rank 0 only: for the
default workload the matrix-free port (the reference's own containers need ~275 GB and days of
single-threaded set-up at 8.4M states), for the 2-D workload the reference's own headers compiled
against the numerics shim (oracle/_ref/ref_driver).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
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
DEFAULT_WORKLOAD = "birth_death_3d16"
SECONDARY_WORKLOAD = "annihilation_2d32"
REL_TOL = 1e-10
RESTART = 30
FP32_SMOOTHER = "gauss_seidel"
MIX_SMOOTHER = "auto"  # the serving mix: the server picks the smoother per problem
MIX_COARSEST = 256     # the serving mix: dense solves of small sectors only (its 1-D boxes and
                       # configuration 1 have many sectors near 4096 states on coarse levels)
FP32_COARSEST = 4096
FP32_SWEEPS = (2, 1)  # pre- and post-smoothing sweeps of the FP32 path
L2_FLUSH_BYTES = 256 << 20
METRIC = "resolvent solves/sec at 1e-10 relative true residual (FP32-MG / FP64-FGMRES)"


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


def problem_of(mk, w: dict):
    dims = [w["cells"]] * w["dim"]
    h = 1.0 / w["cells"]
    dom = mk.voxel_domain(mk.grid(dims, [h] * w["dim"]), w["D"])
    model = mk.reaction_diffusion(dom, [mk.local_reaction(c, f) for c, f in reactions_of(w)])
    box = mk.population_box(int(np.prod(dims)), w["caps"])
    return dom, model, box


def pct(values, p):
    v = sorted(values)
    return v[min(len(v) - 1, int(round(p / 100 * (len(v) - 1))))]


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
    dom, model, box = problem_of(mk, w)
    Q = mk.generator(box, model, "absorbing")
    A = mk.shifted_generator(Q, w["shift"])
    N = box.size()

    # right-hand sides resident in HBM (each rank its own stream of seeds)
    K, W = args.steps, args.warmup
    seeds = replica_seeds(w["seed"], rank, W + K)
    host_b = [rhs_of(w, s, N) for s in seeds]
    dev_b = [torch.from_numpy(b).to(dev) for b in host_b]
    bnorm = [float(np.linalg.norm(b)) for b in host_b]
    pinned_b = [torch.from_numpy(b).pin_memory() for b in host_b]
    pinned_x = torch.zeros(N, dtype=torch.float64).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def true_rel(x, s):
        r = torch.empty_like(x)
        A.apply(x, r)
        return float(torch.linalg.norm(dev_b[s] - r)) / bnorm[s]

    results = {}
    for key, (precision, smoother, coarsest) in PATHS.items():
        solver = make_solver(mk, A, dom, box, w["shift"], precision, smoother, coarsest, bnorm[0])
        solve_steps(solver, dev_b, bnorm, flush, range(W), dev)
        barrier(world)
        torch.cuda.synchronize()
        sampler = ClockSampler(_uuid(dev)) if key == "fp32" else None
        if sampler:
            sampler.__enter__()
        launches0 = mk.api.kernel_launches()
        lat, its, conv, xs = solve_steps(solver, dev_b, bnorm, flush, range(W, W + K), dev)
        torch.cuda.synchronize()
        launches = mk.api.kernel_launches() - launches0
        if sampler:
            sampler.__exit__(None, None, None)
        res = dict(lat=lat, its=its, converged=all(conv), total_ms=max_over_ranks(sum(lat), world, dev),
                   worst_true_rel=max(true_rel(x, W + i) for i, x in enumerate(xs)),
                   clocks=sampler.summary() if sampler else None, launches=launches,
                   x_first=xs[0].cpu().numpy())
        if key == "fp32":
            # e2e through the C ABI with host buffers: b in and x out every step
            lat_h = []
            for s in range(W, W + K):
                solver.set_tolerance(REL_TOL * bnorm[s])
                flush.zero_()
                pinned_x.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                stream = torch.cuda.current_stream()
                e0.record(stream)
                solver.solve_host(pinned_b[s].numpy(), pinned_x.numpy())
                e1.record(stream)
                e1.synchronize()
                lat_h.append(e0.elapsed_time(e1))
            res["e2e_ms"] = max_over_ranks(sum(lat_h), world, dev)
            res["e2e_true_rel"] = true_rel(pinned_x.to(dev), W + K - 1)
        results[key] = res
        del solver, xs
        torch.cuda.empty_cache()

    # the FP32 path with each smoother, a few solves each
    smoothers = {}
    for sm in ("jacobi", "gauss_seidel", "ilu0"):
        solver = make_solver(mk, A, dom, box, w["shift"], "fp32", sm, FP32_COARSEST, bnorm[0])
        solve_steps(solver, dev_b, bnorm, flush, range(1), dev)
        n_s = min(K, 5)
        lat, its, conv, xs = solve_steps(solver, dev_b, bnorm, flush, range(W, W + n_s), dev)
        smoothers[sm] = {"value": round(world * n_s / (max_over_ranks(sum(lat), world, dev) / 1e3), 3),
                         "unit": "solves/s", "iterations_median": int(np.median(its)),
                         "worst_true_rel_residual": max(true_rel(x, W + i) for i, x in enumerate(xs)),
                         "all_converged": all(conv)}
        del solver, xs
    roof = roofline(mk, Q, dev, N, w)
    secondary = None if args.no_secondary else secondary_line(mk, args, world, rank, dev)
    served = None if args.no_serve else serve_measure(mk, box, model, w, host_b, W, K)
    served_mix = serve_mix_measure(mk) if world == 1 and not args.no_serve_mix else None
    fsp = fsp_batch_measure(rank == 0 and world == 1 and not args.no_cpu_baseline) if not args.no_fsp else None
    ssa = ssa_measure(rank == 0 and world == 1 and not args.no_cpu_baseline) if not args.no_ssa else None
    dist_teardown(world)
    if rank != 0:
        return None

    r32, r64 = results["fp32"], results["fp64"]
    solves = world * K
    line = {
        "metric": METRIC,
        "value": round(solves / (r32["total_ms"] / 1e3), 3),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(r32["total_ms"] / K, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (Krylov) + f32 (multigrid)",
        "data": "synthetic: seeded right-hand sides; model built from its definition",
        "config": {
            "workload": w["workload"], "states": N, "voxels": box.n_voxels(), "shift": w["shift"],
            "gmres_restart": RESTART, "tolerance": "1e-10 relative true residual",
            "fp32_multigrid": f"smoother {FP32_SMOOTHER} {FP32_SWEEPS[0]}/{FP32_SWEEPS[1]}, dense solve of "
                              f"sectors <= {FP32_COARSEST} states",
            "parallelism": f"replicas x{world}",
            "l2": f"inputs of {N * 8 / 1e6:.0f} MB per vector and L2 flushed between steps (256 MiB write)",
        },
        "latency_ms": {"p50": round(pct(r32["lat"], 50), 4), "p99": round(pct(r32["lat"], 99), 4)},
        "iterations": {"median": int(np.median(r32["its"])), "max": int(max(r32["its"]))},
        "worst_true_rel_residual": r32["worst_true_rel"],
        "all_converged": r32["converged"],
        "rel_error_fp32_vs_fp64_path": float(np.linalg.norm(r32["x_first"] - r64["x_first"]) /
                                             np.linalg.norm(r64["x_first"])),
        "fp64_path": {
            "value": round(solves / (r64["total_ms"] / 1e3), 3),
            "unit": "solves/s",
            "ms_per_step": round(r64["total_ms"] / K, 4),
            "latency_ms": {"p50": round(pct(r64["lat"], 50), 4), "p99": round(pct(r64["lat"], 99), 4)},
            "iterations_median": int(np.median(r64["its"])),
            "worst_true_rel_residual": r64["worst_true_rel"],
            "multigrid": "the reference's multigrid_options (weighted Jacobi 2/2, coarsest 4), FP64 GMRES(30)",
        },
        "fp32_over_fp64_path": round(r64["total_ms"] / r32["total_ms"], 3),
        "e2e": {
            "value": round(solves / (r32["e2e_ms"] / 1e3), 3),
            "unit": "solves/s",
            "h2d_bytes_per_step": N * 8,
            "d2h_bytes_per_step": N * 8,
            "worst_true_rel_residual": r32["e2e_true_rel"],
        },
        "fp32_smoothers": smoothers,
        "secondary": secondary,
        "served": served,
        "served_mix": served_mix,
        "fsp_batch": fsp,
        "ssa_batch": ssa,
        "roofline": roof,
        "gpu_launches": r32["launches"],
        "clocks": r32["clocks"],
    }
    if served:
        served["fp32_over_plain_fp64_path"] = round(served["fp32"]["value"] / line["fp64_path"]["value"], 3)
    if not args.no_cpu_baseline and world == 1:
        cb, x_port = cpu_baseline(w, seeds[W])
        line["cpu_baseline"] = cb
        if x_port is not None:
            nrm = float(np.linalg.norm(x_port))
            line["rel_error_vs_oracle"] = {
                "fp32_path": float(np.linalg.norm(r32["x_first"] - x_port)) / nrm,
                "fp64_path": float(np.linalg.norm(r64["x_first"] - x_port)) / nrm,
                "oracle": "oracle/_ref/mf_port FP64 solution of the first timed right-hand side "
                          "(the reference's path restated matrix-free, GMRES(30) to 1e-10)",
            }
    print(json.dumps(line), flush=True)
    return line


# headline FP32 path and the plain FP64 drop-in path: (precision, smoother, coarsest sector size)
PATHS = {"fp32": ("fp32", FP32_SMOOTHER, FP32_COARSEST), "fp64": ("fp64", "jacobi", 4)}


def make_solver(mk, A, dom, box, shift, precision, smoother, coarsest, bnorm0):
    sweeps = dict(pre_sweeps=FP32_SWEEPS[0], post_sweeps=FP32_SWEEPS[1]) if precision == "fp32" else {}
    mo = mk.multigrid_options(precision=precision, smoother=smoother, coarsest_size=coarsest, **sweeps)
    M = mk.sector_multigrid(dom, box, shift, mo)
    opts = mk.gmres_options(tolerance=REL_TOL * bnorm0, max_iterations=2000, restart=RESTART,
                            flexible=(precision == "fp32"))
    s = mk.solver(A, M, opts)
    return s


def solve_steps(solver, dev_b, bnorm, flush, steps, dev):
    """One device-timed solve per step from x = 0 (CUDA events on the launching stream, L2
    flushed before each); returns latencies (ms), iterations, convergence flags, solutions."""
    import torch

    lat, its, conv, xs = [], [], [], []
    stream = torch.cuda.current_stream()
    for s in steps:
        solver.set_tolerance(REL_TOL * bnorm[s])
        flush.zero_()
        x = torch.zeros_like(dev_b[s])
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = solver.solve(dev_b[s], x)
        e1.record(stream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
        its.append(r.iterations)
        conv.append(r.converged)
        xs.append(x)
    return lat, its, conv, xs


def secondary_line(mk, args, world, rank, dev) -> dict:
    """The 2-D two-particle annihilation box (1,050,625 states): both paths, a few solves."""
    import torch

    w = WORKLOADS[SECONDARY_WORKLOAD]
    dom, model, box = problem_of(mk, w)
    Q = mk.generator(box, model, "absorbing")
    A = mk.shifted_generator(Q, w["shift"])
    N = box.size()
    n_s = 10
    seeds = replica_seeds(w["seed"], rank, 3 + n_s)
    host_b = [rhs_of(w, s, N) for s in seeds]
    dev_b = [torch.from_numpy(b).to(dev) for b in host_b]
    bnorm = [float(np.linalg.norm(b)) for b in host_b]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    out = {"workload": w["workload"], "states": N, "shift": w["shift"]}
    for key, (precision, smoother, coarsest) in PATHS.items():
        solver = make_solver(mk, A, dom, box, w["shift"], precision, smoother, coarsest, bnorm[0])
        solve_steps(solver, dev_b, bnorm, flush, range(3), dev)
        lat, its, conv, xs = solve_steps(solver, dev_b, bnorm, flush, range(3, 3 + n_s), dev)
        out[key] = {"value": round(world * n_s / (max_over_ranks(sum(lat), world, dev) / 1e3), 3),
                    "unit": "solves/s", "p50_ms": round(pct(lat, 50), 4),
                    "iterations_median": int(np.median(its)), "all_converged": all(conv)}
    out["fp32_over_fp64_path"] = round(out["fp32"]["value"] / out["fp64"]["value"], 3)
    return out


SERVE_SLOTS = 4
SERVE_REQUESTS = 32


def serve_measure(mk, box, model, w, host_b, W, K) -> dict:
    """SERVE_REQUESTS right-hand sides of the bench workload (the K timed ones, then more seeds)
    through the request loop (markovkit_b200.serve): all submitted at once to SERVE_SLOTS workers
    that overlap their solves on the device, host buffers in and out, after warm-up requests
    that make the resident solvers. Host wall clock from the first submit to the last
    completion."""
    from markovkit_b200.serve import server

    n = box.size()
    extra = [rhs_of(w, w["seed"] + 7_000_001 + k, n) for k in range(max(0, SERVE_REQUESTS - K))]
    reqs = (host_b[W:W + K] + extra)[:SERVE_REQUESTS]
    out = {}
    # served path: FP32 multigrid, same-problem requests batched four wide; the FP64 line is the
    # plain path through the same loop (no batching, the reference's multigrid options)
    variants = {"fp32": dict(precision="fp32", batch=4, coarsest_size=FP32_COARSEST, restart=RESTART,
                             smoother=FP32_SMOOTHER),
                "fp64": dict(precision="fp64", batch=1, coarsest_size=4, restart=RESTART, smoother="jacobi")}
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
            lat = [r.latency_ms for r in res]
            out[precision] = {
                "value": round(len(reqs) / wall, 3),
                "unit": "solves/s",
                "p50_ms": round(pct(lat, 50), 3),
                "p99_ms": round(pct(lat, 99), 3),
                "worst_rel_residual": max(r.residual for r in res),
                "all_converged": all(r.status == 0 for r in res),
            }
    out["slots"] = SERVE_SLOTS
    out["fp32_over_fp64"] = round(out["fp32"]["value"] / out["fp64"]["value"], 3)
    out["requests"] = len(reqs)
    out["note"] = (f"requests submitted at once; host b and x; resident solver per slot; fp32: batch 4, "
                   f"FGMRES({RESTART}), smoother {FP32_SMOOTHER}, dense solve of sectors <= {FP32_COARSEST} "
                   f"states; fp64: batch 1, GMRES({RESTART}), the reference's multigrid options")
    return out


MIX_COUNT = 24
MIX_RATE = 20.0  # requests per second


def serve_mix_measure(mk) -> dict:
    """The serving workload: MIX_COUNT seeded requests (markovkit_b200.inputs.serving_requests)
    with Poisson arrivals at MIX_RATE per second, models uniform over configurations 0-2 and 1-D
    birth-death boxes of 64-256 voxels and cap 2-4 (969 to 186,043,585 states), shifts
    log-uniform in [0.1, 10], Dirichlet(1) right-hand sides. Each request is submitted at its
    arrival time (host b and x); latency runs from submit to x on the host; solves/s is the count
    over the wall time from the first arrival to the last completion. The served FP32 path runs
    SERVE_SLOTS slots with requests of one problem batched together whatever their shifts; the
    plain FP64 path solves the requests one at a time in arrival order through the drop-in
    solver (GMRES(30) + the reference's FP64 multigrid, set-up included in each latency)."""
    import torch

    from markovkit_b200.inputs import serving_requests
    from markovkit_b200.serve import server, serving_problem

    reqs = serving_requests(count=MIX_COUNT, rate=MIX_RATE)
    keys = sorted({(r["model"], r["voxels"], r["cap"]) for r in reqs})
    problems = {k: serving_problem(*k) for k in keys}
    sizes = {k: problems[k][0].size() for k in keys}
    bs = [rhs_of({"rhs": "dirichlet"}, r["rhs_seed"], sizes[(r["model"], r["voxels"], r["cap"])]) for r in reqs]
    out = {}
    kw = dict(precision="fp32", slots=SERVE_SLOTS, batch=4, coarsest_size=MIX_COARSEST, restart=RESTART,
              smoother=MIX_SMOOTHER)
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
    lat = [r.latency_ms for r in res]
    out["fp32"] = {
        "value": round(len(res) / wall, 3),
        "unit": "solves/s",
        "p50_ms": round(pct(lat, 50), 3),
        "p99_ms": round(pct(lat, 99), 3),
        "worst_rel_residual": max(r.residual for r in res),
        "all_converged": all(r.status == 0 for r in res),
        "batched_requests": int(sum(1 for r in res if r.batched > 1)),
        "evictions": st["evictions"],
        "memory_waits": st["memory_waits"],
    }
    # the plain FP64 drop-in path on the same arrivals, one request at a time
    dev = torch.device("cuda", torch.cuda.current_device())
    clock = reqs[0]["arrival_s"]
    lat64, rel64, conv64 = [], [], []
    for r, b in zip(reqs, bs):
        box, model = problems[(r["model"], r["voxels"], r["cap"])]
        start = max(clock, r["arrival_s"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Q = mk.generator(box, model, "absorbing")
        A = mk.shifted_generator(Q, r["shift"])
        M = mk.sector_multigrid(model.domain, box, r["shift"], mk.multigrid_options(precision="fp64"))
        bn = float(np.linalg.norm(b))
        s = mk.solver(A, M, mk.gmres_options(tolerance=REL_TOL * bn, max_iterations=2000, restart=RESTART))
        x = np.zeros_like(b)
        res64 = s.solve_host(b, x)
        torch.cuda.synchronize()
        took = time.perf_counter() - t0
        clock = start + took
        lat64.append((clock - r["arrival_s"]) * 1e3)
        rel64.append(res64.residual / bn if bn > 0 else 0.0)
        conv64.append(res64.converged)
        del s, M, A, Q
        torch.cuda.empty_cache()
    out["plain_fp64_path"] = {
        "value": round(len(reqs) / (clock - reqs[0]["arrival_s"]), 3),
        "unit": "solves/s",
        "p50_ms": round(pct(lat64, 50), 3),
        "p99_ms": round(pct(lat64, 99), 3),
        "worst_rel_residual": max(rel64),
        "all_converged": all(conv64),
    }
    out["fp32_over_plain_fp64_path"] = round(out["fp32"]["value"] / out["plain_fp64_path"]["value"], 3)
    out["requests"] = len(reqs)
    out["largest_states"] = max(sizes.values())
    out["note"] = (f"Poisson arrivals at {MIX_RATE}/s, seed 4; fp32: {SERVE_SLOTS} slots, batch 4 (same problem and shift), "
                   f"FGMRES({RESTART}), smoother {MIX_SMOOTHER} (Gauss-Seidel for one species of at most two "
                   f"molecules per state, Jacobi otherwise), dense solve of sectors <= {MIX_COARSEST} "
                   "states; plain fp64: one request at a time, GMRES(30), the reference's multigrid options, "
                   "generator and multigrid set-up inside each latency; 1-D boxes use configuration 0's "
                   "voxel size 1/16")
    return out


FSP_MAX_STEPS = 2000
FSP_CPU_SAMPLE = 16  # instances of each family the CPU baseline runs


def fsp_batch_measure(with_cpu: bool) -> dict:
    """The batching workload: the 512 seeded Krylov-FSP propagations to t = 2 of
    markovkit_b200.inputs.fsp_batch_instances (256 birth-death boxes of 100-2000 states, 256
    toggle switches of 2,601-90,601 states), tolerance 1e-8, at most FSP_MAX_STEPS attempts each,
    in one persistent launch with autotuned shapes (the autotune runs untimed first). Timed with
    CUDA events around the launch. The CPU baseline runs the reference's solve_krylov_fsp
    (oracle/_ref/ref_fsp) on the first FSP_CPU_SAMPLE instances of each family, one process per
    host core, and scales the family-weighted mean time per instance to the batch."""
    import torch

    from markovkit_b200.fsp import _Problem, box as fbox, fsp_batch, krylov_fsp_options
    from markovkit_b200.fsp_models import network_of
    from markovkit_b200.inputs import fsp_batch_instances

    inst = fsp_batch_instances()
    probs = [_Problem(network_of(x), x["initial"], x["final_time"],
                      krylov_fsp_options(inside=fbox(x["bounds"]), tolerance=x["tolerance"], max_steps=FSP_MAX_STEPS))
             for x in inst]
    b = fsp_batch(probs)
    threads, blocks = b.autotune(sample=0)
    b.run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    _, res = b.results()
    finished = sum(1 for r in res if r.status == 0)
    out = {
        "metric": "Krylov-FSP propagations/sec to t = 2 (FSP tolerance 1e-8), one persistent launch",
        "value": round(len(probs) / (ms / 1e3), 2),
        "unit": "instances/s",
        "ms": round(ms, 3),
        "instances": len(probs),
        "finished": finished,
        "capped": len(probs) - finished,
        "max_steps": FSP_MAX_STEPS,
        "shape": {"threads": threads, "blocks": blocks},
    }
    if with_cpu:
        out["cpu_baseline"] = fsp_cpu_baseline(inst)
    return out


def fsp_cpu_baseline(inst) -> dict:
    from concurrent.futures import ThreadPoolExecutor

    from markovkit_b200.inputs import fsp_instance_line

    driver = ROOT / "oracle" / "_ref" / "ref_fsp"
    if not driver.exists():
        return {"value": None, "unit": "instances/s", "cores": None, "kind": "reference",
                "sample": "oracle/_ref/ref_fsp not built"}
    half = len(inst) // 2
    sample = list(range(FSP_CPU_SAMPLE)) + list(range(half, half + FSP_CPU_SAMPLE))
    cores = os.cpu_count() or 1

    def one(k):
        line = fsp_instance_line(inst[k], max_steps=FSP_MAX_STEPS) + "\n"
        t0 = time.perf_counter()
        p = subprocess.run([str(driver)], input=line, capture_output=True, text=True, timeout=600)
        return k, time.perf_counter() - t0, p.returncode

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        done = list(ex.map(one, sample))
    wall = time.perf_counter() - t0
    per = {"birth_death": [], "toggle": []}
    for k, sec, rc in done:
        if rc == 0:
            per[inst[k]["family"]].append(sec)
    # the batch's instances are half of each family: expected single-core seconds per instance
    mean = 0.5 * float(np.mean(per["birth_death"])) + 0.5 * float(np.mean(per["toggle"]))
    value = cores / mean
    return {"value": round(value, 3), "unit": "instances/s", "cores": cores, "kind": "reference",
            "sample": f"{len(sample)} instances (the first {FSP_CPU_SAMPLE} of each family), one ref_fsp "
                      f"process per core, {wall:.1f} s wall; instances/s = cores / family-weighted mean "
                      f"seconds per instance ({mean:.3f} s)"}


SSA_PATHS = 1 << 20
SSA_TOGGLE = (30.0, 25.0, 2.0, 2.5)  # a1, a2, n1, n2: a toggle switch of the FSP batch's family
SSA_CPU_PATHS = 20000                 # paths per host core in the CPU baseline
SSA_REPEATS = 5                       # timed calls of the public SSA path (median)


def ssa_measure(with_cpu: bool) -> dict:
    """The batched SSA: SSA_PATHS Gillespie paths of a toggle switch from (0, 0) to t = 2 in one
    launch, through the public call (markovkit_b200.ssa.simulate: propensity table built and
    uploaded, the launch, final states, jumps and statuses copied back), timed by wall clock
    after an untimed run of the same seed that sizes the propensity box; the median of
    SSA_REPEATS calls (each replays the same paths). The CPU baseline runs the reference's own
    gillespie (oracle/_ref/ref_ssa), one process per host core."""
    from markovkit_b200.fsp_models import toggle
    from markovkit_b200.ssa import simulate

    model = toggle(*SSA_TOGGLE)
    sized = simulate(model, [0, 0], 2.0, SSA_PATHS, seed=3)
    times = []
    for _ in range(SSA_REPEATS):
        t0 = time.perf_counter()
        ens = simulate(model, [0, 0], 2.0, SSA_PATHS, seed=3, bounds=sized.bounds)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    jumps = int(ens.steps.sum())
    out = {
        "metric": "Gillespie paths/sec to t = 2 (toggle switch a1 30, a2 25, n1 2, n2 2.5), one launch",
        "value": round(SSA_PATHS / sec, 1),
        "unit": "paths/s",
        "ms": round(1e3 * sec, 3),
        "paths": SSA_PATHS,
        "jumps_per_s": round(jumps / sec, 1),
        "mean_final": [round(float(v), 4) for v in ens.final_means()],
        "box": ens.bounds,
        "timing": f"wall clock around the public call (host table, upload, launch, copies out), median of "
                  f"{SSA_REPEATS} calls",
    }
    if with_cpu:
        out["cpu_baseline"] = ssa_cpu_baseline()
    return out


def ssa_cpu_baseline() -> dict:
    from concurrent.futures import ThreadPoolExecutor

    driver = ROOT / "oracle" / "_ref" / "ref_ssa"
    if not driver.exists():
        return {"value": None, "unit": "paths/s", "cores": None, "kind": "reference",
                "sample": "oracle/_ref/ref_ssa not built"}
    cores = os.cpu_count() or 1
    a1, a2, n1, n2 = SSA_TOGGLE

    def one(k):
        args = [str(driver), "model=toggle", f"paths={SSA_CPU_PATHS}", "T=2", f"seed={k + 1}",
                f"a1={a1}", f"a2={a2}", f"n1={n1}", f"n2={n2}"]
        p = subprocess.run(args, capture_output=True, text=True, timeout=600)
        return p.returncode

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        rcs = list(ex.map(one, range(cores)))
    wall = time.perf_counter() - t0
    ok = sum(1 for rc in rcs if rc == 0)
    return {"value": round(ok * SSA_CPU_PATHS / wall, 1), "unit": "paths/s", "cores": cores, "kind": "reference",
            "sample": f"{SSA_CPU_PATHS} paths per core, one ref_ssa process per core, {wall:.2f} s wall"}


def _uuid(dev) -> str | None:
    import torch

    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def _time_apply(Q, N, dev, flush, reps=20) -> float:
    """Average ms of one FP64 apply_shifted (every kernel of the pass), CUDA events on its launch
    stream, each launch timed on its own with L2 flushed before it."""
    import torch

    x = torch.rand(N, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    for _ in range(3):
        Q.apply_shifted(1.0, x, y)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(reps):
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
    """dram__bytes_read.sum + dram__bytes_write.sum per apply from the committed ncu summary of
    the kernel (the row 'traffic (read + write) | X MB per apply' of profiles/<name>.md)."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("| traffic (read + write)"):
            return float(line.split("|")[2].split()[0]) * 1e6
    return None


SPMV_PROFILE = "spmv_pair_rows_birth_death_3d16"


def roofline(mk, Q, dev, N, w) -> dict:
    """The generator SpMV of the workload, the kernel the roofline target names: FP64
    apply_shifted, one compulsory read of x and write of y, 16 bytes per state (134 MB per apply
    on the 16^3 box, larger than L2), L2 flushed before each timed apply; every kernel of the
    pass is inside the timed region (the pair-strip kernel for the two-molecule rows, the
    grouped and single heavy-row kernels for the rows whose in-jumps come from every voxel)."""
    import torch

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    pk = peaks()
    ms = _time_apply(Q, N, dev, flush)
    algo = N * 16
    achieved = algo / (ms * 1e-3) / 1e9
    return {
        "kernel": "generator apply_shifted, FP64 gather SpMV (pair_strip_kernel: the two-molecule rows, a block "
                  "per pair of triangle rows; pair_heavy_group_kernel: the one-molecule rows fed from every "
                  "voxel, eight a block; pair_heavy_kernel: the empty state)",
        "bound": "hbm",
        "achieved": round(achieved, 1),
        "peak": pk["hbm_gbs"],
        "peak_source": pk["source"],
        "unit": "GB/s",
        "frac": round(achieved / pk["hbm_gbs"], 4),
        "traffic": ncu_traffic(SPMV_PROFILE) if w["workload"].startswith("rdme_birth_death_3d_16") else None,
        "traffic_source": f"profiles/{SPMV_PROFILE}.md (ncu dram bytes, the three kernels of one apply)",
        "us_per_apply": round(ms * 1e3, 3),
        "algorithmic_bytes_per_apply": algo,
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


def cpu_baseline(w, seed: int):
    """The matrix-free CPU port of the reference's path (oracle/_ref/mf_port) on this host's
    cores: one full solve of the first timed right-hand side, set-up excluded. Returns the
    baseline and the port's FP64 solution (the oracle the GPU paths are compared with)."""
    port = ROOT / "oracle" / "_ref" / "mf_port"
    if not port.exists():
        return {"value": None, "unit": "solves/s", "cores": None, "kind": "port",
                "sample": "oracle/_ref/mf_port not built"}, None
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as tmp:
        args = [str(port), *_problem_args(w), f"rhs={w['rhs']}", f"seed={seed}", "tol=1e-10",
                f"restart={RESTART}", f"threads={threads}", "solves=1", f"out={tmp}"]
        proc = subprocess.run(args, capture_output=True, text=True, timeout=3600)
        if proc.returncode != 0:
            return {"value": None, "unit": "solves/s", "cores": threads, "kind": "port",
                    "sample": proc.stderr[-200:]}, None
        m = json.loads(proc.stdout.strip().splitlines()[-1])
        x = np.fromfile(Path(tmp) / "x_port.f64", dtype=np.float64)
    secs = sum(m["solve_ms"]) / 1e3
    return {
        "value": round(1.0 / secs, 5), "unit": "solves/s", "cores": m["threads"], "kind": "port",
        "sample": f"1 full solve ({m['iterations']} MG-GMRES iterations, true rel. residual "
                  f"{m['true_rel_residual']:.2e}) after an untimed {m['setup_ms'] / 1e3:.1f} s set-up",
    }, x


REF_SAMPLE_ITERS = 3


def run_reference(args) -> None:
    """The reference's CPU path on this host's cores. For the 2-D workload the reference's own
    headers against the numerics shim (oracle/_ref/ref_driver), single-threaded as the reference
    is; for the other workloads the matrix-free port (oracle/_ref/mf_port) on all cores, because
    the reference's containers need ~275 GB and its generator set-up copies a 4096-entry state
    for each of ~3.4e10 jumps at 8.4M states. Set-up runs untimed once; one full solve gives the
    iteration count; each step is a bounded sample of REF_SAMPLE_ITERS Arnoldi iterations and
    solves/sec = REF_SAMPLE_ITERS / (iterations * step time)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    K, W = args.steps, args.warmup
    use_ref = args.workload == "annihilation_2d32"
    exe = ROOT / "oracle" / "_ref" / ("ref_driver" if use_ref else "mf_port")
    if not exe.exists():
        print(json.dumps({"impl": "reference", "unavailable": f"{exe.relative_to(ROOT)} is not built"}))
        return
    threads = 1 if use_ref else (os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as tmp:
        if use_ref:
            cmd = [str(exe), *_problem_args(w), f"rhs={w['rhs']}", f"seed={w['seed']}", "tol=1e-10",
                   f"restart={RESTART}", "do_apply=0", "do_plain=0", "warmup=1", f"solves={W + K}",
                   f"sample_iters={REF_SAMPLE_ITERS}", f"out={tmp}"]
        else:
            cmd = [str(exe), *_problem_args(w), f"rhs={w['rhs']}", f"seed={w['seed']}", "tol=1e-10",
                   f"restart={RESTART}", f"threads={threads}", "warmup=1", f"solves={W + K}",
                   f"sample_iters={REF_SAMPLE_ITERS}"]
        t0 = time.time()
        proc = subprocess.run(cmd, capture_output=True, text=True)
        wall = time.time() - t0
    if proc.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"{exe.name} failed: " +
                          proc.stderr[-200:].replace("\n", " ")}))
        return
    m = json.loads(proc.stdout.strip().splitlines()[-1])
    if use_ref:
        its = m["full_solve_iterations"]
        steps_ms = m["gmres_mg"]["solve_ms"][W:]
        setup_s = (m["box_ms"] + m["generator_ms"] + m["mg_setup_ms"]) / 1e3
        kind = "reference"
    else:
        # the warm-up solve ran to convergence: its iteration count is the full solve's
        its = m["full_iterations"]
        steps_ms = m["solve_ms"][W:]
        setup_s = m["setup_ms"] / 1e3
        kind = "port"
    per_solve_s = (sum(steps_ms) / len(steps_ms)) / 1e3 * its / REF_SAMPLE_ITERS
    value = 1.0 / per_solve_s
    sample = (f"each step: {REF_SAMPLE_ITERS} of the {its} MG-GMRES iterations of a full solve, scaled; "
              f"untimed set-up {setup_s:.0f} s; {threads} host thread(s)")
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 5), "unit": "solves/s",
        "n_gpus": args.gpus, "steps": K, "warmup": W, "ms_per_step": round(per_solve_s * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded right-hand side",
        "config": {"workload": w["workload"], "states": m["N"], "parallelism": f"{threads} host thread(s)"},
        "cpu_baseline": {"value": round(value, 5), "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 5), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1),
    }
    print(json.dumps(line), flush=True)


def relaunch_under_torchrun(args) -> None:
    """--gpus N outside torchrun: run this script as N ranks of one node."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    raise SystemExit(subprocess.call(cmd))


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the served line")
    ap.add_argument("--no-serve-mix", action="store_true", help="skip the mixed serving workload")
    ap.add_argument("--no-fsp", action="store_true", help="skip the Krylov-FSP batch line")
    ap.add_argument("--no-ssa", action="store_true", help="skip the batched SSA line")
    ap.add_argument("--no-secondary", action="store_true", help="skip the 2-D secondary workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(args)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
