"""Small fixed workloads of the library's kernels, for running under a profiler.

    python -m markovkit_b200.profile_kernels <case>

Cases:
  spmv_birth_death_3d16      FP64 generator apply_shifted on the 3-D 16^3-voxel birth-death box of
                             cap 2 (8,394,753 states): 2 untimed launches, then 3 more
  solve_annihilation_2d32    one FP32-multigrid FGMRES resolvent solve of the 2-D 32 x 32
                             annihilation box {1, 1} (1,050,625 states) after one warm-up solve,
                             red-black Gauss-Seidel smoothing as the bench's FP32 path
  solve_birth_death_3d16     the same on the 3-D box above
  mg_birth_death_3d16        one FP32 sector-multigrid V-cycle on the 3-D box (after one warm-up)
  mg_annihilation_2d32       the same on the 2-D annihilation box (sectors of <= 256 states
                             solved densely)
  fsp_toggle                 one batched Krylov-FSP launch of 8 toggle-switch instances of the
                             batching workload (after one warm-up launch)
  ssa_toggle                 two batched-SSA launches of 65,536 Gillespie paths of the bench's
                             toggle switch to t = 2 (the second is the one to capture)

Each prints one JSON line with what it ran. Nothing here is timed: profilers time the kernels.
"""

from __future__ import annotations

import json
import sys

import numpy as np


def _rdme(mk, dim, cells, caps, model, shift):
    h = 1.0 / cells
    D = [1.0] * len(caps)
    dom = mk.voxel_domain(mk.grid([cells] * dim, [h] * dim), D)
    if model == "annihilation":
        rx = [mk.local_reaction([-1, -1], lambda n, vol: 10.0 * n[0] * n[1] / vol)]
    else:
        rx = [mk.local_reaction([1], lambda n, vol: 0.05 * vol),
              mk.local_reaction([-1], lambda n, vol: 0.02 * n[0])]
    model_ = mk.reaction_diffusion(dom, rx)
    box = mk.population_box(cells ** dim, caps)
    Q = mk.generator(box, model_, "absorbing")
    return dom, box, Q, mk.shifted_generator(Q, shift)


def main(case: str) -> None:
    import torch

    import markovkit_b200 as mk
    from markovkit_b200.inputs import dirichlet_rhs, uniform_rhs

    dev = torch.device("cuda", 0)
    if case == "spmv_birth_death_3d16":
        _, box, Q, _ = _rdme(mk, 3, 16, [2], "birth_death", 0.5)
        x = torch.rand(box.size(), dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        for _ in range(5):
            Q.apply_shifted(1.0, x, y)
        torch.cuda.synchronize()
        print(json.dumps({"case": case, "states": box.size(), "launches": 5}))
    elif case in ("solve_annihilation_2d32", "solve_birth_death_3d16", "mg_birth_death_3d16",
                  "mg_annihilation_2d32"):
        if case in ("solve_annihilation_2d32", "mg_annihilation_2d32"):
            dom, box, Q, A = _rdme(mk, 2, 32, [1, 1], "annihilation", 1.0)
            rhs = dirichlet_rhs
        else:
            dom, box, Q, A = _rdme(mk, 3, 16, [2], "birth_death", 0.5)
            rhs = uniform_rhs
        N = box.size()
        M = mk.sector_multigrid(dom, box, A.shift(), mk.multigrid_options(precision="fp32", coarsest_size=256,
                                                                          smoother="gauss_seidel"))
        if case.startswith("mg_"):
            b = torch.from_numpy(rhs(2, N)).to(dev)
            x = torch.zeros_like(b)
            M.apply(b, x)
            M.apply(b, x)
            torch.cuda.synchronize()
            print(json.dumps({"case": case, "states": N, "cycles": 2}))
            return
        its = []
        for seed in (1, 2):
            b = torch.from_numpy(rhs(seed, N)).to(dev)
            x = torch.zeros_like(b)
            s = mk.solver(A, M, mk.gmres_options(tolerance=1e-10 * float(torch.linalg.norm(b)),
                                                 max_iterations=2000, restart=30, flexible=True))
            its.append(s.solve(b, x).iterations)
        torch.cuda.synchronize()
        print(json.dumps({"case": case, "states": N, "solves": 2, "iterations": its}))
    elif case == "fsp_toggle":
        from markovkit_b200.fsp import _Problem, box as fbox, fsp_batch, krylov_fsp_options
        from markovkit_b200.fsp_models import network_of
        from markovkit_b200.inputs import fsp_batch_instances

        inst = [x for x in fsp_batch_instances() if x["family"] == "toggle"][:8]
        probs = [_Problem(network_of(x), x["initial"], x["final_time"],
                          krylov_fsp_options(inside=fbox(x["bounds"]), tolerance=x["tolerance"], max_steps=2000))
                 for x in inst]
        b = fsp_batch(probs)
        b.run()
        b.run()
        _, res = b.results()
        print(json.dumps({"case": case, "instances": len(probs), "applies": int(sum(r.applies for r in res))}))
    elif case == "ssa_toggle":
        from markovkit_b200.fsp_models import toggle
        from markovkit_b200.ssa import simulate

        model = toggle(30.0, 25.0, 2.0, 2.5)
        for seed in (1, 2):
            ens = simulate(model, [0, 0], 2.0, 65536, seed=seed, bounds=[64, 64])
        print(json.dumps({"case": case, "paths": 65536, "launches": 2, "jumps": int(ens.steps.sum())}))
    else:
        raise SystemExit(f"unknown case {case!r}; see the module docstring")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "")
