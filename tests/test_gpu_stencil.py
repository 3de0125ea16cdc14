"""The stencil row kernels against the general row kernel on the device, and the multigrid's
fixed-order transfers. The stencil kernels serve the light rows of structured-grid levels, the
general one the rest. Rows of up to four molecules of one species (stencil forms) agree with the
general kernel bit for bit; rows of one species of cap 2 or two of cap 1 (pair forms) add the
exit terms in another order and agree to rounding (1e-14 relative here). Each path is bitwise
reproducible, and so is every multigrid cycle."""

import ctypes as C

import numpy as np
import pytest

import markovkit_b200 as mk
from markovkit_b200 import _lib

pytestmark = pytest.mark.gpu


def _birth_death(b=0.05, d=0.02):
    return [mk.local_reaction([1], lambda n, v: b * v), mk.local_reaction([-1], lambda n, v: d * n[0])]


# (grid cells per axis, dimension, diffusivities, reactions, box caps, boundary)
PROBLEMS = {
    "birth_death_1d16_cap3": ([16], [1.0], _birth_death(), [3], "absorbing"),
    "birth_death_3d16_cap2": ([16] * 3, [1.0], _birth_death(), [2], "absorbing"),
    "birth_death_3d8_cap2_reflecting": ([8] * 3, [1.0], _birth_death(2.0, 1.0), [2], "reflecting"),
    "annihilation_2d32": ([32, 32], [1.0, 1.0], [mk.local_reaction([-1, -1], lambda n, v: 10.0 * n[0] * n[1] / v)],
                          [1, 1], "absorbing"),
    "birth_death_1d128_cap4": ([128], [1.0], _birth_death(), [4], "absorbing"),
    "diffusion_2d6_cap4": ([6, 6], [0.8], [], [4], "absorbing"),
    # grids of at least 1024 voxels take the pair-strip form on their two-molecule sectors
    "birth_death_1d2048_cap2_reflecting": ([2048], [1.0], _birth_death(2.0, 1.0), [2], "reflecting"),
    "birth_death_2d32_cap2": ([32, 32], [0.7], _birth_death(), [2], "absorbing"),
}


def _problem(name):
    dims, D, rx, caps, boundary = PROBLEMS[name]
    dom = mk.voxel_domain(mk.grid(dims, [1.0 / dims[0]] * len(dims)), D)
    model = mk.reaction_diffusion(dom, rx)
    box = mk.population_box(int(np.prod(dims)), caps)
    return dom, model, box, mk.generator(box, model, boundary)


@pytest.fixture
def general_after():
    yield
    mk.set_row_path("stencil")


PAIR_SHAPES = {"birth_death_3d16_cap2", "birth_death_3d8_cap2_reflecting", "annihilation_2d32",
               "birth_death_1d2048_cap2_reflecting", "birth_death_2d32_cap2"}


def _same(a, b, name, rel=1e-14):
    import torch

    if name in PAIR_SHAPES:
        scale = float(torch.max(torch.abs(b)))
        assert float(torch.max(torch.abs(a - b))) <= rel * scale
    else:
        assert torch.equal(a, b)


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_apply_matches_general_kernel(cuda, general_after, name):
    import torch

    _, _, box, Q = _problem(name)
    n = box.size()
    g = torch.Generator(device="cpu").manual_seed(7)
    x = torch.rand(n, dtype=torch.float64, generator=g).to(cuda)
    outs = {}
    for path in ("stencil", "general"):
        mk.set_row_path(path)
        y = torch.empty_like(x)
        Q.apply_shifted(0.5, x, y)
        y32 = torch.empty(n, dtype=torch.float32, device=cuda)
        Q.apply_shifted(0.5, x.float(), y32)
        qx = torch.empty_like(x)
        Q.apply(x, qx)
        y2 = torch.empty_like(x)
        Q.apply_shifted(0.5, x, y2)
        torch.cuda.synchronize()
        assert torch.equal(y, y2)  # reproducible run to run
        outs[path] = (y.cpu(), y32.cpu().double(), qx.cpu())
    for k, (a, b) in enumerate(zip(outs["stencil"], outs["general"])):
        _same(a, b, name, 1e-6 if k == 1 else 1e-14)


@pytest.mark.parametrize("name", ["birth_death_1d16_cap3", "birth_death_3d8_cap2_reflecting", "annihilation_2d32",
                                  "diffusion_2d6_cap4"])
@pytest.mark.parametrize("smoother", ["jacobi", "gauss_seidel", "ilu0"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cycle_matches_general_and_is_reproducible(cuda, general_after, name, smoother, precision):
    """One V-cycle per kernel path, twice each: the same bits twice on each path, and the two
    paths agree (bit for bit on stencil forms, to rounding on pair forms; FP32 cycles to 1e-5)."""
    import torch

    dom, _, box, _ = _problem(name)
    n = box.size()
    g = torch.Generator(device="cpu").manual_seed(11)
    b = torch.rand(n, dtype=torch.float64, generator=g).to(cuda)
    outs = []
    for path in ("stencil", "general"):
        mk.set_row_path(path)
        M = mk.sector_multigrid(dom, box, 0.7, mk.multigrid_options(smoother=smoother, precision=precision))
        for _ in range(2):
            z = torch.empty_like(b)
            M.apply(b, z)
            torch.cuda.synchronize()
            outs.append(z.cpu())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[2], outs[3])
    if precision == "fp64":
        _same(outs[0], outs[2], name)
    else:
        scale = float(torch.max(torch.abs(outs[2])))
        assert float(torch.max(torch.abs(outs[0] - outs[2]))) <= 1e-5 * scale


@pytest.mark.parametrize("name", ["birth_death_3d16_cap2", "birth_death_1d2048_cap2_reflecting",
                                  "birth_death_2d32_cap2"])
def test_pair_strip_matches_pair_kernel_bitwise(cuda, general_after, name):
    """The pair-strip kernel (a block per pair of triangle rows, on grids of at least 1024
    voxels) on the two-molecule sectors against the stencil kernel's pair form on the same rows:
    every operator pass, FP64 and FP32, one and four right-hand sides, and V-cycles with each
    smoother, bit for bit; 1-, 2- and 3-D grids."""
    import torch

    dom, _, box, Q = _problem(name)
    n = box.size()
    g = torch.Generator(device="cpu").manual_seed(5)
    x = torch.rand(n, dtype=torch.float64, generator=g).to(cuda)
    xb = torch.rand(4, n, dtype=torch.float64, generator=g).to(cuda)
    outs = {}
    for path in ("stencil", "no_strip"):
        mk.set_row_path(path)
        r = []
        for dt in (torch.float64, torch.float32):
            y = torch.empty(n, dtype=dt, device=cuda)
            Q.apply_shifted(0.5, x.to(dt), y)
            r.append(y.double().cpu())
            qx = torch.empty(n, dtype=dt, device=cuda)
            Q.apply(x.to(dt), qx)
            r.append(qx.double().cpu())
        yb = torch.empty_like(xb)
        _lib.check(_lib.load().mk_generator_apply_shifted_batch(
            Q._h, 0.5, C.c_void_p(xb.data_ptr()), C.c_void_p(yb.data_ptr()), n, 4,
            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        r.append(yb.cpu())
        for smoother in ("jacobi", "gauss_seidel", "ilu0"):
            for precision in ("fp64", "fp32"):
                M = mk.sector_multigrid(dom, box, 0.7, mk.multigrid_options(smoother=smoother, precision=precision))
                z = torch.empty_like(x)
                M.apply(x, z)
                r.append(z.cpu())
        torch.cuda.synchronize()
        outs[path] = r
    for k, (a, b) in enumerate(zip(outs["stencil"], outs["no_strip"])):
        assert torch.equal(a, b), k
