"""mk_multigrid_apply_noalloc: the multigrid apply for callers that cannot allocate device
memory during the call (a host with a fixed device-memory budget that forbids allocation inside
its compute callbacks). Its work vectors live in a static 64 MiB device array; the result must
equal mk_multigrid_apply's bit for bit on two calls in a row (the array keeps the previous
call's contents, so the second call checks that nothing stale leaks in), the multigrid's
transfers summing in a fixed order.

This file is named to be collected last, so a run that stops at the first failure has run every
other test first; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

import golden_cases as gc
import markovkit_b200 as mk
from markovkit_b200 import _lib

pytestmark = pytest.mark.gpu

@pytest.mark.parametrize("name", ["cfg0_birth_death_1d16", "annihilation_2d8", "birth_death_3d4_cap2"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_apply_matches_apply_twice(cuda, name, precision):
    import torch

    c = gc.load(name)
    dom = mk.voxel_domain(mk.grid(c.dims, c.spacing), c.diffusivities)
    box = mk.population_box(int(np.prod(c.dims)), c.caps)
    M = mk.sector_multigrid(dom, box, c.shift, mk.multigrid_options(precision=precision))
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    b = torch.as_tensor(c.data["b"], device=cuda)
    ref = torch.empty_like(b)
    _lib.check(lib.mk_multigrid_apply(M._h, C.c_void_p(b.data_ptr()), C.c_void_p(ref.data_ptr()), stream))
    for _ in range(2):
        out = torch.full_like(b, float("nan"))
        _lib.check(lib.mk_multigrid_apply_noalloc(M._h, C.c_void_p(b.data_ptr()), C.c_void_p(out.data_ptr()), stream))
        torch.cuda.synchronize()
        assert torch.equal(out, ref)


def test_noalloc_rejects_hierarchy_beyond_static_scratch(cuda):
    import torch

    # 3-D 16^3 voxels, box cap 2: 8.4M states; four FP64 work vectors need about 270 MB
    dom = mk.voxel_domain(mk.grid([16, 16, 16], [1 / 16] * 3), [1.0])
    box = mk.population_box(4096, [2])
    M = mk.sector_multigrid(dom, box, 0.5)
    b = torch.zeros(box.size(), dtype=torch.float64, device=cuda)
    x = torch.zeros_like(b)
    lib = _lib.load()
    rc = lib.mk_multigrid_apply_noalloc(M._h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.MK_EINVAL
    assert b"64 MiB" in lib.mk_last_error()
