"""Python mirror of MarkovKit's resolvent-path API over the C ABI.

Names and argument meaning follow the reference: population_box / population_sector
(markovkit/rdme/population_space.hpp), grid + voxel_domain + local_reaction +
reaction_diffusion (markovkit/rdme/reaction_diffusion.hpp), generator / shifted_generator
(markovkit/generator.hpp), sector_multigrid (markovkit/rdme/multigrid.hpp) and num::gmres.
Vectors are torch CUDA tensors (device memory is torch's; the compute is the library's
sm_100a kernels). Errors raise the matching Python exceptions (ValueError for
std::invalid_argument, OverflowError for std::overflow_error).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import GmresOptions, MultigridOptions, SolverResult, check, load


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _stream(stream=None) -> C.c_void_p:
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _ints(values: Sequence[int]):
    arr = (C.c_int * len(values))(*[int(v) for v in values])
    return arr


class _Handle:
    _destroy = ""

    def __init__(self):
        self._h = C.c_void_p()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and _lib._lib is not None:
            getattr(_lib._lib, self._destroy)(h)
            self._h = C.c_void_p()


class _Space(_Handle):
    _destroy = "mk_space_destroy"

    def __init__(self, n_voxels: int, limits: Sequence[int], box: bool):
        super().__init__()
        lib = load()
        self.n_voxels_ = int(n_voxels)
        self.limits = [int(v) for v in limits]
        fn = lib.mk_space_create_box if box else lib.mk_space_create_sector
        check(fn(self.n_voxels_, len(self.limits), _ints(self.limits), C.byref(self._h)))
        self.is_box = box

    def size(self) -> int:
        n = C.c_int64()
        check(load().mk_space_size(self._h, C.byref(n)))
        return n.value

    def __len__(self) -> int:
        return self.size()

    def n_voxels(self) -> int:
        return self.n_voxels_

    def n_species(self) -> int:
        return len(self.limits)

    def n_sectors(self) -> int:
        n = C.c_int64()
        check(load().mk_space_n_sectors(self._h, C.byref(n)))
        return n.value

    def sector_begin(self, k: int) -> int:
        b = C.c_int64()
        check(load().mk_space_sector_begin(self._h, int(k), C.byref(b)))
        return b.value

    def sector_end(self, k: int) -> int:
        return self.sector_begin(k + 1)

    def sector_totals(self, k: int) -> list[int]:
        t = (C.c_int * self.n_species())()
        check(load().mk_space_sector_totals(self._h, int(k), t))
        return list(t)

    def sector_of(self, i: int) -> int:
        k = C.c_int64()
        check(load().mk_space_sector_of(self._h, int(i), C.byref(k)))
        return k.value

    def find_sector(self, totals: Sequence[int]) -> Optional[int]:
        k = C.c_int64()
        check(load().mk_space_find_sector(self._h, _ints(totals), C.byref(k)))
        return None if k.value < 0 else k.value

    def find(self, state: Sequence[int]) -> Optional[int]:
        if len(state) != self.n_voxels_ * self.n_species():
            return None
        idx = C.c_int64()
        check(load().mk_space_find_host(self._h, _ints(state), C.byref(idx)))
        return None if idx.value < 0 else idx.value

    def __getitem__(self, i: int) -> list[int]:
        out = (C.c_int * (self.n_voxels_ * self.n_species()))()
        check(load().mk_space_state_host(self._h, int(i), out))
        return list(out)

    def rank(self, states, stream=None):
        """Device ranks of a (count, n_voxels * n_species) int32 CUDA tensor; -1 if absent."""
        import torch

        count = states.shape[0]
        out = torch.empty(count, dtype=torch.int64, device=states.device)
        check(load().mk_space_rank(self._h, _ptr(states), count, _ptr(out), _stream(stream)))
        return out

    def unrank(self, index, stream=None):
        import torch

        count = index.shape[0]
        out = torch.empty((count, self.n_voxels_ * self.n_species()), dtype=torch.int32, device=index.device)
        check(load().mk_space_unrank(self._h, _ptr(index), count, _ptr(out), _stream(stream)))
        return out


class population_box(_Space):
    """Every sector with 0 <= totals[s] <= max_totals[s] (population_space.hpp:131-196)."""

    def __init__(self, n_voxels: int, max_totals: Sequence[int]):
        super().__init__(n_voxels, max_totals, True)


class population_sector(_Space):
    """Every state with totals[s] molecules of species s (population_space.hpp:105-127)."""

    def __init__(self, n_voxels: int, totals: Sequence[int]):
        super().__init__(n_voxels, totals, False)

    def totals(self) -> list[int]:
        return list(self.limits)


@dataclass
class grid:
    """Cartesian voxel grid, axis 0 fastest, closed boundary (structured_grid_graph<D>)."""

    dimensions: Sequence[int]
    spacing: Optional[Sequence[float]] = None

    def __post_init__(self):
        self.dimensions = [int(d) for d in self.dimensions]
        if self.spacing is None:
            self.spacing = [1.0] * len(self.dimensions)
        self.spacing = [float(h) for h in self.spacing]

    def n_vertices(self) -> int:
        return int(np.prod(self.dimensions))

    def cell_volume(self) -> float:
        return float(np.prod(self.spacing))


@dataclass
class voxel_domain:
    """RDME geometry (reaction_diffusion.hpp:23-56); volumes are the grid's cell volume."""

    graph: grid
    diffusivities: Sequence[float]

    def n_voxels(self) -> int:
        return self.graph.n_vertices()

    def n_species(self) -> int:
        return len(self.diffusivities)

    @property
    def volumes(self) -> list[float]:
        return [self.graph.cell_volume()] * self.n_voxels()


@dataclass
class local_reaction:
    """A reaction inside one voxel: change per species and rate(counts, volume)."""

    change: Sequence[int]
    rate: Callable[[Sequence[int], float], float]


@dataclass
class reaction_diffusion:
    domain: voxel_domain
    reactions: list = field(default_factory=list)

    def n_voxels(self) -> int:
        return self.domain.n_voxels()

    def n_species(self) -> int:
        return self.domain.n_species()

    def index(self, voxel: int, species: int) -> int:
        return voxel * self.n_species() + species


class _Model(_Handle):
    _destroy = "mk_model_destroy"

    def __init__(self, model, tuple_max: Optional[Sequence[int]] = None):
        super().__init__()
        lib = load()
        dom = model.domain if isinstance(model, reaction_diffusion) else model
        g = dom.graph
        dims = (C.c_int64 * 3)(*(list(g.dimensions) + [1] * (3 - len(g.dimensions))))
        spacing = (C.c_double * 3)(*(list(g.spacing) + [1.0] * (3 - len(g.spacing))))
        diff = (C.c_double * dom.n_species())(*dom.diffusivities)
        check(lib.mk_model_create_grid(len(g.dimensions), dims, spacing, dom.n_species(), diff, C.byref(self._h)))
        reactions = model.reactions if isinstance(model, reaction_diffusion) else []
        if reactions and tuple_max is not None:
            S = dom.n_species()
            tmax = [int(t) for t in tuple_max]
            shape = [t + 1 for t in tmax]
            ntuple = int(np.prod(shape))
            vol = g.cell_volume()
            rates = np.zeros((len(reactions), 1, ntuple))
            change = []
            for r, rx in enumerate(reactions):
                change.extend(int(c) for c in rx.change)
                for t, counts in enumerate(np.ndindex(*shape)):
                    rates[r, 0, t] = float(rx.rate(list(counts), vol))
            rates_c = rates.ravel().ctypes.data_as(C.POINTER(C.c_double))
            self._rates_keep = rates
            check(lib.mk_model_set_reactions(self._h, len(reactions), _ints(change), _ints(tmax), 1, None, rates_c))


class generator(_Handle):
    """Q of an RDME restricted to a population space (generator.hpp:17-113)."""

    _destroy = "mk_generator_destroy"

    def __init__(self, space: _Space, model: reaction_diffusion, leaks: str = "absorbing"):
        super().__init__()
        self.space = space
        self.model = _Model(model, tuple_max=list(space.limits))
        check(load().mk_generator_create(space._h, self.model._h, 1 if leaks == "absorbing" else 0, C.byref(self._h)))

    def rows(self) -> int:
        n = C.c_int64()
        check(load().mk_generator_rows(self._h, C.byref(n)))
        return n.value

    def cols(self) -> int:
        return self.rows()

    def exit_leak(self, stream=None):
        import torch

        n = self.rows()
        e = torch.empty(n, dtype=torch.float64, device="cuda")
        l = torch.empty(n, dtype=torch.float64, device="cuda")
        check(load().mk_generator_exit_leak(self._h, _ptr(e), _ptr(l), _stream(stream)))
        return e, l

    def exit_rates(self):
        return self.exit_leak()[0]

    def leak_rates(self):
        return self.exit_leak()[1]

    def apply(self, x, y, stream=None):
        import torch

        if x.dtype == torch.float32:
            check(load().mk_generator_apply_f32(self._h, _ptr(x), _ptr(y), _stream(stream)))
        else:
            check(load().mk_generator_apply(self._h, _ptr(x), _ptr(y), _stream(stream)))
        return y

    def apply_shifted(self, shift: float, x, y, stream=None):
        import torch

        if x.dtype == torch.float32:
            check(load().mk_generator_apply_shifted_f32(self._h, C.c_float(shift), _ptr(x), _ptr(y), _stream(stream)))
        else:
            check(load().mk_generator_apply_shifted(self._h, float(shift), _ptr(x), _ptr(y), _stream(stream)))
        return y

    def n_jumps(self) -> int:
        """The jumps between states of the space (generator.hpp:48)."""
        n = C.c_int64()
        check(load().mk_generator_n_jumps(self._h, C.byref(n), None))
        return n.value

    def jumps(self, j: int) -> list:
        """The jumps out of state j that stay in the space, as (to, rate) pairs in the
        reference's order (generator.hpp:50-53): diffusion by voxel, edge and species, then
        reactions by voxel and reaction. Computed on the host from the model."""
        lib = load()
        count = C.c_int64()
        check(lib.mk_generator_jumps(self._h, int(j), None, None, 0, C.byref(count)))
        to = (C.c_int64 * max(count.value, 1))()
        rate = (C.c_double * max(count.value, 1))()
        check(lib.mk_generator_jumps(self._h, int(j), to, rate, count.value, C.byref(count)))
        return [jump(int(to[k]), float(rate[k])) for k in range(count.value)]

    def matrix(self, device: bool = False):
        """Q assembled (generator.hpp:84): a scipy.sparse CSR matrix on the host, or with
        device=True a csr_matrix of device tensors."""
        return csr_matrix._assemble(self, None, device)

    def characteristic_matrix(self, shift: float, device: bool = False):
        """shift I - Q assembled (generator.hpp:87-90)."""
        return csr_matrix._assemble(self, float(shift), device)


@dataclass(frozen=True)
class jump:
    """a jump out of a state (generator.hpp:22-25)"""
    to: int
    rate: float


class csr_matrix(_Handle):
    """An assembled generator in device memory (mk_csr): row_ptr, col (int64) and val (float64)
    as CUDA tensors viewing the library's arrays; kept alive by this object."""

    _destroy = "mk_csr_destroy"

    @classmethod
    def _assemble(cls, Q: "generator", shift, device: bool):
        m = cls()
        if shift is None:
            check(load().mk_generator_matrix(Q._h, C.byref(m._h), None))
        else:
            check(load().mk_generator_characteristic_matrix(Q._h, shift, C.byref(m._h), None))
        return m if device else m.to_scipy()

    def size(self) -> tuple[int, int]:
        rows, nnz = C.c_int64(), C.c_int64()
        check(load().mk_csr_size(self._h, C.byref(rows), C.byref(nnz)))
        return rows.value, nnz.value

    def to_scipy(self):
        import numpy as np
        import scipy.sparse as sp

        rows, nnz = self.size()
        ptr = np.empty(rows + 1, dtype=np.int64)
        col = np.empty(max(nnz, 1), dtype=np.int64)
        val = np.empty(max(nnz, 1), dtype=np.float64)
        check(load().mk_csr_copy_host(self._h, ptr.ctypes.data_as(C.POINTER(C.c_int64)),
                                      col.ctypes.data_as(C.POINTER(C.c_int64)),
                                      val.ctypes.data_as(C.POINTER(C.c_double))))
        return sp.csr_matrix((val[:nnz], col[:nnz], ptr), shape=(rows, rows))

    def tensors(self):
        """(row_ptr, col, val) as CUDA tensors over the library's arrays (no copy); each
        tensor keeps this matrix alive."""
        import torch

        rows, nnz = self.size()
        p, c, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(load().mk_csr_device(self._h, C.byref(p), C.byref(c), C.byref(v)))
        return (torch.as_tensor(_DeviceArray(self, p.value, rows + 1, "<i8"), device="cuda"),
                torch.as_tensor(_DeviceArray(self, c.value, nnz, "<i8"), device="cuda"),
                torch.as_tensor(_DeviceArray(self, v.value, nnz, "<f8"), device="cuda"))


class _DeviceArray:
    """A library-owned device array seen through __cuda_array_interface__; holds its owner."""

    def __init__(self, owner, ptr, n, typestr):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr or 0), False), "version": 3}


class shifted_generator:
    """shift I - Q; reads Q by reference (generator.hpp:116-133)."""

    def __init__(self, Q: generator, shift: float):
        self.Q = Q
        self._shift = float(shift)

    def rows(self) -> int:
        return self.Q.rows()

    def cols(self) -> int:
        return self.Q.rows()

    def shift(self) -> float:
        return self._shift

    def apply(self, x, y, stream=None):
        return self.Q.apply_shifted(self._shift, x, y, stream)

    def matrix(self, device: bool = False):
        """shift I - Q assembled (generator.hpp:128)."""
        return self.Q.characteristic_matrix(self._shift, device)


def multigrid_options(**kw) -> MultigridOptions:
    o = MultigridOptions()
    load().mk_multigrid_options_default(C.byref(o))
    for k, v in kw.items():
        if k == "smoother" and isinstance(v, str):
            v = {"jacobi": 0, "gauss_seidel": 1, "ilu0": 2, "aggregate_block": 3}[v]
        if k == "precision" and isinstance(v, str):
            v = {"fp64": 0, "fp32": 1}[v]
        if k == "cycle_type" and isinstance(v, str):
            v = {"standard": 0, "k": 1}[v]
        setattr(o, k, v)
    return o


class sector_multigrid(_Handle):
    """One multigrid cycle per population sector (multigrid.hpp:369-408); on a
    population_sector it is population_multigrid (multigrid.hpp:136-361)."""

    _destroy = "mk_multigrid_destroy"

    def __init__(self, domain: voxel_domain, space: _Space, shift: float, options: Optional[MultigridOptions] = None):
        super().__init__()
        self.model = _Model(domain)
        self.space = space
        self._shift = float(shift)
        opts = options if options is not None else multigrid_options()
        self.options = opts
        check(load().mk_multigrid_create(space._h, self.model._h, float(shift), C.byref(opts), C.byref(self._h)))

    def rows(self) -> int:
        return self.level_size(0)

    def cols(self) -> int:
        return self.rows()

    def max_levels(self) -> int:
        v = C.c_int()
        check(load().mk_multigrid_max_levels(self._h, C.byref(v)))
        return v.value

    def depth(self) -> int:
        v = C.c_int()
        check(load().mk_multigrid_depth(self._h, C.byref(v)))
        return v.value

    def level_size(self, d: int) -> int:
        v = C.c_int64()
        check(load().mk_multigrid_level_size(self._h, int(d), C.byref(v)))
        return v.value

    def apply(self, b, x, stream=None):
        check(load().mk_multigrid_apply(self._h, _ptr(b), _ptr(x), _stream(stream)))
        return x

    def restrict(self, depth: int, fine, coarse, stream=None):
        check(load().mk_multigrid_restrict(self._h, int(depth), _ptr(fine), _ptr(coarse), _stream(stream)))
        return coarse

    def prolong(self, depth: int, coarse, fine, stream=None):
        check(load().mk_multigrid_prolong(self._h, int(depth), _ptr(coarse), _ptr(fine), _stream(stream)))
        return fine

    def apply_system(self, depth: int, x, y, stream=None):
        check(load().mk_multigrid_apply_system(self._h, int(depth), _ptr(x), _ptr(y), _stream(stream)))
        return y

    def smooth(self, depth: int, b, x, stream=None):
        """one sweep of the level's smoother on (b, x), in place on x (FP64 hierarchies)"""
        check(load().mk_multigrid_smooth(self._h, int(depth), _ptr(b), _ptr(x), _stream(stream)))
        return x


class _Preconditioner(_Handle):
    """A right preconditioner handle of the C ABI (mk_precond): z = M v on device vectors."""

    _destroy = "mk_precond_destroy"

    def rows(self) -> int:
        n = C.c_int64()
        check(load().mk_precond_size(self._h, C.byref(n)))
        return n.value

    def cols(self) -> int:
        return self.rows()

    def apply(self, v, z, stream=None):
        check(load().mk_precond_apply(self._h, _ptr(v), _ptr(z), _stream(stream)))
        return z


class jacobi_preconditioner(_Preconditioner):
    """num::jacobi_preconditioner(inverse_diagonal): z = d .* v
    (examples/rdme_multigrid_benchmark.cpp:109-114)."""

    def __init__(self, inverse_diagonal):
        super().__init__()
        d = np.ascontiguousarray(np.asarray(inverse_diagonal, dtype=np.float64))
        check(load().mk_precond_create_diagonal(d.size, d.ctypes.data_as(C.POINTER(C.c_double)), C.byref(self._h)))


class ilu0_preconditioner(_Preconditioner):
    """num::ilu0_preconditioner(A): ILU(0) of an assembled matrix (a scipy.sparse CSR matrix,
    e.g. shifted_generator.matrix()) in its row order, factored and applied on the device
    (examples/rdme_multigrid_benchmark.cpp:115)."""

    def __init__(self, A, stream=None):
        super().__init__()
        import scipy.sparse as sp

        A = sp.csr_matrix(A)
        A.sort_indices()
        if A.shape[0] != A.shape[1]:
            raise ValueError("ilu0_preconditioner: the matrix must be square")
        ptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
        col = np.ascontiguousarray(A.indices, dtype=np.int64)
        val = np.ascontiguousarray(A.data, dtype=np.float64)
        I64P = C.POINTER(C.c_int64)
        check(load().mk_precond_create_ilu0(A.shape[0], ptr.ctypes.data_as(I64P), col.ctypes.data_as(I64P),
                                            val.ctypes.data_as(C.POINTER(C.c_double)), _stream(stream),
                                            C.byref(self._h)))

    def schedule(self) -> dict:
        """depth of the forward and backward level sets and kernel launches per application"""
        lo, up, launches = C.c_int64(), C.c_int64(), C.c_int64()
        check(load().mk_precond_ilu0_schedule(self._h, C.byref(lo), C.byref(up), C.byref(launches)))
        return {"lower_levels": lo.value, "upper_levels": up.value, "launches_per_apply": launches.value}


class host_preconditioner(_Preconditioner):
    """Any operator as a preconditioner: fn(v) -> z on host float64 arrays of n entries, called
    on the solving thread for every application (v is copied out of and z back into device
    memory). An exception in fn fails the solve with MK_EINVAL."""

    def __init__(self, n: int, fn):
        super().__init__()
        self._fn = fn

        def trampoline(ctx, v, z, m):
            try:
                out = np.asarray(fn(np.ctypeslib.as_array(v, shape=(m,)).copy()), dtype=np.float64)
                if out.shape != (m,):
                    return 1
                np.ctypeslib.as_array(z, shape=(m,))[:] = out
                return 0
            except Exception:  # noqa: BLE001 - reported through the solve's status
                return 1

        self._cb = _lib.PRECOND_HOST_FN(trampoline)
        check(load().mk_precond_create_host(int(n), self._cb, None, C.byref(self._h)))


def _coarsened(dims: Sequence[int]):
    """coarsen() of the reference (multigrid.hpp:25-42): every axis longer than one cell halved,
    None when an axis is odd or none is longer than one"""
    if all(d == 1 for d in dims):
        return None
    out = []
    for d in dims:
        if d == 1:
            out.append(1)
        elif d % 2:
            return None
        else:
            out.append(d // 2)
    return out


class full_multigrid(sector_multigrid):
    """The paper driver's full-operator multigrid (rdme/cpp/rdme_full_multigrid.cpp:348-560,
    819-850): every level is the whole space on a coarser grid, reactions included, with the
    diffusivities doubled per level and the reactions re-tabulated at each level's voxel volume;
    the coarsest level is solved densely. Weighted Jacobi smoothing; coarse_cycles=2 for the
    W-cycle. A GMRES preconditioner (mk.solver(A, M)) or a solver of its own (stationary)."""

    def __init__(self, model: reaction_diffusion, space: _Space, shift: float,
                 options: Optional[MultigridOptions] = None):
        _Handle.__init__(self)
        self.space = space
        self._shift = float(shift)
        opts = options if options is not None else multigrid_options()
        self.options = opts
        g = model.domain.graph
        dims, spacing = list(g.dimensions), list(g.spacing)
        self._models = []
        while True:
            dom = voxel_domain(grid(dims, spacing), list(model.domain.diffusivities))
            self._models.append(_Model(reaction_diffusion(dom, model.reactions), tuple_max=list(space.limits)))
            coarse = _coarsened(dims)
            if coarse is None or len(self._models) >= opts.max_levels:
                break
            spacing = [h * 2.0 if d > 1 else h for d, h in zip(dims, spacing)]
            dims = coarse
        self.model = self._models[0]
        handles = (C.c_void_p * len(self._models))(*[m._h.value for m in self._models])
        check(load().mk_multigrid_create_full(space._h, handles, len(self._models), float(shift), C.byref(opts),
                                              C.byref(self._h)))

    def stationary(self, Q: "generator", b, x, tolerance: float, max_cycles: int = 1000, stream=None) -> "solver_result":
        """x <- x + M (b - A x) with A = shift I - Q until ||b - A x||_2 <= tolerance"""
        r = SolverResult()
        check(load().mk_multigrid_stationary(self._h, Q._h, _ptr(b), _ptr(x), float(tolerance), int(max_cycles),
                                             C.byref(r), _stream(stream)), allow=(_lib.MK_ENOTCONV,))
        return solver_result(r.iterations, r.residual, bool(r.converged), r.status)


def kernel_launches() -> int:
    """Kernels the library has launched in this process (graph launches count their nodes)."""
    v = C.c_uint64()
    check(load().mk_kernel_launches(C.byref(v)))
    return v.value


def set_row_path(path: str = "stencil") -> None:
    """Which kernel runs the rows of the solve passes: "stencil" (default: the stencil row kernel
    wherever a level allows it, the pair-strip kernel on sectors of every pair of voxels of one
    species), "general" (the general row kernel everywhere) or "no_strip" (as "stencil" without
    the pair-strip kernel). "stencil" and "no_strip" agree bit for bit; "general" agrees with them
    bit for bit on stencil forms and to rounding on pair forms. Process-wide."""
    check(load().mk_set_row_path({"stencil": 0, "general": 1, "no_strip": 2}[path]))


def gmres_options(tolerance: float = 1e-8, max_iterations: int = 1000, restart: int = 30, flexible: bool = False) -> GmresOptions:
    o = GmresOptions()
    o.tolerance = float(tolerance)
    o.max_iterations = int(max_iterations)
    o.restart = int(restart)
    o.flexible = int(bool(flexible))
    return o


@dataclass
class solver_result:
    iterations: int
    residual: float
    converged: bool
    status: int


class solver(_Handle):
    """A resident GMRES solver for shift I - Q, optionally preconditioned."""

    _destroy = "mk_solver_destroy"

    def __init__(self, A: shifted_generator, M=None, options: Optional[GmresOptions] = None):
        super().__init__()
        self.A, self.M = A, M
        opts = options if options is not None else gmres_options()
        if isinstance(M, _Preconditioner):
            check(load().mk_solver_create_pc(A.Q._h, A.shift(), M._h, C.byref(opts), C.byref(self._h)))
        else:
            check(load().mk_solver_create(A.Q._h, A.shift(), M._h if M is not None else None, C.byref(opts),
                                          C.byref(self._h)))

    def set_tolerance(self, tolerance: float) -> None:
        check(load().mk_solver_set_tolerance(self._h, float(tolerance)))

    def solve(self, b, x, stream=None) -> solver_result:
        r = SolverResult()
        check(load().mk_solver_solve(self._h, _ptr(b), _ptr(x), C.byref(r), _stream(stream)), allow=(_lib.MK_ENOTCONV,))
        return solver_result(r.iterations, r.residual, bool(r.converged), r.status)

    def solve_host(self, b: np.ndarray, x: np.ndarray, stream=None) -> solver_result:
        r = SolverResult()
        assert b.dtype == np.float64 and x.dtype == np.float64 and b.flags.c_contiguous and x.flags.c_contiguous
        check(
            load().mk_solver_solve_host(self._h, b.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p), C.byref(r), _stream(stream)),
            allow=(_lib.MK_ENOTCONV,),
        )
        return solver_result(r.iterations, r.residual, bool(r.converged), r.status)

    def time_steps(self, p, steps: int, integrator: str = "be", rel_tolerance: float = 1e-10,
                   stream=None) -> list:
        """Advance the device vector p in place by `steps` steps of backward Euler ("be", step
        1/shift) or Crank-Nicolson with a Rannacher start ("cn", shift = 2/dt, step dt), each
        solve to rel_tolerance; returns one solver_result per solve."""
        kind = {"be": 0, "cn": 1}[integrator]
        n = max(1, steps + (kind if steps > 0 else 0))
        rs = (SolverResult * n)()
        check(load().mk_solver_time_steps(self._h, kind, int(steps), float(rel_tolerance), _ptr(p), rs,
                                          _stream(stream)), allow=(_lib.MK_ENOTCONV,))
        return [solver_result(r.iterations, r.residual, bool(r.converged), r.status)
                for r in rs[: steps + (kind if steps > 0 else 0)]]


class batch_solver(_Handle):
    """Flexible GMRES for up to `width` right-hand sides of one system at once: one batched
    operator apply and one batched multigrid cycle per step (M built with batch >= width)."""

    _destroy = "mk_batch_solver_destroy"

    def __init__(self, A: shifted_generator, M: sector_multigrid, options: Optional[GmresOptions] = None,
                 width: int = 4):
        super().__init__()
        self.A, self.M, self.width = A, M, int(width)
        opts = options if options is not None else gmres_options()
        check(load().mk_batch_solver_create(A.Q._h, A.shift(), M._h, C.byref(opts), self.width, C.byref(self._h)))

    def solve(self, B, X, tolerances, stream=None) -> list:
        """B, X: (nb, n) contiguous float64 CUDA tensors (X holds initial guesses); column c
        stops at the absolute tolerance tolerances[c]"""
        nb, n = B.shape
        tol = (C.c_double * nb)(*[float(t) for t in tolerances])
        res = (SolverResult * nb)()
        check(load().mk_batch_solver_solve(self._h, _ptr(B), _ptr(X), int(B.stride(0)), nb, tol, res, _stream(stream)),
              allow=(_lib.MK_ENOTCONV,))
        return [solver_result(r.iterations, r.residual, bool(r.converged), r.status) for r in res]


def gmres(A: shifted_generator, *args, **kw) -> solver_result:
    """num::gmres(A, [M], b, x, options): x holds the initial guess and gets the solution."""
    if len(args) >= 3 and isinstance(args[0], (sector_multigrid, _Preconditioner)):
        M, b, x = args[0], args[1], args[2]
        rest = args[3:]
    else:
        M = None
        b, x = args[0], args[1]
        rest = args[2:]
    options = rest[0] if rest else kw.get("options")
    s = solver(A, M, options)
    return s.solve(b, x)
