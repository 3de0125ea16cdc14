// The stencil row kernels: one thread per light row of a structured-grid level (two consecutive
// rows per thread in the colour passes of Gauss-Seidel and ILU(0), so that the rows of the other
// colour cost a warp no lanes), for the passes of the solve, each pass a separate instantiation.
// Rows of one species of at most two molecules or two species of at most one take the pair and
// single-molecule forms (pair_rows.cuh); rows of up to four molecules of one species the stencil
// forms (stencil_row.cuh). Rows whose in-jumps come from every voxel take pair_heavy_kernel in the
// operator passes (a warp or a block per row); the rows of two-molecule sectors of one species
// take pair_strip_kernel (a block per pair of triangle rows). The build compiles this file once per (precision
// MK_T, batch width MK_NB); the tiles each kernel gets list only rows its forms serve.
#include "pair_rows.cuh"
#include "row_kernels_impl.cuh"
#include "stencil_row.cuh"

#include <type_traits>

#if !defined(MK_T) || !defined(MK_NB)
#error "compile with -DMK_T=<double|float> -DMK_NB=<1|4>"
#endif

namespace mkb::detail {
namespace {

static_assert(sizeof(SectorDesc) % sizeof(int) == 0, "sector descriptors copy as words");
static_assert(sizeof(StencilSector<MK_T>) % sizeof(int) == 0, "stencil sectors copy as words");

template <int MODE>
constexpr bool kColourPass = MODE == kGaussSeidel || MODE == kIluFirst || MODE == kIluSecond ||
                             MODE == kIluThird;
template <int MODE>
constexpr int kRowsPerThread = kColourPass<MODE> ? 2 : 1;

template <typename S>
__device__ __forceinline__ void copy_to_shared(const S *src, S &dst) {
    constexpr int kWords = static_cast<int>(sizeof(S) / sizeof(int));
    const int *from = reinterpret_cast<const int *>(src);
    int *to = reinterpret_cast<int *>(&dst);
    for (int k = static_cast<int>(threadIdx.x); k < kWords; k += static_cast<int>(blockDim.x)) {
        to[k] = from[k];
    }
}

// the value at p, read only when on (a bool: the read is predicated, the sum gets 0 otherwise);
// an `on` of another type is a visitor's reverse rate and the read always happens
template <typename T, typename On>
__device__ __forceinline__ T fetch(On on, const T *p) {
    if constexpr (std::is_same_v<On, bool>) {
        T v = T(0);
        if (on) {
            v = *p;
        }
        return v;
    } else {
        return *p;
    }
}

template <typename On>
__device__ __forceinline__ float4 fetch4(On on, const float *p) {
    if constexpr (std::is_same_v<On, bool>) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (on) {
            v = *reinterpret_cast<const float4 *>(p);
        }
        return v;
    } else {
        return *reinterpret_cast<const float4 *>(p);
    }
}

// The in-jump sums of one row for pass MODE (row_terms for any row visitor):
// visit(std::bool_constant<WANT_IN>, acc) runs the row with acc(source, rate, on), where `on`
// is a bool for visitors that name candidate in-jumps (see fetch) and a reverse rate otherwise.
template <typename T, int NB, int MODE, typename Visit>
__device__ __forceinline__ void accumulate_terms(const RowParams<T> &p, Visit &&visit, T (&in)[NB],
                                                 T (&in2)[NB]) {
    if constexpr (MODE == kJacobiZero) {
        visit(std::false_type{}, [](int, T, auto) {});
        return;
    } else {
        // Gauss-Seidel and the ILU passes update x (= y) in place: rows of one colour read only
        // the other colour's entries, through plain coherent loads
        const T *xs = MODE == kGaussSeidel ? p.y : p.x;
        const T *ax = p.aux;
        if constexpr (NB == 1) {
            if constexpr (MODE == kIluThird) {
                visit(std::true_type{}, [&](int j, T a, auto on) { in2[0] += a * fetch(on, ax + j); });
            } else if constexpr (MODE == kIluSecond) {
                visit(std::true_type{}, [&](int j, T a, auto on) {
                    in[0] += a * fetch(on, xs + j);
                    in2[0] += a * fetch(on, ax + j);
                });
            } else {
                visit(std::true_type{}, [&](int j, T a, auto on) { in[0] += a * fetch(on, xs + j); });
            }
        } else if constexpr (kInterleaved<T, NB>) {
            // the kRowBatch source values of an in-jump in one 16-byte load
            visit(std::true_type{}, [&](int j, T a, auto on) {
                const std::int64_t k = static_cast<std::int64_t>(j) * NB;
                if constexpr (MODE != kIluThird) {
                    const float4 v = fetch4(on, xs + k);
                    in[0] += a * v.x;
                    in[1] += a * v.y;
                    in[2] += a * v.z;
                    in[3] += a * v.w;
                }
                if constexpr (MODE == kIluSecond || MODE == kIluThird) {
                    const float4 u = fetch4(on, ax + k);
                    in2[0] += a * u.x;
                    in2[1] += a * u.y;
                    in2[2] += a * u.z;
                    in2[3] += a * u.w;
                }
            });
        } else {
            const int nb = p.nb;
            const std::int64_t ldv = p.ldv;
            visit(std::true_type{}, [&](int j, T a, auto on) {
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    if (c >= nb) {
                        break;
                    }
                    const std::int64_t k = j + c * ldv;
                    if constexpr (MODE == kIluThird) {
                        in2[c] += a * fetch(on, ax + k);
                    } else {
                        in[c] += a * fetch(on, xs + k);
                        if constexpr (MODE == kIluSecond) {
                            in2[c] += a * fetch(on, ax + k);
                        }
                    }
                }
            });
        }
    }
}

// rows of up to four molecules of one species (stencil_row.cuh)
template <typename T, int NB, int MODE>
__global__ void __launch_bounds__(kRowBlock) stencil_kernel(const __grid_constant__ RowParams<T> p) {
    constexpr int NS = 1, TMAX = 4, RPT = kRowsPerThread<MODE>;
    __shared__ SectorDesc s_sec;
    const Tile tile = p.tiles[blockIdx.x];
    if (p.sector_class >= 0 && p.sectors[tile.sector].gs_class != p.sector_class) {
        return; // another colour class's pass (the whole block)
    }
    copy_to_shared(p.sectors + tile.sector, s_sec);
    __syncthreads();
    const SectorDesc &sec = s_sec;
    const int colour = pass_colour(MODE, p.colour);
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
        const int in_tile = static_cast<int>(threadIdx.x) * RPT + q;
        if (in_tile >= tile.count) {
            break;
        }
        const int local = static_cast<int>(tile.local0) + in_tile;
        const int row = static_cast<int>(sec.begin) + local;
        StencilState<NS, TMAX> st;
        stencil_load<T, NS, TMAX>(sec, p.md, local, st);
        if (colour >= 0 && stencil_colour<NS, TMAX>(st) != colour) {
            continue;
        }
        T exit = T(0), leak = T(0);
        T in[NB], in2[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            in[c] = T(0);
            in2[c] = T(0);
        }
        accumulate_terms<T, NB, MODE>(
            p,
            [&](auto want_in, auto &&acc) {
                stencil_visit<T, NS, TMAX, decltype(want_in)::value>(p.B, p.sectors, sec, p.md, st,
                                                                     row, exit, leak, acc);
            },
            in, in2);
        finish_row<T, NB, MODE>(p, row, exit, leak, in, in2);
    }
}

// the molecules and voxel masks of one pair or single-molecule row
struct PairState {
    int u0 = 0, u1 = 0;
    unsigned m0 = 0U, m1 = 0U;
};

template <int NS, typename T>
__device__ __forceinline__ PairState pair_load(const StencilSector<T> &ss, const ModelView<T> &md,
                                               int local) {
    PairState s;
    const int V = md.V;
    if constexpr (NS == 1) {
        const int t = ss.total[0];
        if (t == 2) {
            unrank_pair(local, s.u0, s.u1);
            s.m1 = load_ro(md.vmask + (V - 1 - s.u1));
        } else {
            s.u0 = local;
        }
        if (t >= 1) {
            s.m0 = load_ro(md.vmask + (V - 1 - s.u0));
        }
    } else {
        // species 0's rank is the quotient by stride0 (one molecule: rank = u)
        if (ss.total[0] && ss.total[1]) {
            s.u0 = div_small(local, ss.stride0, 1.0f / static_cast<float>(ss.stride0));
            s.u1 = local - s.u0 * ss.stride0;
        } else {
            s.u0 = s.u1 = local;
        }
        if (ss.total[0]) {
            s.m0 = load_ro(md.vmask + (V - 1 - s.u0));
        }
        if (ss.total[1]) {
            s.m1 = load_ro(md.vmask + (V - 1 - s.u1));
        }
    }
    return s;
}

// rows of one species of at most two molecules (NS = 1) or two species of at most one (NS = 2)
template <typename T, int NS, int NB, int MODE>
__global__ void __launch_bounds__(kRowBlock) pair_kernel(const __grid_constant__ RowParams<T> p) {
    constexpr int RPT = kRowsPerThread<MODE>;
    __shared__ StencilSector<T> s_ss;
    const Tile tile = p.tiles[blockIdx.x];
    if (p.sector_class >= 0 && p.sectors[tile.sector].gs_class != p.sector_class) {
        return; // another colour class's pass (the whole block)
    }
    copy_to_shared(p.sv.sectors + tile.sector, s_ss);
    __syncthreads();
    const StencilSector<T> &ss = s_ss;
    const int colour = pass_colour(MODE, p.colour);
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
        const int in_tile = static_cast<int>(threadIdx.x) * RPT + q;
        if (in_tile >= tile.count) {
            break;
        }
        const int local = static_cast<int>(tile.local0) + in_tile;
        const int row = ss.begin + local;
        const PairState s = pair_load<NS>(ss, p.md, local);
        if (colour >= 0 && static_cast<int>(((s.m0 ^ s.m1) >> kVoxelColourBit) & 1U) != colour) {
            continue;
        }
        T exit = T(0), leak = T(0);
        T in[NB], in2[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            in[c] = T(0);
            in2[c] = T(0);
        }
        accumulate_terms<T, NB, MODE>(
            p,
            [&](auto want_in, auto &&acc) {
                constexpr bool W = decltype(want_in)::value;
                if constexpr (NS == 1) {
                    pair_row<T, W>(p.md, p.sv, ss, ss.total[0], s.u0, s.u1, s.m0, s.m1, row, exit,
                                   leak, acc);
                } else {
                    singles_row<T, W>(p.md, p.sv, ss, s.u0, s.u1, s.m0, s.m1, row, exit, leak, acc);
                }
            },
            in, in2);
        finish_row<T, NB, MODE>(p, row, exit, leak, in, in2);
    }
}

// Rows of one species whose in-jumps come from every voxel (tile kind 1: a warp per row, kind 2:
// the block), in the operator passes: lane 0 takes the row's light terms, every lane a share of
// the voxels; sums in a fixed order.
template <typename T, int NB, int MODE>
__global__ void __launch_bounds__(kRowBlock) pair_heavy_kernel(const __grid_constant__ RowParams<T> p) {
    __shared__ StencilSector<T> s_ss;
    __shared__ T s_red[2 + NB][kRowBlock / 32];
    const Tile tile = p.tiles[blockIdx.x];
    if (p.sector_class >= 0 && p.sectors[tile.sector].gs_class != p.sector_class) {
        return; // another colour class's pass (the whole block)
    }
    copy_to_shared(p.sv.sectors + tile.sector, s_ss);
    __syncthreads();
    const StencilSector<T> &ss = s_ss;
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    int local, row_lane, row_lanes;
    if (tile.kind == 1) {
        if (warp >= tile.count) {
            return;
        }
        local = static_cast<int>(tile.local0) + warp;
        row_lane = lane;
        row_lanes = 32;
    } else {
        local = static_cast<int>(tile.local0);
        row_lane = static_cast<int>(threadIdx.x);
        row_lanes = kRowBlock;
    }
    const int row = ss.begin + local;
    const PairState s = pair_load<1>(ss, p.md, local);
    const int t = ss.total[0];
    T exit = T(0), leak = T(0);
    T in[NB], in2[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = T(0);
        in2[c] = T(0);
    }
    accumulate_terms<T, NB, MODE>(
        p,
        [&](auto want_in, auto &&acc) {
            constexpr bool W = decltype(want_in)::value;
            if (row_lane == 0) {
                pair_row<T, W>(p.md, p.sv, ss, t, s.u0, s.u1, s.m0, s.m1, row, exit, leak, acc);
            }
            if constexpr (W) {
                pair_heavy_terms<T>(ss, p.md.V, t, s.u0, row_lane, row_lanes, acc);
            }
        },
        in, in2);
    exit = warp_sum(exit);
    leak = warp_sum(leak);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = warp_sum(in[c]);
    }
    if (tile.kind == 1) {
        if (lane == 0) {
            finish_row<T, NB, MODE>(p, row, exit, leak, in, in2);
        }
        return;
    }
    if (lane == 0) {
        s_red[0][warp] = exit;
        s_red[1][warp] = leak;
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            s_red[2 + c][warp] = in[c];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        exit = leak = T(0);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            in[c] = T(0);
        }
        for (int w = 0; w < kRowBlock / 32; ++w) {
            exit += s_red[0][w];
            leak += s_red[1][w];
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                in[c] += s_red[2 + c][w];
            }
        }
        finish_row<T, NB, MODE>(p, row, exit, leak, in, in2);
    }
}

// One row of pair_strip_kernel: FAR (outside the band) with its sources at the row's fixed
// offsets, else pair_row's form; exit, leak and the sums stay in registers.
template <typename T, int NB, int MODE, bool FAR>
__device__ __forceinline__ void strip_row(const RowParams<T> &p, const StencilSector<T> &ss, int u0, int w,
                                          unsigned m0, unsigned m1, int row, int up0, int up1, int up2,
                                          int down0, int down1, int down2) {
    T exit = T(0), leak = T(0);
    T in[NB], in2[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = T(0);
        in2[c] = T(0);
    }
    accumulate_terms<T, NB, MODE>(
        p,
        [&](auto want_in, auto &&acc) {
            constexpr bool W = decltype(want_in)::value;
            if constexpr (!FAR) {
                pair_row<T, W>(p.md, p.sv, ss, 2, u0, w, m0, m1, row, exit, leak, acc);
            } else {
                pair_row<T, false>(p.md, p.sv, ss, 2, u0, w, m0, m1, row, exit, leak, acc);
                if constexpr (W) {
                    // the axes in order, as pair_row; an axis past the grid's adds 0 (no read)
                    const int gd = p.md.grid_dim;
                    const int g0 = p.md.gstride[0], g1 = p.md.gstride[1], g2 = p.md.gstride[2];
                    acc(row + g0, p.sv.da[0][0], gd > 0 && has_lower(m0, 0));
                    acc(row - g0, p.sv.da[0][0], gd > 0 && has_upper(m0, 0));
                    acc(row + g1, p.sv.da[0][1], gd > 1 && has_lower(m0, 1));
                    acc(row - g1, p.sv.da[0][1], gd > 1 && has_upper(m0, 1));
                    acc(row + g2, p.sv.da[0][2], gd > 2 && has_lower(m0, 2));
                    acc(row - g2, p.sv.da[0][2], gd > 2 && has_upper(m0, 2));
                    acc(row + up0, p.sv.da[0][0], gd > 0 && has_lower(m1, 0));
                    acc(row + down0, p.sv.da[0][0], gd > 0 && has_upper(m1, 0));
                    acc(row + up1, p.sv.da[0][1], gd > 1 && has_lower(m1, 1));
                    acc(row + down1, p.sv.da[0][1], gd > 1 && has_upper(m1, 1));
                    acc(row + up2, p.sv.da[0][2], gd > 2 && has_lower(m1, 2));
                    acc(row + down2, p.sv.da[0][2], gd > 2 && has_upper(m1, 2));
                    for (int k = 0; k < ss.n_in; ++k) {
                        if (ss.in_copies[k] == 1) {
                            const T a = ss.rin[k][1];
                            if (a > T(0)) {
                                acc(ss.in_src[k] + w, a, true);
                                acc(ss.in_src[k] + u0, a, true);
                            }
                        }
                    }
                }
            }
        },
        in, in2);
    finish_row<T, NB, MODE>(p, row, exit, leak, in, in2);

}

// Rows of a two-molecule sector of one species (u0 <= u1, rank u0 + T(u1): every pair of V
// voxels) a block per pair of triangle rows u1 = w and V - 1 - w, so that every block takes
// V + 1 rows and no row is unranked. A row outside the band u1 - u0 <= gmax has its sources at
// offsets fixed per triangle row (computed once per row w); it visits the same in-jumps in the
// same order as pair_row, whose other rows it calls, so the results equal pair_kernel's bit for
// bit. p.tiles: kind-3 tiles, local0 = the pair index.
template <typename T, int NB, int MODE>
__global__ void __launch_bounds__(kRowBlock, NB == 1 ? 5 : 4) pair_strip_kernel(const __grid_constant__ RowParams<T> p) {
    __shared__ StencilSector<T> s_ss;
    const Tile tile = p.tiles[blockIdx.x];
    if (p.sector_class >= 0 && p.sectors[tile.sector].gs_class != p.sector_class) {
        return; // another colour class's pass (the whole block)
    }
    copy_to_shared(p.sv.sectors + tile.sector, s_ss);
    __syncthreads();
    const StencilSector<T> &ss = s_ss;
    const int V = p.md.V;
    const int colour = pass_colour(MODE, p.colour);
    const int pair = static_cast<int>(tile.local0);
    for (int h = 0; h < 2; ++h) {
        const int w = h == 0 ? pair : V - 1 - pair;
        if (h == 1 && w == pair) {
            break;
        }
        const int tw = tri(w);
        const unsigned m1 = load_ro(p.md.vmask + (V - 1 - w));
        // molecule 1 from w + g and from w - g, relative to the row, per axis
        const int g0 = p.md.gstride[0], g1 = p.md.gstride[1], g2 = p.md.gstride[2];
        const int up0 = g0 * w + tri(g0), up1 = g1 * w + tri(g1), up2 = g2 * w + tri(g2);
        const int down0 = -g0 * w + tri(g0 - 1), down1 = -g1 * w + tri(g1 - 1), down2 = -g2 * w + tri(g2 - 1);
        const int far_end = w - p.sv.gmax; // rows u0 < far_end are outside the band
        // colour passes: two consecutive rows per thread, of which mostly one has the pass's colour
        // (the colours alternate along a grid line), so that few lanes idle
        constexpr int RPT = kRowsPerThread<MODE>;
        for (int base = RPT * static_cast<int>(threadIdx.x); base <= w; base += RPT * kRowBlock) {
#pragma unroll
            for (int q = 0; q < RPT; ++q) {
                const int u0 = base + q;
                if (u0 > w) {
                    break;
                }
                const int row = ss.begin + tw + u0;
                const unsigned m0 = load_ro(p.md.vmask + (V - 1 - u0));
                if (colour >= 0 && static_cast<int>(((m0 ^ m1) >> kVoxelColourBit) & 1U) != colour) {
                    continue;
                }
                if (u0 < far_end) {
                    strip_row<T, NB, MODE, true>(p, ss, u0, w, m0, m1, row, up0, up1, up2, down0, down1, down2);
                } else {
                    strip_row<T, NB, MODE, false>(p, ss, u0, w, m0, m1, row, up0, up1, up2, down0, down1, down2);
                }
            }
        }
    }
}

constexpr int kHeavyGroup = kHeavyGroupRows;           // rows of a group tile
constexpr int kHeavyThreads = 1024;                     // threads of a group's block
constexpr int kHeavySlots = kHeavyThreads / kHeavyGroup; // threads per row of the group

// Rows of one molecule (u = local) of one species whose heavy reactions come from the pair sector
// (the source holds one more copy in any voxel w: {w, u} of rank min + T(max)), kHeavyGroup rows
// u0 .. u0 + count - 1 a block (kind-4 tiles). Thread (slot, j) takes row j and the voxels
// w = slot, slot + kHeavySlots, ...; the threads of one w read the sources of the group's rows
// side by side: {u, w} for w > u sits at u + T(w), so the group's sources of one w are adjacent.
// Per row the sums run over w in a fixed order and meet in a fixed tree; the row's own terms
// (pair_row) come last. Operator passes only (kApplyQ, kApplyShifted, kResidual).
template <typename T, int NB, int MODE>
__global__ void __launch_bounds__(kHeavyThreads) pair_heavy_group_kernel(const __grid_constant__ RowParams<T> p) {
    __shared__ StencilSector<T> s_ss;
    __shared__ T s_red[kHeavyThreads / 32][kHeavyGroup][NB];
    const Tile tile = p.tiles[blockIdx.x];
    if (p.sector_class >= 0 && p.sectors[tile.sector].gs_class != p.sector_class) {
        return;
    }
    copy_to_shared(p.sv.sectors + tile.sector, s_ss);
    __syncthreads();
    const StencilSector<T> &ss = s_ss;
    const int V = p.md.V;
    const int j = static_cast<int>(threadIdx.x) % kHeavyGroup;
    const int slot = static_cast<int>(threadIdx.x) / kHeavyGroup;
    const int u0 = static_cast<int>(tile.local0);
    const int u = u0 + j;
    const bool active = j < tile.count;
    T in[NB], in2[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] = T(0);
        in2[c] = T(0);
    }
    accumulate_terms<T, NB, MODE>(
        p,
        [&](auto want_in, auto &&acc) {
            if constexpr (decltype(want_in)::value) {
                const int tu = tri(u);
                for (int k = 0; k < ss.n_heavy; ++k) {
                    const int src = ss.heavy_src[k];
                    const T a0 = ss.rheavy[k][0], a1 = ss.rheavy[k][1];
                    // {w, u} for w <= u: the run src + T(u) .. src + T(u) + u
#pragma unroll 4
                    for (int w = slot; w <= u; w += kHeavySlots) {
                        const T a = w == u ? a1 : a0;
                        acc(src + tu + w, a, active && a > T(0));
                    }
                    // {u, w} for w > u: src + u + T(w), the group's rows side by side
#pragma unroll 4
                    for (int w = u0 + 1 + slot; w < V; w += kHeavySlots) {
                        acc(src + u + tri(w), a0, active && w > u && a0 > T(0));
                    }
                }
            }
        },
        in, in2);
    // the threads of row j: lanes j, j + 8, j + 16, j + 24 of each warp, then the warps in order
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        in[c] += __shfl_xor_sync(0xffffffffU, in[c], 8);
        in[c] += __shfl_xor_sync(0xffffffffU, in[c], 16);
    }
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    if (lane < kHeavyGroup) {
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            s_red[warp][lane][c] = in[c];
        }
    }
    __syncthreads();
    if (threadIdx.x >= static_cast<unsigned>(tile.count)) {
        return;
    }
    // thread j < count: the row's own terms, then the heavy sum
    const int row = ss.begin + u;
    const unsigned m = load_ro(p.md.vmask + (V - 1 - u));
    T exit = T(0), leak = T(0);
    T own[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        own[c] = T(0);
    }
    accumulate_terms<T, NB, MODE>(
        p,
        [&](auto want_in, auto &&acc) {
            constexpr bool W = decltype(want_in)::value;
            pair_row<T, W>(p.md, p.sv, ss, 1, u, 0, m, 0U, row, exit, leak, acc);
        },
        own, in2);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        T h = T(0);
        for (int w = 0; w < kHeavyThreads / 32; ++w) {
            h += s_red[w][j][c];
        }
        own[c] += h;
    }
    finish_row<T, NB, MODE>(p, row, exit, leak, own, in2);
}

template <typename T, int NB, int MODE>
cudaError_t launch_light(const RowParams<T> &p, int S, int cap, cudaStream_t stream) {
    const int threads = kRowBlock / kRowsPerThread<MODE>;
    if (pair_shape(S, cap)) {
        if (!p.sv.sectors) {
            return cudaErrorInvalidValue;
        }
        if (S == 1) {
            pair_kernel<T, 1, NB, MODE><<<p.n_tiles, threads, 0, stream>>>(p);
        } else {
            pair_kernel<T, 2, NB, MODE><<<p.n_tiles, threads, 0, stream>>>(p);
        }
    } else {
        stencil_kernel<T, NB, MODE><<<p.n_tiles, threads, 0, stream>>>(p);
    }
    return cudaGetLastError();
}

} // namespace

template <typename T, int NB>
cudaError_t launch_stencil(const RowParams<T> &p, int S, int cap, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    count_launches(1);
    switch (p.mode) {
    case kApplyQ:
        return launch_light<T, NB, kApplyQ>(p, S, cap, stream);
    case kApplyShifted:
        return launch_light<T, NB, kApplyShifted>(p, S, cap, stream);
    case kResidual:
        return launch_light<T, NB, kResidual>(p, S, cap, stream);
    case kJacobiZero:
        return launch_light<T, NB, kJacobiZero>(p, S, cap, stream);
    case kJacobi:
        return launch_light<T, NB, kJacobi>(p, S, cap, stream);
    case kGaussSeidel:
        return launch_light<T, NB, kGaussSeidel>(p, S, cap, stream);
    case kIluFirst:
        return launch_light<T, NB, kIluFirst>(p, S, cap, stream);
    case kIluSecond:
        return launch_light<T, NB, kIluSecond>(p, S, cap, stream);
    case kIluThird:
        return launch_light<T, NB, kIluThird>(p, S, cap, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

template <typename T, int NB>
cudaError_t launch_pair_heavy(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    if (!p.sv.sectors) {
        return cudaErrorInvalidValue;
    }
    count_launches(1);
    switch (p.mode) {
    case kApplyQ:
        pair_heavy_kernel<T, NB, kApplyQ><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kApplyShifted:
        pair_heavy_kernel<T, NB, kApplyShifted><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kResidual:
        pair_heavy_kernel<T, NB, kResidual><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, int NB>
cudaError_t launch_pair_heavy_group(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    if (!p.sv.sectors) {
        return cudaErrorInvalidValue;
    }
    count_launches(1);
    switch (p.mode) {
    case kApplyQ:
        pair_heavy_group_kernel<T, NB, kApplyQ><<<p.n_tiles, kHeavyThreads, 0, stream>>>(p);
        break;
    case kApplyShifted:
        pair_heavy_group_kernel<T, NB, kApplyShifted><<<p.n_tiles, kHeavyThreads, 0, stream>>>(p);
        break;
    case kResidual:
        pair_heavy_group_kernel<T, NB, kResidual><<<p.n_tiles, kHeavyThreads, 0, stream>>>(p);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, int NB>
cudaError_t launch_pair_strip(const RowParams<T> &p, cudaStream_t stream) {
    if (p.n_tiles == 0) {
        return cudaSuccess;
    }
    if (!p.sv.sectors) {
        return cudaErrorInvalidValue;
    }
    count_launches(1);
    switch (p.mode) {
    case kApplyQ:
        pair_strip_kernel<T, NB, kApplyQ><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kApplyShifted:
        pair_strip_kernel<T, NB, kApplyShifted><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kResidual:
        pair_strip_kernel<T, NB, kResidual><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kJacobiZero:
        pair_strip_kernel<T, NB, kJacobiZero><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kJacobi:
        pair_strip_kernel<T, NB, kJacobi><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kGaussSeidel:
        pair_strip_kernel<T, NB, kGaussSeidel><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kIluFirst:
        pair_strip_kernel<T, NB, kIluFirst><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kIluSecond:
        pair_strip_kernel<T, NB, kIluSecond><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    case kIluThird:
        pair_strip_kernel<T, NB, kIluThird><<<p.n_tiles, kRowBlock, 0, stream>>>(p);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template cudaError_t launch_stencil<MK_T, MK_NB>(const RowParams<MK_T> &, int, int, cudaStream_t);
template cudaError_t launch_pair_strip<MK_T, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
template cudaError_t launch_pair_heavy_group<MK_T, MK_NB>(const RowParams<MK_T> &, cudaStream_t);
template cudaError_t launch_pair_heavy<MK_T, MK_NB>(const RowParams<MK_T> &, cudaStream_t);

} // namespace mkb::detail
