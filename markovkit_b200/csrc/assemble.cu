// Explicit CSR assembly of sign * (Q - shift I) on the device (markovkit/generator.hpp:84-107).
//
// The reference assembles column by column from its stored jump lists (one triplet for the
// diagonal, -sign (exit + shift), and one per jump, sign * rate) and sorts the triplets by
// (row, column), summing equal positions (num::spmat::from_triplets). Here each row's entries
// come from the same matrix-free row visit as the gather SpMV: the diagonal, then one entry per
// in-jump. Rows run on the generator's tiles (a thread, a warp or a block per row), in phases:
//   0: count each row's entries;   scan: row offsets;   1: fill (lanes of a shared row write
//   at their exclusive prefix);    a stable sort of each row by column;   a merge of equal
//   columns, summing their values in visit order.
#include "assemble.hpp"
#include "generator_row.cuh"

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <climits>

namespace mkb {
namespace {

struct AssembleParams {
    BinomTable B;
    const SectorDesc *sectors = nullptr;
    const Tile *tiles = nullptr;
    ModelView<double> md;
    std::int64_t n = 0;
    std::int64_t *count = nullptr;         // phase 0: entries of each row
    const std::int64_t *row_ptr = nullptr; // phase 1: where each row's entries start
    std::int64_t *col = nullptr;
    double *val = nullptr;
    double shift = 0.0;
    double sign = 1.0;
    int *bad = nullptr; // set when an in-jump source lies outside [0, n)
};

__device__ __forceinline__ std::int64_t warp_sum_i64(std::int64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    return v;
}

// sum of v over the lanes below this one
__device__ __forceinline__ std::int64_t warp_exclusive(std::int64_t v, int lane) {
    std::int64_t s = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const std::int64_t t = __shfl_up_sync(0xffffffffu, s, off);
        s += lane >= off ? t : 0;
    }
    return s - v;
}

template <int NS, int TMAX>
__global__ void __launch_bounds__(kRowBlock)
    assemble_kernel(const __grid_constant__ AssembleParams p, int phase) {
    __shared__ SectorDesc s_sec;
    __shared__ std::int64_t s_count[kRowBlock / 32];
    __shared__ double s_exit[kRowBlock / 32];
    const Tile tile = p.tiles[blockIdx.x];
    if (threadIdx.x == 0) {
        s_sec = p.sectors[tile.sector];
    }
    __syncthreads();
    const SectorDesc &sec = s_sec;
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;

    std::int64_t local;
    int row_lane, row_lanes;
    if (tile.kind == 0) {
        if (static_cast<int>(threadIdx.x) >= tile.count) {
            return;
        }
        local = tile.local0 + threadIdx.x;
        row_lane = 0;
        row_lanes = 1;
    } else if (tile.kind == 1) {
        if (warp >= tile.count) {
            return;
        }
        local = tile.local0 + warp;
        row_lane = lane;
        row_lanes = 32;
    } else {
        local = tile.local0;
        row_lane = static_cast<int>(threadIdx.x);
        row_lanes = kRowBlock;
    }
    RowState<NS, TMAX> st;
    load_state<NS, TMAX>(p.B, sec, p.md.S, p.md.V, local, st);
    const std::int64_t i = sec.begin + local;
    const bool light = row_lane == 0; // this lane holds the diagonal and the light terms

    double exit = 0.0, leak = 0.0;
    std::int64_t mine = light ? 1 : 0;
    visit_row<double, NS, TMAX>(p.B, p.sectors, sec, p.md, local, st, light, row_lane, row_lanes,
                                exit, leak, [&](int, double, double) { ++mine; });
    // the row's entry count, this lane's offset among the row's lanes, the row's exit rate
    std::int64_t total = mine, before = 0;
    if (tile.kind == 1) {
        before = warp_exclusive(mine, lane);
        total = warp_sum_i64(mine);
        exit = warp_sum_f64(exit);
    } else if (tile.kind == 2) {
        const std::int64_t in_warp = warp_exclusive(mine, lane);
        const std::int64_t warp_total = warp_sum_i64(mine);
        const double warp_exit = warp_sum_f64(exit);
        if (lane == 0) {
            s_count[warp] = warp_total;
            s_exit[warp] = warp_exit;
        }
        __syncthreads();
        std::int64_t base = 0;
        total = 0;
        exit = 0.0;
        for (int w = 0; w < kRowBlock / 32; ++w) {
            base += w < warp ? s_count[w] : 0;
            total += s_count[w];
            exit += s_exit[w];
        }
        before = base + in_warp;
    }
    if (phase == 0) {
        if (light) {
            p.count[i] = total;
        }
        return;
    }
    std::int64_t k = p.row_ptr[i] + before;
    if (light) {
        p.col[k] = i;
        p.val[k] = -p.sign * (exit + p.shift);
        ++k;
    }
    double exit2 = 0.0, leak2 = 0.0;
    visit_row<double, NS, TMAX>(p.B, p.sectors, sec, p.md, local, st, light, row_lane, row_lanes,
                                exit2, leak2, [&](int j, double a, double) {
                                    if (j < 0 || j >= p.n) {
                                        atomicExch(p.bad, 1);
                                    }
                                    p.col[k] = j;
                                    p.val[k] = p.sign * a;
                                    ++k;
                                });
}

// entries of each row after merging equal (sorted) columns
__global__ void unique_count_kernel(const std::int64_t *row_ptr, const std::int64_t *col,
                                    std::int64_t n, std::int64_t *count) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t r = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += stride) {
        std::int64_t c = 0;
        for (std::int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            c += (k == row_ptr[r] || col[k] != col[k - 1]) ? 1 : 0;
        }
        count[r] = c;
    }
}

__global__ void unique_fill_kernel(const std::int64_t *row_ptr, const std::int64_t *col,
                                   const double *val, const std::int64_t *out_ptr,
                                   std::int64_t n, std::int64_t *out_col, double *out_val) {
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t r = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; r < n;
         r += stride) {
        std::int64_t o = out_ptr[r] - 1;
        for (std::int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            if (k == row_ptr[r] || col[k] != col[k - 1]) {
                ++o;
                out_col[o] = col[k];
                out_val[o] = val[k];
            } else {
                out_val[o] += val[k];
            }
        }
    }
}

unsigned grid_for(std::int64_t n) {
    return static_cast<unsigned>(std::max<std::int64_t>(1, std::min<std::int64_t>((n + 255) / 256, 148 * 8)));
}

AssembleParams params_of(const Generator &g) {
    AssembleParams p;
    p.B = g.op.binom->device_view();
    p.sectors = g.op.d_sectors.get();
    p.tiles = g.op.d_tiles.get();
    p.md = g.op.t64.dev;
    p.n = g.op.n;
    return p;
}

void run_phase(const Generator &g, const AssembleParams &p, int phase, cudaStream_t stream) {
    const auto tiles = static_cast<unsigned>(g.op.tiles.size());
    if (tiles == 0) {
        return;
    }
    with_shape(g.op.S, g.op.mol_cap, [&]<int NS, int TMAX>() {
        count_launches(1);
        assemble_kernel<NS, TMAX><<<tiles, kRowBlock, 0, stream>>>(p, phase);
        return 0;
    });
    check_cuda(cudaGetLastError(), "assemble kernel");
}

// out[0..n] = exclusive prefix sums of in[0..n) with in[n] = 0; returns out[n]
std::int64_t offsets(DeviceArray<std::int64_t> &in, std::int64_t n, DeviceArray<std::int64_t> &out,
                     cudaStream_t stream) {
    check_cuda(cudaMemsetAsync(in.get() + n, 0, sizeof(std::int64_t), stream), "scan tail");
    out.resize(static_cast<std::size_t>(n + 1));
    std::size_t bytes = 0;
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in.get(), out.get(), n + 1, stream),
               "scan size");
    DeviceArray<char> tmp(std::max<std::size_t>(bytes, 1));
    check_cuda(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in.get(), out.get(), n + 1, stream),
               "scan");
    std::int64_t total = 0;
    check_cuda(cudaMemcpyAsync(&total, out.get() + n, sizeof total, cudaMemcpyDeviceToHost, stream),
               "scan total");
    check_cuda(cudaStreamSynchronize(stream), "scan sync");
    return total;
}

} // namespace

std::int64_t count_jumps(const Generator &g, cudaStream_t stream) {
    const std::int64_t n = g.op.n;
    DeviceArray<std::int64_t> count(static_cast<std::size_t>(n + 1)), ptr;
    AssembleParams p = params_of(g);
    p.count = count.get();
    run_phase(g, p, 0, stream);
    return offsets(count, n, ptr, stream) - n; // every row also holds its diagonal
}

void assemble(const Generator &g, double shift, double sign, Csr &out, cudaStream_t stream) {
    const std::int64_t n = g.op.n;
    out.rows = n;
    DeviceArray<std::int64_t> count(static_cast<std::size_t>(n + 1)), raw_ptr;
    DeviceArray<int> bad(1);
    check_cuda(cudaMemsetAsync(bad.get(), 0, sizeof(int), stream), "assemble flag");
    AssembleParams p = params_of(g);
    p.count = count.get();
    p.bad = bad.get();
    p.shift = shift;
    p.sign = sign;
    run_phase(g, p, 0, stream);
    const std::int64_t raw = offsets(count, n, raw_ptr, stream);
    if (raw > INT_MAX || n > INT_MAX) {
        throw Error(kEOverflow, "assembled generator: more than 2^31 - 1 entries or rows");
    }
    DeviceArray<std::int64_t> col(static_cast<std::size_t>(raw)), col_sorted(static_cast<std::size_t>(raw));
    DeviceArray<double> val(static_cast<std::size_t>(raw)), val_sorted(static_cast<std::size_t>(raw));
    p.row_ptr = raw_ptr.get();
    p.col = col.get();
    p.val = val.get();
    run_phase(g, p, 1, stream);
    int flag = 0;
    check_cuda(cudaMemcpyAsync(&flag, bad.get(), sizeof flag, cudaMemcpyDeviceToHost, stream),
               "assemble flag");
    check_cuda(cudaStreamSynchronize(stream), "assemble sync");
    if (flag) {
        throw Error(kEInval, "assembled generator: an in-jump source lies outside the space");
    }
    // each row by column, equal columns kept in visit order
    if (raw > 0) {
        std::size_t bytes = 0;
        check_cuda(cub::DeviceSegmentedSort::StableSortPairs(
                       nullptr, bytes, col.get(), col_sorted.get(), val.get(), val_sorted.get(),
                       static_cast<int>(raw), static_cast<int>(n), raw_ptr.get(), raw_ptr.get() + 1,
                       stream),
                   "row sort size");
        DeviceArray<char> tmp(std::max<std::size_t>(bytes, 1));
        check_cuda(cub::DeviceSegmentedSort::StableSortPairs(
                       tmp.get(), bytes, col.get(), col_sorted.get(), val.get(), val_sorted.get(),
                       static_cast<int>(raw), static_cast<int>(n), raw_ptr.get(), raw_ptr.get() + 1,
                       stream),
                   "row sort");
    }
    // merge equal columns
    DeviceArray<std::int64_t> ucount(static_cast<std::size_t>(n + 1));
    if (n > 0) {
        count_launches(1);
        unique_count_kernel<<<grid_for(n), 256, 0, stream>>>(raw_ptr.get(), col_sorted.get(), n,
                                                             ucount.get());
        check_cuda(cudaGetLastError(), "merge count");
    }
    out.nnz = offsets(ucount, n, out.row_ptr, stream);
    out.col.resize(static_cast<std::size_t>(out.nnz));
    out.val.resize(static_cast<std::size_t>(out.nnz));
    if (n > 0) {
        count_launches(1);
        unique_fill_kernel<<<grid_for(n), 256, 0, stream>>>(raw_ptr.get(), col_sorted.get(),
                                                            val_sorted.get(), out.row_ptr.get(), n,
                                                            out.col.get(), out.val.get());
        check_cuda(cudaGetLastError(), "merge fill");
    }
    check_cuda(cudaStreamSynchronize(stream), "assemble sync");
}

} // namespace mkb
