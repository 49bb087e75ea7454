// sgm_band.cuh — band-limited semi_global_costs (crates/chiaro-fusion/src/depth.rs:1279-1383)
// with a windowed full-range fallback. The reference has no such mode; it is the
// banded SGM of the learned-band design, checked label for label against the
// oracle's restatement (oracle_sgm_banded).
//
// Every node aggregates only the `band` (<= 32) labels [O, O + band) of its
// tile's offset O: one label per lane, so a path is one warp with one register
// per label instead of ceil(D / 32). Along a path the band may shift between
// tiles by delta = O - O_prev: the previous value of label l is the previous
// lane l - O_prev, fetched by a shuffle from lane j + delta (+inf outside the
// previous band), and the recurrence is otherwise that of accumulate_path
// (depth.rs:1363-1381) in its order. Lane j computes the offset and the
// penalties of step base + j once per 32 steps; the step reads them by shuffle.
// The 8 directions run at once into their own path buffers and one kernel adds
// them in the reference's order and picks the first minimum over the band; a
// tile whose winner sits on a band edge is flagged for the fallback, which runs
// the full-range SGM (the batched SGM) on a window around each rectangle of
// fallback tiles and takes the window's winners for the rectangle's nodes.
#pragma once

#include "sgm.cuh"

namespace chiaro {

constexpr long long KEY64_NONE = 0x7fffffffffffffffLL;

struct BandGrid {
    const int *tile_offset;  // [tiles_y][tiles_x], 1 <= O <= D - band
    int tile, tiles_x, band;
};

__device__ __forceinline__ int band_offset_at(const BandGrid &b, int row, int column) {
    return __ldg(b.tile_offset + (row / b.tile) * b.tiles_x + column / b.tile);
}

// Banded path costs of every path of every direction; pass k writes paths + k * pitch ([N][band]).
// Each step loads its own costs: the kernel stays small enough (registers) for all paths of
// a full-resolution grid to be resident at once, and the other warps hide the load.
// Cost rows are either full ([N][labels]: label l at l) or the banded cost volume's
// compact rows ([N][1 + band]: label 0, then the node's band in order; compact != 0).
__global__ void __launch_bounds__(32 * SGM_PATHS_PER_CTA) sgm_band_paths_kernel(
    const float *__restrict__ data, const float *__restrict__ guidance, BandGrid grid, float *__restrict__ paths,
    size_t pitch, int columns, int rows, int labels, int compact) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp_path = blockIdx.x * SGM_PATHS_PER_CTA + (threadIdx.x >> 5);
    if (warp_path >= (int)sgm_total_paths(columns, rows)) return;  // whole warp
    int pass, path;
    sgm_path_of(warp_path, columns, rows, pass, path);
    int r0, c0, dr, dc, len;
    sgm_path(pass >> 1, path, columns, rows, r0, c0, dr, dc, len);
    if (pass & 1) {
        r0 += dr * (len - 1);
        c0 += dc * (len - 1);
        dr = -dr;
        dc = -dc;
    }
    const int band = grid.band;
    const bool valid = lane < band;
    const long node_step = (long)dr * columns + dc;
    const long node0 = (long)r0 * columns + c0;
    float *wp = paths + (size_t)pass * pitch + (size_t)node0 * band + lane;
    int offset = band_offset_at(grid, r0, c0);
    const int stride = compact ? 1 + band : labels;
    float prev = valid ? __ldg(data + (size_t)node0 * stride + (compact ? 1 : offset) + lane) : INFINITY;
    if (valid) *wp = prev;
    float p1s = 0.0f, p2s = 0.0f;
    int offsets = 0;
    for (int base = 1; base < len; base += 32) {
        {  // lane j: offset and penalties of step base + j (depth.rs:1358-1361)
            const int s = base + lane;
            if (s < len) {
                const float g = __ldg(guidance + node0 + s * node_step);
                const float g_prev = __ldg(guidance + node0 + (s - 1) * node_step);
                const float edge_scale = __frcp_rn(1.0f + 4.0f * fabsf(g - g_prev));  // == 1 / x, correctly rounded
                p1s = SGM_SMALL_PENALTY * fmaxf(edge_scale, 0.35f);
                p2s = SGM_LARGE_PENALTY * fmaxf(edge_scale, 0.12f);
                offsets = band_offset_at(grid, r0 + s * dr, c0 + s * dc);
            }
        }
        const int steps = min(32, len - base);
        for (int j = 0; j < steps; ++j) {
            const long node = node0 + (long)(base + j) * node_step;
            const int o = __shfl_sync(full, offsets, j);
            const float p1 = __shfl_sync(full, p1s, j), p2 = __shfl_sync(full, p2s, j);
            const float cur = valid ? __ldg(data + (size_t)node * stride + (compact ? 1 : o) + lane) : INFINITY;
            const float minimum_previous = warp_min_f32(prev);
            const int s = lane + (o - offset);  // this label's slot in the previous band
            const float same = __shfl_sync(full, prev, s & 31);
            const float below = __shfl_sync(full, prev, (s - 1) & 31);
            const float above = __shfl_sync(full, prev, (s + 1) & 31);
            const int label = o + lane;
            const float same_v = s >= 0 && s < band ? same : INFINITY;
            const float lower = label > 0 && s - 1 >= 0 && s - 1 < band ? below + p1 : INFINITY;
            const float higher = label + 1 < labels && s + 1 >= 0 && s + 1 < band ? above + p1 : INFINITY;
            const float jump = minimum_previous + p2;
            const float v = cur + fminf(fminf(fminf(same_v, lower), higher), jump) - minimum_previous;
            prev = valid ? v : INFINITY;
            offset = o;
            if (valid) paths[(size_t)pass * pitch + (size_t)node * band + lane] = v;
        }
    }
}

// ((0 + L1) + L2) + ... + L8 per (node, slot), the first minimum over the band, and the
// fallback flag of a tile whose winner is on a band edge with labels beyond it (an
// edge at label 1 or D - 1 is the label range's own end). A warp per node.
__global__ void __launch_bounds__(256) sgm_band_select_kernel(const float *__restrict__ paths, size_t pitch,
                                                              BandGrid grid, int columns, int rows, int labels,
                                                              int *winner, uint8_t *fallback) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (node >= columns * rows) return;  // whole warp
    const int band = grid.band;
    float s = 0.0f;
    if (lane < band) {
#pragma unroll
        for (int k = 0; k < 8; ++k) s = s + __ldcs(paths + k * pitch + (size_t)node * band + lane);
    }
    // (total-order key, slot): the first minimum
    const long long key = lane < band ? (long long)total_key(s) * 256 + lane : KEY64_NONE;
    long long best = key;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const long long other = __shfl_xor_sync(full, best, off);
        best = other < best ? other : best;
    }
    if (lane == 0) {
        const int row = node / columns, column = node - row * columns;
        const int slot = (int)(best & 0xff);
        const int offset = band_offset_at(grid, row, column);
        winner[node] = offset + slot;  // the key's low 8 bits
        if ((slot == 0 && offset > 1) || (slot == band - 1 && offset + band < labels))
            fallback[(row / grid.tile) * grid.tiles_x + column / grid.tile] = 1;
    }
}

// Flags an offset outside [1, labels - band] (the banded loads would leave the node's labels).
__global__ void band_check_kernel(const int *__restrict__ tile_offset, int tiles, int labels, int band, int *bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < tiles; i += gridDim.x * blockDim.x) {
        const int o = tile_offset[i];
        if (o < 1 || o + band > labels) atomicExch(bad, 1);
    }
}

// A fallback window: a rectangle of fallback tiles' nodes and the window around it
// in the full grid.
struct BandWindow {
    int c0, r0, wc, wr;   // window origin and size (nodes)
    int tc0, tr0, tc, tr;  // the rectangle's nodes
    size_t cost_offset;    // into the window cost / aggregate scratch ([wc * wr][D])
    size_t node_offset;    // into the window guidance scratch ([wc * wr])
};

// Copy every window's costs and guidance out of the full grid. Grid-stride over
// (window, cell) with one block row per window.
__global__ void band_crop_kernel(const float *__restrict__ costs, const float *__restrict__ guidance, int columns,
                                 int labels, const BandWindow *__restrict__ windows, float *__restrict__ wcosts,
                                 float *__restrict__ wguidance) {
    const BandWindow w = windows[blockIdx.y];
    const long cells = (long)w.wc * w.wr * labels;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += (long)gridDim.x * blockDim.x) {
        const long n = i / labels;
        const int l = (int)(i - n * labels);
        const int r = (int)(n / w.wc), c = (int)(n - (long)r * w.wc);
        const size_t src = (size_t)(w.r0 + r) * columns + (w.c0 + c);
        wcosts[w.cost_offset + i] = costs[src * labels + l];
        if (l == 0) wguidance[w.node_offset + n] = guidance[src];
    }
}

// The window's winner (labels 1..D-1, first minimum) for each node of its rectangle
// whose tile fell back (all of a rectangle's tiles, unless the window is the whole
// grid). A warp per node.
__global__ void band_window_winner_kernel(const float *__restrict__ aggregates, int columns, int labels,
                                          const BandWindow *__restrict__ windows, BandGrid grid,
                                          const uint8_t *__restrict__ fallback, int *winner) {
    const unsigned full = 0xffffffffu;
    const BandWindow w = windows[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= w.tc * w.tr) return;  // whole warp
    const int r = w.tr0 + k / w.tc, c = w.tc0 + k % w.tc;
    if (!fallback[(r / grid.tile) * grid.tiles_x + c / grid.tile]) return;  // whole warp
    const float *agg = aggregates + w.cost_offset + ((size_t)(r - w.r0) * w.wc + (c - w.c0)) * labels;
    long long best = KEY64_NONE;
    for (int l = 1 + lane; l < labels; l += 32) {
        const long long key = (long long)total_key(agg[l]) * 65536 + l;
        best = key < best ? key : best;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const long long other = __shfl_xor_sync(full, best, off);
        best = other < best ? other : best;
    }
    if (lane == 0) winner[(size_t)r * columns + c] = (int)(best & 0xffff);
}

}  // namespace chiaro
