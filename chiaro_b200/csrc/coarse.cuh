// coarse.cuh — the coarse depth search of the stage as its own operator: the cost
// volume (build_cost_volume, crates/chiaro-fusion/src/depth.rs:1187-1277), the SGM
// (semi_global_costs, depth.rs:1279-1383) and each node's winning label over the
// finite labels (the first minimum, as select_depths takes it, depth.rs:1406-1413).
//
// Besides the plain form, the learned-band form replaces the full-range search. The
// reference has no such mode; these are the design's kernels around it:
//   * a pre-pass scores label 0 and 16 sampled labels at every node (cost.cuh's
//     label-list mode); the band proposal reads those costs;
//   * the banded cost volume scores label 0 and each tile's band (band mode);
//   * the banded SGM (sgm_band.cuh) reads the banded rows;
//   * a tile falls back to the full range when its winner sits on a band edge, or
//     when its winners fail the cross-view check: a node is contradicted where the
//     views' aggregated score at its winner is more than 0.12 below their score under
//     the global warp (label 0), the threshold of the reference's per-target decision
//     (depth.rs:458-485); a tile falls back when more than a set fraction of its tested
//     nodes are contradicted;
//   * the fallback windows' full-range costs come from the cost kernel's node-list
//     mode and their SGMs from the batched SGM.
#pragma once

#include "bandnet.cuh"
#include "sgm_band.cuh"

namespace chiaro {

// The winner over labels 1..D-1 of an aggregate row (first minimum in total order, as
// min_by(total_cmp) keeps it). A warp per node.
__global__ void __launch_bounds__(256) aggregate_winner_kernel(const float *__restrict__ aggregate, int nodes,
                                                               int labels, int *__restrict__ winner) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int node = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (node >= nodes) return;  // whole warp
    const float *row = aggregate + (size_t)node * labels;
    long long best = KEY64_NONE;
    for (int l = 1 + lane; l < labels; l += 32) {
        const long long key = (long long)total_key(__ldcs(row + l)) * 65536 + l;
        best = key < best ? key : best;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const long long other = __shfl_xor_sync(full, best, off);
        best = other < best ? other : best;
    }
    if (lane == 0) winner[node] = labels > 1 ? (int)(best & 0xffff) : 0;
}

// The pre-pass's label list: label 0, then the 16 sampled labels (net_sample_label).
constexpr int PREPASS_SLOTS = 1 + NET_BINS;

// The band without learning: per tile, the median over its nodes of the first sampled
// label holding the node's lowest pre-pass cost, the band centred there (clamped to
// [1, labels - band]). A thread per tile; tiles of at most 8 x 8 nodes.
constexpr int NAIVE_MAX_TILE = 8;

__global__ void naive_band_offsets_kernel(const float *__restrict__ prepass, int columns, int rows, int labels,
                                          int tile, int band, int *__restrict__ offsets) {
    const int tiles_x = (columns + tile - 1) / tile, tiles_y = (rows + tile - 1) / tile;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles_x * tiles_y) return;
    const int tx = t % tiles_x, ty = t / tiles_x;
    int values[NAIVE_MAX_TILE * NAIVE_MAX_TILE];
    int n = 0;
    for (int r = ty * tile; r < min(rows, (ty + 1) * tile); ++r)
        for (int c = tx * tile; c < min(columns, (tx + 1) * tile); ++c) {
            const float *row = prepass + ((size_t)r * columns + c) * PREPASS_SLOTS;
            float lowest = INFINITY;
            int label = 1;
            for (int b = 0; b < NET_BINS; ++b) {
                const float v = row[1 + b];
                if (v < lowest) {
                    lowest = v;
                    label = net_sample_label(b, labels);
                }
            }
            int i = n++;  // insertion sort: at most 64 values
            while (i > 0 && values[i - 1] > label) {
                values[i] = values[i - 1];
                --i;
            }
            values[i] = label;
        }
    const float median = (n & 1) ? (float)values[n / 2] : 0.5f * (float)(values[n / 2 - 1] + values[n / 2]);
    const int o = (int)rintf(median) - band / 2;
    offsets[t] = max(1, min(labels - band, o));
}

// The cross-view check of the banded winners, per tile (a thread per tile): counts its
// tested nodes and those whose aggregated score at the winner is more than 0.12 below
// the score under the global warp; flags the tile (consistency[t], and fallback[t])
// when contradicted > fraction * tested.
__global__ void band_consistency_kernel(const float *__restrict__ band_scores, const uint8_t *__restrict__ tested,
                                        const int *__restrict__ winner, BandGrid grid, int columns, int rows,
                                        float fraction, uint8_t *__restrict__ consistency,
                                        uint8_t *__restrict__ fallback) {
    const int tiles_y = (rows + grid.tile - 1) / grid.tile;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= grid.tiles_x * tiles_y) return;
    const int tx = t % grid.tiles_x, ty = t / grid.tiles_x;
    const int offset = grid.tile_offset[t];
    int n_tested = 0, contradicted = 0;
    for (int r = ty * grid.tile; r < min(rows, (ty + 1) * grid.tile); ++r)
        for (int c = tx * grid.tile; c < min(columns, (tx + 1) * grid.tile); ++c) {
            const int node = r * columns + c;
            if (!tested[node]) continue;
            ++n_tested;
            const float *row = band_scores + (size_t)node * (1 + grid.band);
            const float at_winner = row[1 + winner[node] - offset], at_global = row[0];
            contradicted += isfinite(at_winner) && isfinite(at_global) && at_winner + 0.12f < at_global;
        }
    const bool flag = (float)contradicted > fraction * (float)n_tested;
    consistency[t] = flag;
    if (flag) fallback[t] = 1;
}

}  // namespace chiaro
