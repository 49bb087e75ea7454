// sgm.cuh — semi_global_costs (crates/chiaro-fusion/src/depth.rs:1279-1383).
//
// Eight-path SGM over the label-minor f32 volume. One warp walks one path; a
// lane holds labels lane, lane+32, ... in registers, the previous node's
// minimum comes from a warp-shuffle min, and label +-1 neighbours from
// shuffles. The reference adds the eight path costs into one output in a
// fixed order per node: rows forward, rows reverse, columns forward, columns
// reverse, down-right forward/reverse, down-left forward/reverse
// (depth.rs:1287-1309). Float addition is not associative, so the launches
// follow that order: each direction is one launch that adds its path costs to
// the output (the first one stores 0 + L), which keeps the sum bit-identical.
#pragma once

#include "common.cuh"

namespace chiaro {

enum SgmFamily { SGM_ROWS = 0, SGM_COLUMNS = 1, SGM_DOWN_RIGHT = 2, SGM_DOWN_LEFT = 3 };

__host__ __device__ inline int sgm_path_count(int family, int columns, int rows) {
    switch (family) {
        case SGM_ROWS: return rows;
        case SGM_COLUMNS: return columns;
        default: return columns + rows - 1;
    }
}

// Path p of a family in the reference's enumeration (depth.rs:1287-1338):
// start node, step and length of its forward direction.
__device__ inline void sgm_path(int family, int p, int columns, int rows, int &r0, int &c0, int &dr, int &dc,
                                int &len) {
    switch (family) {
        case SGM_ROWS: r0 = p; c0 = 0; dr = 0; dc = 1; len = columns; return;
        case SGM_COLUMNS: r0 = 0; c0 = p; dr = 1; dc = 0; len = rows; return;
        case SGM_DOWN_RIGHT:
            dr = 1; dc = 1;
            if (p < columns) { r0 = 0; c0 = p; len = min(columns - p, rows); }
            else { r0 = p - columns + 1; c0 = 0; len = min(rows - r0, columns); }
            return;
        default:
            dr = 1; dc = -1;
            if (p < columns) { r0 = 0; c0 = p; len = min(p + 1, rows); }
            else { r0 = p - columns + 1; c0 = columns - 1; len = min(rows - r0, columns); }
            return;
    }
}

// accumulate_path for every path of one family and direction.
// accumulate == 0: out = 0 + L (first direction); otherwise out += L.
template <int K>
__global__ void __launch_bounds__(256) sgm_direction_kernel(const float *__restrict__ data,
                                                            const float *__restrict__ guidance, float *out,
                                                            int columns, int rows, int labels, int family,
                                                            int reverse, int accumulate) {
    const int lane = threadIdx.x & 31;
    const int path = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (path >= sgm_path_count(family, columns, rows)) return;
    int r0, c0, dr, dc, len;
    sgm_path(family, path, columns, rows, r0, c0, dr, dc, len);
    if (reverse) {
        r0 += dr * (len - 1);
        c0 += dc * (len - 1);
        dr = -dr;
        dc = -dc;
    }
    const unsigned full = 0xffffffffu;
    float prev[K];
    int node = r0 * columns + c0;
    // first node: L = C
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int l = lane + 32 * k;
        prev[k] = l < labels ? __ldg(data + (size_t)node * labels + l) : INFINITY;
        if (l < labels) {
            float *o = out + (size_t)node * labels + l;
            *o = accumulate ? *o + prev[k] : 0.0f + prev[k];
        }
    }
    float g_prev = __ldg(guidance + node);
    int r = r0, c = c0;
    for (int i = 1; i < len; ++i) {
        r += dr;
        c += dc;
        node = r * columns + c;
        float cur_data[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int l = lane + 32 * k;
            cur_data[k] = l < labels ? __ldg(data + (size_t)node * labels + l) : 0.0f;
        }
        float g = __ldg(guidance + node);
        float edge = fabsf(g - g_prev);
        g_prev = g;
        float edge_scale = 1.0f / (1.0f + 4.0f * edge);
        float p1 = SGM_SMALL_PENALTY * fmaxf(edge_scale, 0.35f);
        float p2 = SGM_LARGE_PENALTY * fmaxf(edge_scale, 0.12f);
        float m = prev[0];
#pragma unroll
        for (int k = 1; k < K; ++k) m = fminf(m, prev[k]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) m = fminf(m, __shfl_xor_sync(full, m, off));
        const float minimum_previous = m;
        const float jump = minimum_previous + p2;
        float cur[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int l = lane + 32 * k;
            float below = __shfl_up_sync(full, prev[k], 1);
            float above = __shfl_down_sync(full, prev[k], 1);
            float wrap_below = k > 0 ? __shfl_sync(full, prev[k > 0 ? k - 1 : 0], 31) : INFINITY;
            float wrap_above = k + 1 < K ? __shfl_sync(full, prev[k + 1 < K ? k + 1 : k], 0) : INFINITY;
            if (lane == 0) below = wrap_below;
            if (lane == 31) above = wrap_above;
            float lower = l > 0 ? below + p1 : INFINITY;
            float higher = l + 1 < labels ? above + p1 : INFINITY;
            float v = cur_data[k] + fminf(fminf(fminf(prev[k], lower), higher), jump) - minimum_previous;
            cur[k] = l < labels ? v : INFINITY;
            if (l < labels) {
                float *o = out + (size_t)node * labels + l;
                *o = accumulate ? *o + v : 0.0f + v;
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) prev[k] = cur[k];
    }
}

}  // namespace chiaro
