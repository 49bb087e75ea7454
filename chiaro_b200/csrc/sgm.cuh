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
// The cost vector and (when accumulating) the output vector of the node PREFETCH
// steps ahead are loaded into a register ring, so memory latency stays off the
// recurrence's critical path (the warp-shuffle minimum and a few adds).
template <int K>
struct SgmPrefetch {  // ring depth that keeps the ring in registers without spills
    static constexpr int value = K <= 4 ? 8 : (K <= 6 ? 6 : 3);
};
constexpr int SGM_THREADS = 64;  // two paths per CTA: spread few long paths over all SMs

template <int K>
__device__ __forceinline__ void sgm_load(const float *__restrict__ data, const float *out, int node, int labels,
                                         int lane, bool accumulate, float (&c)[K], float (&o)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
        int l = lane + 32 * k;
        bool in = l < labels;
        c[k] = in ? __ldg(data + (size_t)node * labels + l) : 0.0f;
        o[k] = (in && accumulate) ? __ldcg(out + (size_t)node * labels + l) : 0.0f;
    }
}

template <int K>
__global__ void __launch_bounds__(SGM_THREADS) sgm_direction_kernel(const float *__restrict__ data,
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
    const int dstep = dr * columns + dc;  // node index increment along the path
    const unsigned full = 0xffffffffu;
    const bool acc = accumulate != 0;
    constexpr int SGM_PREFETCH = SgmPrefetch<K>::value;
    float prev[K];
    int node = r0 * columns + c0;
    {
        float c[K], o[K];
        sgm_load<K>(data, out, node, labels, lane, acc, c, o);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int l = lane + 32 * k;
            prev[k] = l < labels ? c[k] : INFINITY;
            if (l < labels) out[(size_t)node * labels + l] = acc ? o[k] + c[k] : 0.0f + c[k];
        }
    }
    float g_prev = __ldg(guidance + node);
    // register ring of the next PREFETCH nodes
    float ring_c[SGM_PREFETCH][K], ring_o[SGM_PREFETCH][K], ring_g[SGM_PREFETCH];
#pragma unroll
    for (int j = 0; j < SGM_PREFETCH; ++j) {
        int step = 1 + j;
        if (step < len) {
            int nj = node + step * dstep;
            sgm_load<K>(data, out, nj, labels, lane, acc, ring_c[j], ring_o[j]);
            ring_g[j] = __ldg(guidance + nj);
        }
    }
    for (int base = 1; base < len; base += SGM_PREFETCH) {
#pragma unroll
        for (int j = 0; j < SGM_PREFETCH; ++j) {
            const int step = base + j;
            if (step >= len) break;  // warp-uniform
            const int nd = node + step * dstep;
            float cur_data[K], cur_out[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                cur_data[k] = ring_c[j][k];
                cur_out[k] = ring_o[j][k];
            }
            const float g = ring_g[j];
            if (step + SGM_PREFETCH < len) {
                int nn = node + (step + SGM_PREFETCH) * dstep;
                sgm_load<K>(data, out, nn, labels, lane, acc, ring_c[j], ring_o[j]);
                ring_g[j] = __ldg(guidance + nn);
            }
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
                if (l < labels) out[(size_t)nd * labels + l] = acc ? cur_out[k] + v : 0.0f + v;
            }
#pragma unroll
            for (int k = 0; k < K; ++k) prev[k] = cur[k];
        }
    }
}

}  // namespace chiaro
