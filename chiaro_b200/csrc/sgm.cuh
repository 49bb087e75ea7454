// sgm.cuh — semi_global_costs (crates/chiaro-fusion/src/depth.rs:1279-1383).
//
// Eight-path SGM over the label-minor f32 volume. The reference adds the eight path costs into one output in a
// fixed order per node: rows forward, rows reverse, columns forward, columns
// reverse, down-right forward/reverse, down-left forward/reverse
// (depth.rs:1287-1309). Float addition is not associative, so the passes keep
// that order exactly (see the schedule below), which keeps the sum bit-identical.
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

// One launch per direction, in the reference's order, so each node receives
// 0 + L1, then + L2, ..., + L8 exactly as depth.rs:1287-1309 adds them.
//
// A path is walked by K warps, one per 32-label chunk (K = ceil(labels / 32)),
// so each warp handles one label per lane per step. Per step, each warp takes
// its chunk's minimum with redux.sync.min.f32, publishes it together with its
// first and last label values in shared memory, and after the path's named
// barrier reads the other chunks' minima (min is exact, so the combination
// order does not matter) and its neighbours across the chunk boundary. The
// exchange buffers alternate between steps, so one barrier per step suffices.
// Each warp prefetches its chunk of the cost and output vectors P steps ahead.
constexpr int SGM_PREFETCH = 8;

__device__ __forceinline__ float warp_min_f32(float v) {
    float r;
    asm volatile("redux.sync.min.f32 %0, %1, %2;" : "=f"(r) : "f"(v), "r"(0xffffffffu));
    return r;
}

__device__ __forceinline__ void path_barrier(int threads) {
    asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

// One direction of one family: every block walks one path, forward or in
// reverse, adding its costs to `out` (`first` stores 0 + L).
template <int K>
__global__ void __launch_bounds__(32 * K, 4) sgm_direction_kernel(const float *__restrict__ data,
                                                                 const float *__restrict__ guidance, float *out,
                                                                 int columns, int rows, int labels, int family,
                                                                 int first, int reverse) {
    __shared__ float xmin[2][K], xfirst[2][K], xlast[2][K];
    const int lane = threadIdx.x & 31;
    const int chunk = threadIdx.x >> 5;
    int r0, c0, dr, dc, len;
    sgm_path(family, blockIdx.x, columns, rows, r0, c0, dr, dc, len);
    if (reverse) {
        r0 += dr * (len - 1);
        c0 += dc * (len - 1);
        dr = -dr;
        dc = -dc;
    }
    constexpr int P = SGM_PREFETCH;
    const int l = chunk * 32 + lane;
    const bool valid = l < labels;
    const bool fold = !first;  // out = first ? 0 + L : out + L
    const long node_step = (long)dr * columns + dc;
    const long stride = node_step * labels;
    const int node0 = r0 * columns + c0;
    const size_t e0 = (size_t)node0 * labels + l;
    const float *dp = data + e0;
    float *wp = out + e0;
    const float *op = out + e0;
    const float *gp = guidance + node0;
    float prev;
    {
        float c = valid ? __ldg(dp) : 0.0f;
        float b = valid && fold ? __ldcg(op) : 0.0f;
        prev = valid ? c : INFINITY;
        if (valid) *wp = fold ? b + c : 0.0f + c;
    }
    float g_prev = __ldg(gp);
    float ring_c[P], ring_o[P], ring_g[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        if (1 + j < len) {
            ring_c[j] = valid ? __ldg(dp + (1 + j) * stride) : 0.0f;
            ring_o[j] = valid && fold ? __ldcg(op + (1 + j) * stride) : 0.0f;
            ring_g[j] = __ldg(gp + (1 + j) * node_step);
        }
    }
    int parity = 0;
    for (int base = 1; base < len; base += P) {
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const int step = base + j;
            if (step >= len) break;  // uniform across the path's warps
            wp += stride;
            const float cur_data = ring_c[j], cur_base = ring_o[j], g = ring_g[j];
            if (step + P < len) {
                ring_c[j] = valid ? __ldg(dp + (step + P) * stride) : 0.0f;
                ring_o[j] = valid && fold ? __ldcg(op + (step + P) * stride) : 0.0f;
                ring_g[j] = __ldg(gp + (step + P) * node_step);
            }
            // publish this chunk's minimum and boundary labels, then combine
            const float chunk_min = warp_min_f32(prev);
            if (lane == 0) {
                xmin[parity][chunk] = chunk_min;
                xfirst[parity][chunk] = prev;
            }
            if (lane == 31) xlast[parity][chunk] = prev;
            const float rot_up = __shfl_sync(0xffffffffu, prev, (lane + 31) & 31);
            const float rot_down = __shfl_sync(0xffffffffu, prev, (lane + 1) & 31);
            const float edge = fabsf(g - g_prev);
            g_prev = g;
            const float edge_scale = __frcp_rn(1.0f + 4.0f * edge);  // == 1 / x, correctly rounded
            const float p1 = SGM_SMALL_PENALTY * fmaxf(edge_scale, 0.35f);
            const float p2 = SGM_LARGE_PENALTY * fmaxf(edge_scale, 0.12f);
            if (K > 1) path_barrier(32 * K);
            float minimum_previous = K > 1 ? xmin[parity][0] : chunk_min;
#pragma unroll
            for (int k = 1; k < K; ++k) minimum_previous = fminf(minimum_previous, xmin[parity][k]);
            float below = rot_up, above = rot_down;
            if (lane == 0) below = chunk > 0 ? xlast[parity][chunk > 0 ? chunk - 1 : 0] : INFINITY;
            if (lane == 31) above = chunk + 1 < K ? xfirst[parity][chunk + 1 < K ? chunk + 1 : chunk] : INFINITY;
            parity ^= 1;
            const float jump = minimum_previous + p2;
            const float lower = below + p1;  // INFINITY + p1 = INFINITY
            const float higher = l + 1 < labels ? above + p1 : INFINITY;
            const float v = cur_data + fminf(fminf(fminf(prev, lower), higher), jump) - minimum_previous;
            prev = valid ? v : INFINITY;
            if (valid) *wp = fold ? cur_base + v : 0.0f + v;
        }
    }
}

}  // namespace chiaro
