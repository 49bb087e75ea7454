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
__host__ __device__ inline void sgm_path(int family, int p, int columns, int rows, int &r0, int &c0, int &dr, int &dc,
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

// All eight directions run in one launch, each path writing its own path
// costs L_k into buffer k; a second kernel then forms, per cell,
// ((0 + L1) + L2) + ... + L8 in the reference's order (depth.rs:1287-1309), so
// the sum is bit-identical to the reference's in-place accumulation while the
// GPU walks every path of every direction at once.
//
// A path is walked by one warp. Lane i holds labels i, i + 32, ..., i + 32 (K - 1)
// (K = ceil(labels / 32) sets), so the step's minimum is a local min and one
// redux.sync.min.f32, and the label neighbours come from two shuffles per set:
// the neighbour below lane 0 of set k is lane 31 of set k - 1, the one above
// lane 31 of set k is lane 0 of set k + 1. No shared memory and no barrier sit
// on the step's critical path. The penalties p1, p2 depend only on the guidance
// along the path: lane j computes those of step base + j once per 32 steps and
// each step reads them by shuffle. Labels past the last one carry +inf data,
// which keeps them at +inf without a select. The data is prefetched P steps
// ahead.
constexpr int SGM_PREFETCH = 4;
constexpr int SGM_PATHS_PER_CTA = 4;

__device__ __forceinline__ float warp_min_f32(float v) {
    float r;
    asm volatile("redux.sync.min.f32 %0, %1, %2;" : "=f"(r) : "f"(v), "r"(0xffffffffu));
    return r;
}

// Paths of the launch: for each family (rows, columns, down-right, down-left)
// its forward paths, then its reverse paths. Pass = 2 * family + reverse is
// the reference's summation order.
__host__ __device__ inline unsigned sgm_total_paths(int columns, int rows) {
    return 2u * (unsigned)(rows + columns + 2 * (columns + rows - 1));
}

__host__ __device__ inline void sgm_path_of(int b, int columns, int rows, int &pass, int &path) {
    for (int family = 0; family < 4; ++family) {
        const int n = sgm_path_count(family, columns, rows);
        if (b < 2 * n) {
            pass = 2 * family + (b >= n ? 1 : 0);
            path = b >= n ? b - n : b;
            return;
        }
        b -= 2 * n;
    }
    pass = 0;
    path = 0;
}

// Path `warp_path` of the launch's enumeration (sgm_path_of), walked by the
// calling warp; pass k writes paths + k * pitch. P: steps of data prefetched ahead.
template <int K, int P = SGM_PREFETCH>
__device__ __forceinline__ void sgm_walk_path(const float *__restrict__ data, const float *__restrict__ guidance,
                                              float *__restrict__ paths, size_t pitch, int columns, int rows,
                                              int labels, int warp_path) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
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
    bool valid[K];
#pragma unroll
    for (int k = 0; k < K; ++k) valid[k] = lane + 32 * k < labels;
    const long node_step = (long)dr * columns + dc;
    const long stride = node_step * labels;
    const int node0 = r0 * columns + c0;
    const size_t e0 = (size_t)node0 * labels + lane;
    const float *pf = data + e0;                      // data of step + P (after the ring fill)
    float *wp = paths + (size_t)pass * pitch + e0;    // path costs of the current step
    const float *gp = guidance + node0;
    float prev[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        prev[k] = valid[k] ? __ldg(pf + 32 * k) : INFINITY;
        if (valid[k]) wp[32 * k] = prev[k];
    }
    float ring[P][K];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        pf += stride;
#pragma unroll
        for (int k = 0; k < K; ++k) ring[j][k] = valid[k] && 1 + j < len ? __ldg(pf + 32 * k) : INFINITY;
    }
    float p1s = 0.0f, p2s = 0.0f;
    for (int base = 1; base < len; base += 32) {
        {  // lane j: penalties of step base + j (depth.rs:1358-1361)
            const int s = base + lane;
            if (s < len) {
                const float g = __ldg(gp + s * node_step), g_prev = __ldg(gp + (s - 1) * node_step);
                const float edge_scale = __frcp_rn(1.0f + 4.0f * fabsf(g - g_prev));  // == 1 / x, correctly rounded
                p1s = SGM_SMALL_PENALTY * fmaxf(edge_scale, 0.35f);
                p2s = SGM_LARGE_PENALTY * fmaxf(edge_scale, 0.12f);
            }
        }
        for (int jj = 0; jj < 32; jj += P) {
#pragma unroll
            for (int j = 0; j < P; ++j) {
                const int step = base + jj + j;
                if (step >= len) break;  // uniform over the warp
                float cur[K];
                pf += stride;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    cur[k] = ring[j][k];
                    ring[j][k] = valid[k] && step + P < len ? __ldg(pf + 32 * k) : INFINITY;
                }
                const float p1 = __shfl_sync(full, p1s, jj + j), p2 = __shfl_sync(full, p2s, jj + j);
                float local = prev[0];
#pragma unroll
                for (int k = 1; k < K; ++k) local = fminf(local, prev[k]);
                const float minimum_previous = warp_min_f32(local);
                float up[K], down[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    up[k] = __shfl_sync(full, prev[k], (lane + 31) & 31);   // label - 1 (lane 0: set k - 1's last)
                    down[k] = __shfl_sync(full, prev[k], (lane + 1) & 31);  // label + 1 (lane 31: set k + 1's first)
                }
                const float jump = minimum_previous + p2;
                wp += stride;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float below = lane == 0 ? (k > 0 ? up[k > 0 ? k - 1 : 0] : INFINITY) : up[k];
                    const float above = lane == 31 ? (k + 1 < K ? down[k + 1 < K ? k + 1 : k] : INFINITY) : down[k];
                    const float v =
                        cur[k] + fminf(fminf(fminf(prev[k], below + p1), above + p1), jump) - minimum_previous;
                    prev[k] = v;
                    if (valid[k]) wp[32 * k] = v;
                }
            }
        }
    }
}

// Path costs of every path of every direction; pass k writes paths + k * pitch.
template <int K>
__global__ void __launch_bounds__(32 * SGM_PATHS_PER_CTA) sgm_paths_kernel(const float *__restrict__ data,
                                                                          const float *__restrict__ guidance,
                                                                          float *__restrict__ paths, size_t pitch,
                                                                          int columns, int rows, int labels) {
    const int warp_path = blockIdx.x * SGM_PATHS_PER_CTA + (threadIdx.x >> 5);
    if (warp_path >= (int)sgm_total_paths(columns, rows)) return;  // whole warp
    sgm_walk_path<K>(data, guidance, paths, pitch, columns, rows, labels, warp_path);
}

// The same with one step of prefetch and registers held down so that more CTAs fit an SM:
// on a grid with more paths than the form above keeps resident, every path runs at once
// instead of the last ones starting as the first finish. The same path code, so the same bits.
constexpr int sgm_resident_blocks(int K) { return K <= 5 ? 12 : (K <= 7 ? 10 : 8); }

template <int K>
__global__ void __launch_bounds__(32 * SGM_PATHS_PER_CTA, sgm_resident_blocks(K))
    sgm_paths_resident_kernel(const float *__restrict__ data, const float *__restrict__ guidance,
                              float *__restrict__ paths, size_t pitch, int columns, int rows, int labels) {
    const int warp_path = blockIdx.x * SGM_PATHS_PER_CTA + (threadIdx.x >> 5);
    if (warp_path >= (int)sgm_total_paths(columns, rows)) return;  // whole warp
    sgm_walk_path<K, 1>(data, guidance, paths, pitch, columns, rows, labels, warp_path);
}

// out = ((0 + L1) + L2) + ... + L8 per cell, the reference's order.
__global__ void sgm_sum_kernel(const float *__restrict__ paths, size_t pitch, size_t total,
                               float *__restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) s = s + __ldcs(paths + k * pitch + i);
        out[i] = s;
    }
}

}  // namespace chiaro
