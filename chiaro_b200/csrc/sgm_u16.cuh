// sgm_u16.cuh — the quantised performance mode of semi_global_costs
// (crates/chiaro-fusion/src/depth.rs:1279-1383). The reference has no such mode;
// it is the packed-integer SGM of the design, checked bit for bit against the
// oracle's integer restatement (oracle_sgm_u16) and within one plane against the
// f32 path.
//
// Costs become u16 fixed point, Q = 2048 per cost unit (the stage's costs lie in
// [0, 2.25], so at most 4608); the edge penalties p1, p2 are the reference's f32
// values quantised the same way (at most 922). A path cost is then at most
// 4608 + 922 = 5530 and the sum of the 8 paths at most 44240, so the recurrence
// and the sum are exact in 16 bits: no saturation ever applies to a real label.
// Integer addition is associative, so the 8 directions need no summation order:
// every path adds its costs straight into one packed aggregate with a 32-bit
// atomic add (a red.global.add, resolved in L2). A real label's 8-path sum never
// exceeds 16 bits, so no carry crosses into the pair's high half; the pad label
// of an odd count (0xFFFF on every path) sits in the high half, where its carry
// leaves the word, and no one reads it. No per-direction buffer is written: the
// cells cross DRAM about once each way (quantised costs in, aggregate out) while
// the 8 walks read the costs and add into the aggregate in L2.
//
// Labels travel in pairs, (2j, 2j + 1) packed in one 32-bit word, and the
// recurrence runs on both halves at once with __vaddus2 / __vminu2 / __vsub2.
// A path is walked by one warp; lane i holds pairs i, i + 32, ... (K sets). The
// neighbour below a pair's low label is the high label of the previous lane's
// pair (lane 31 of the previous set for lane 0), the neighbour above its high
// label the low label of the next lane's pair; __byte_perm assembles both
// shifted words from the two shuffles. Labels past the last one, including the
// pad label of an odd count, hold 0xFFFF and stay there (saturating adds).
#pragma once

#include "sgm.cuh"

namespace chiaro {

constexpr float SGM_Q = 2048.0f;
constexpr unsigned SGM_COST_MAX_Q = 4608u;  // 2.25 * Q
constexpr unsigned SGM_U16_PAD = 0xFFFFu;

__device__ __forceinline__ unsigned quantise_sgm_cost(float c) {
    if (!(c == c)) return SGM_COST_MAX_Q;  // NaN: the missing cost
    const float v = rintf(c * SGM_Q);      // round half to even, like the host's nearbyint
    if (v <= 0.0f) return 0u;
    return v >= (float)SGM_COST_MAX_Q ? SGM_COST_MAX_Q : (unsigned)v;
}

__device__ __forceinline__ unsigned quantise_penalty(float p) { return (unsigned)rintf(p * SGM_Q); }

// f32 [N][D] costs -> u16 pairs [N][pairs], pairs = ceil(D / 2); the pad label is 0xFFFF.
// The aggregate's words are cleared in the same pass.
__global__ void sgm_quantise_kernel(const float *__restrict__ costs, int nodes, int labels,
                                    unsigned *__restrict__ quantised, unsigned *__restrict__ aggregate) {
    const int pairs = (labels + 1) / 2;
    const long total = (long)nodes * pairs;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int node = (int)(i / pairs), j = (int)(i - (long)node * pairs);
        const float *c = costs + (size_t)node * labels + 2 * j;
        const unsigned lo = quantise_sgm_cost(c[0]);
        const unsigned hi = 2 * j + 1 < labels ? quantise_sgm_cost(c[1]) : SGM_U16_PAD;
        quantised[i] = lo | (hi << 16);
        aggregate[i] = 0u;
    }
}

// Every path of every direction, each adding its path costs into the packed
// aggregate [N][pairs] (cleared beforehand).
template <int K>
__global__ void __launch_bounds__(32 * SGM_PATHS_PER_CTA) sgm_u16_paths_kernel(const unsigned *__restrict__ data,
                                                                              const float *__restrict__ guidance,
                                                                              unsigned *__restrict__ aggregate,
                                                                              int columns, int rows, int labels) {
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
    constexpr int P = SGM_PREFETCH;
    const int pairs = (labels + 1) / 2;
    bool valid[K];
#pragma unroll
    for (int k = 0; k < K; ++k) valid[k] = lane + 32 * k < pairs;
    const long node_step = (long)dr * columns + dc;
    const long stride = node_step * pairs;
    const int node0 = r0 * columns + c0;
    const size_t e0 = (size_t)node0 * pairs + lane;
    const unsigned *pf = data + e0;
    unsigned *wp = aggregate + e0;
    const float *gp = guidance + node0;
    unsigned prev[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        prev[k] = valid[k] ? __ldg(pf + 32 * k) : full;
        if (valid[k]) atomicAdd(wp + 32 * k, prev[k]);
    }
    unsigned ring[P][K];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        pf += stride;
#pragma unroll
        for (int k = 0; k < K; ++k) ring[j][k] = valid[k] && 1 + j < len ? __ldg(pf + 32 * k) : full;
    }
    unsigned p1s = 0u, p2s = 0u;
    for (int base = 1; base < len; base += 32) {
        {  // lane j: quantised penalties of step base + j (depth.rs:1358-1361)
            const int s = base + lane;
            if (s < len) {
                const float g = __ldg(gp + s * node_step), g_prev = __ldg(gp + (s - 1) * node_step);
                const float edge_scale = __frcp_rn(1.0f + 4.0f * fabsf(g - g_prev));  // == 1 / x, correctly rounded
                p1s = quantise_penalty(SGM_SMALL_PENALTY * fmaxf(edge_scale, 0.35f));
                p2s = quantise_penalty(SGM_LARGE_PENALTY * fmaxf(edge_scale, 0.12f));
            }
        }
        for (int jj = 0; jj < 32; jj += P) {
#pragma unroll
            for (int j = 0; j < P; ++j) {
                const int step = base + jj + j;
                if (step >= len) break;  // uniform over the warp
                unsigned cur[K];
                pf += stride;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    cur[k] = ring[j][k];
                    ring[j][k] = valid[k] && step + P < len ? __ldg(pf + 32 * k) : full;
                }
                const unsigned p1 = __shfl_sync(full, p1s, jj + j) * 0x10001u;
                const unsigned p2 = __shfl_sync(full, p2s, jj + j);
                unsigned local = prev[0];
#pragma unroll
                for (int k = 1; k < K; ++k) local = __vminu2(local, prev[k]);
                const unsigned minimum_previous = __reduce_min_sync(full, min(local & 0xFFFFu, local >> 16));
                const unsigned floor2 = minimum_previous * 0x10001u;
                const unsigned jump = (minimum_previous + p2) * 0x10001u;
                unsigned up[K], down[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    up[k] = __shfl_sync(full, prev[k], (lane + 31) & 31);   // lane 0: lane 31 of this set
                    down[k] = __shfl_sync(full, prev[k], (lane + 1) & 31);  // lane 31: lane 0 of this set
                }
                wp += stride;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    // the word holding label 2j - 1 in its high half, and the one holding 2j + 2 in its low half
                    const unsigned left = lane == 0 ? (k > 0 ? up[k > 0 ? k - 1 : 0] : full) : up[k];
                    const unsigned right = lane == 31 ? (k + 1 < K ? down[k + 1 < K ? k + 1 : k] : full) : down[k];
                    const unsigned below = __byte_perm(left, prev[k], 0x5432);  // (label 2j - 1, label 2j)
                    const unsigned above = __byte_perm(prev[k], right, 0x5432);  // (label 2j + 1, label 2j + 2)
                    unsigned best = __vminu2(prev[k], __vaddus2(below, p1));
                    best = __vminu2(best, __vaddus2(above, p1));
                    best = __vminu2(best, jump);
                    const unsigned v = __vaddus2(cur[k], __vsub2(best, floor2));
                    prev[k] = v;
                    if (valid[k]) atomicAdd(wp + 32 * k, v);
                }
            }
        }
    }
}

// The packed aggregate written unpadded ([N][D], optional) and the winner over
// labels 1..D-1 (first minimum, optional). A warp per node.
__global__ void __launch_bounds__(256) sgm_u16_select_kernel(const unsigned *__restrict__ packed, int nodes,
                                                             int labels, uint16_t *aggregate, uint16_t *best) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (node >= nodes) return;  // whole warp
    const int pairs = (labels + 1) / 2;
    unsigned key = full;  // (cost << 16) | label: the minimum is the first minimum
    for (int j = lane; j < pairs; j += 32) {
        const unsigned s = __ldcs(packed + (size_t)node * pairs + j);
        const int lo = 2 * j, hi = 2 * j + 1;
        if (aggregate) {
            aggregate[(size_t)node * labels + lo] = (uint16_t)(s & 0xFFFFu);
            if (hi < labels) aggregate[(size_t)node * labels + hi] = (uint16_t)(s >> 16);
        }
        if (lo >= 1) key = min(key, ((s & 0xFFFFu) << 16) | (unsigned)lo);
        if (hi < labels) key = min(key, (s & 0xFFFF0000u) | (unsigned)hi);
    }
    key = __reduce_min_sync(full, key);
    if (best && lane == 0) best[node] = labels > 1 ? (uint16_t)(key & 0xFFFFu) : (uint16_t)0;
}

}  // namespace chiaro
