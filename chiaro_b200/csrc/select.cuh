// select.cuh — select_depths (crates/chiaro-fusion/src/depth.rs:1385-1467),
// sublabel_depth (depth.rs:1469-1488) and complete_depth_field
// (depth.rs:1490-1564).
//
// One warp per coarse node: the winner-take-all over the finite labels is a
// warp argmin on (total-order key, label), which keeps the first minimum like
// Iterator::min_by; the competing cost is a warp min over labels more than two
// away from the winner.
#pragma once

#include "common.cuh"

namespace chiaro {

struct Field {  // Option<NodeDepth> per node (depth.rs:248-254)
    uint8_t *has;
    double *depth;
    float *confidence;
    float *improvement;
    uint8_t *regularized;
};

struct SelectParams {
    const float *scores, *regularised;
    const uint8_t *tested;
    const double *label_depth;  // [D], label 0 unused
    int nodes, labels;
    float minimum_score, minimum_margin, minimum_improvement;
    Field field;
    uint8_t *fillable;
};

__device__ inline double sublabel_depth(const double *labels, const float *costs, int best, int n) {
    double centre_depth = labels[best];
    if (best <= 1 || best + 1 >= n) return centre_depth;
    float left = costs[best - 1], centre = costs[best], right = costs[best + 1];
    float curvature = left - 2.0f * centre + right;
    if (!isfinite(curvature) || curvature <= 1.0e-6f) return centre_depth;
    double offset = (double)clampf_r(0.5f * (left - right) / curvature, -0.75f, 0.75f);
    double lower_inverse = 1.0 / labels[best - 1];
    double upper_inverse = 1.0 / labels[best + 1];
    double inverse_step = (upper_inverse - lower_inverse) * 0.5;
    return 1.0 / (1.0 / centre_depth + offset * inverse_step);
}

__global__ void __launch_bounds__(256) select_depths_kernel(SelectParams p) {
    const int lane = threadIdx.x & 31;
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (node >= p.nodes) return;
    const unsigned full = 0xffffffffu;
    Field f = p.field;
    if (lane == 0) {  // None unless a depth is selected below
        f.has[node] = 0;
        f.depth[node] = NAN;
        f.confidence[node] = 0.0f;
        f.improvement[node] = 0.0f;
        f.regularized[node] = 0;
        p.fillable[node] = 0;
    }
    if (!p.tested[node]) return;
    const float *reg = p.regularised + (size_t)node * p.labels;
    // argmin over labels 1..D-1: smallest (key, label)
    int32_t best_key = INT32_MAX;
    int best_label = INT32_MAX;
    for (int l = 1 + lane; l < p.labels; l += 32) {
        int32_t key = total_key(reg[l]);
        if (key < best_key) {
            best_key = key;
            best_label = l;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        int32_t ok = __shfl_xor_sync(full, best_key, off);
        int ol = __shfl_xor_sync(full, best_label, off);
        if (ok < best_key || (ok == best_key && ol < best_label)) {
            best_key = ok;
            best_label = ol;
        }
    }
    const float best_cost = reg[best_label];
    // competing: min over |label - best| > 2
    int32_t comp_key = INT32_MAX;
    for (int l = 1 + lane; l < p.labels; l += 32) {
        int d = l - best_label;
        if (d > 2 || d < -2) comp_key = min(comp_key, total_key(reg[l]));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) comp_key = min(comp_key, __shfl_xor_sync(full, comp_key, off));
    float competing = best_cost;
    if (comp_key != INT32_MAX) {
        // recover the value of the minimum key
        for (int l = 1 + lane; l < p.labels; l += 32) {
            int d = l - best_label;
            if ((d > 2 || d < -2) && total_key(reg[l]) == comp_key) competing = reg[l];
        }
        unsigned has_it = __ballot_sync(full, total_key(competing) == comp_key);
        competing = __shfl_sync(full, competing, __ffs(has_it) - 1);
    }
    if (lane != 0) return;
    double depth = sublabel_depth(p.label_depth, reg, best_label, p.labels);
    float score = p.scores[(size_t)node * p.labels + best_label];
    if (!isfinite(score) || score < MINIMUM_REGULARIZED_SCORE) {
        p.fillable[node] = 1;
        return;
    }
    float margin = fmaxf((competing - best_cost) / SGM_DIRECTIONS, 0.0f);
    float baseline = p.scores[(size_t)node * p.labels];
    float improvement = isfinite(baseline) ? score - baseline : 0.0f;
    if (isfinite(baseline) && improvement < -MAXIMUM_REGULARIZED_BASELINE_LOSS) return;
    bool measured = score >= p.minimum_score && improvement >= p.minimum_improvement * 0.5f &&
                    (margin >= p.minimum_margin || improvement >= p.minimum_improvement);
    float score_confidence =
        clampf_r((score - p.minimum_score) / fmaxf(1.0f - p.minimum_score, 1.0e-3f), 0.0f, 1.0f);
    float margin_confidence = clampf_r(margin / fmaxf(p.minimum_margin, 1.0e-3f), 0.0f, 1.0f);
    float improvement_confidence = clampf_r(improvement / fmaxf(p.minimum_improvement, 1.0e-3f), 0.0f, 1.0f);
    float confidence = measured ? clampf_r(0.30f + 0.45f * score_confidence + 0.25f * margin_confidence, 0.0f, 1.0f)
                                : clampf_r(0.10f + 0.25f * score_confidence + 0.15f * margin_confidence +
                                               0.10f * improvement_confidence,
                                           0.10f, 0.55f);
    f.has[node] = 1;
    f.depth[node] = depth;
    f.confidence[node] = confidence;
    f.improvement[node] = improvement;
    f.regularized[node] = measured ? 0 : 1;
}

// One iteration of complete_depth_field (depth.rs:1498-1563): reads `src`,
// writes `dst` (a copy of src on entry). Running the configured number of
// iterations without the early exit gives the same field: an iteration that
// changes nothing is a fixed point.
struct CompleteParams {
    Field src, dst;
    const float *guidance;
    const uint8_t *fillable;
    int columns, rows, minimum_neighbour_support;
};

__global__ void complete_depth_kernel(CompleteParams p) {
    int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= p.columns * p.rows) return;
    if (p.src.has[index] || !p.fillable[index]) return;
    int column = index % p.columns, row = index / p.columns;
    double inv[8];
    float wt[8];
    int n = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int x = column + dx, y = row + dy;
            if (x < 0 || y < 0 || x >= p.columns || y >= p.rows) continue;
            int ni = y * p.columns + x;
            if (!p.src.has[ni]) continue;
            float edge = fabsf(p.guidance[index] - p.guidance[ni]);
            if (edge > 0.35f) continue;
            float spatial = (dx != 0 && dy != 0) ? 0.707f : 1.0f;
            float weight = p.src.confidence[ni] * spatial * exp_f32(-3.0f * edge);
            if (weight >= 0.05f) {
                inv[n] = 1.0 / p.src.depth[ni];
                wt[n] = weight;
                ++n;
            }
        }
    if (n < p.minimum_neighbour_support) return;
    // stable sort by inverse depth (total order)
    for (int i = 1; i < n; ++i) {
        double vi = inv[i];
        float wi = wt[i];
        int j = i - 1;
        while (j >= 0 && (int64_t)(d2u(inv[j]) ^ (((uint64_t)((int64_t)d2u(inv[j]) >> 63)) >> 1)) >
                             (int64_t)(d2u(vi) ^ (((uint64_t)((int64_t)d2u(vi) >> 63)) >> 1))) {
            inv[j + 1] = inv[j];
            wt[j + 1] = wt[j];
            --j;
        }
        inv[j + 1] = vi;
        wt[j + 1] = wi;
    }
    float total = -0.0f;
    for (int i = 0; i < n; ++i) total += wt[i];
    float accumulated = 0.0f;
    double inverse_depth = inv[n / 2];
    for (int i = 0; i < n; ++i) {
        accumulated += wt[i];
        if (accumulated >= total * 0.5f) {
            inverse_depth = inv[i];
            break;
        }
    }
    float maxw = 0.0f;
    for (int i = 0; i < n; ++i) maxw = fmaxf(maxw, wt[i]);
    p.dst.has[index] = 1;
    p.dst.depth[index] = 1.0 / inverse_depth;
    p.dst.confidence[index] = clampf_r(maxw * 0.92f, 0.15f, 0.75f);
    p.dst.improvement[index] = 0.0f;
    p.dst.regularized[index] = 1;
}

}  // namespace chiaro
