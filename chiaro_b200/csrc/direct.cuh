// direct.cuh — measure_direct_depths (crates/chiaro-fusion/src/depth.rs:715-876)
// with nearest_coarse_depth (1062-1076), direct_depth_candidates (1078-1107),
// select_direct_depth (1109-1165) and best_depth_candidate (1167-1185).
//
// One CTA per fine-grid node. The candidate list is built serially (its
// deduplication depends on the previous entry); the baseline and candidate
// scores are independent (candidate, view) ZNCC items spread over the CTA;
// the selection and the optional wide-radius retry follow the reference.
#pragma once

#include "cost.cuh"
#include "select.cuh"

namespace chiaro {

constexpr int MAX_DIRECT_CANDIDATES = 32;

struct DirectParams {
    const DevView *views;
    int reference, n_targets;
    int targets[MAX_VIEWS];
    int columns, rows, step;                           // fine grid
    Field coarse;                                      // SGM seed field
    int coarse_columns, coarse_rows, coarse_step;
    double inverse_step, near_depth, far_depth;
    const double *unseeded;                            // 32 candidates, far to near
    int radius, wide_radius;
    const float *spatial, *spatial_wide;
    float minimum_score, minimum_margin, minimum_improvement;
    int minimum_support, best_view_count;
    Field out;
    float *guidance;
    uint8_t *tested;
};

// select_direct_depth on (depth, score) pairs; score NaN = None. One thread.
__device__ inline bool select_direct(const double *depths, const float *scores, int n, bool has_baseline,
                                     float baseline, bool seeded, double far_depth, double near_depth,
                                     float minimum_score, float minimum_margin, float minimum_improvement,
                                     double &out_depth, float &out_confidence, float &out_improvement) {
    double far_inverse = 1.0 / far_depth;
    double inverse_range = 1.0 / near_depth - far_inverse;
    int idx[MAX_DIRECT_CANDIDATES + 1];
    float obj[MAX_DIRECT_CANDIDATES + 1];
    int m = 0;
    for (int i = 0; i < n; ++i) {
        if (scores[i] != scores[i]) continue;
        double near_fraction = clampd_r((1.0 / depths[i] - far_inverse) / inverse_range, 0.0, 1.0);
        float objective = scores[i] - NEAR_DEPTH_PRIOR * (float)near_fraction;
        // stable insertion, descending by total order
        int j = m - 1;
        while (j >= 0 && total_key(obj[j]) < total_key(objective)) {
            idx[j + 1] = idx[j];
            obj[j + 1] = obj[j];
            --j;
        }
        idx[j + 1] = i;
        obj[j + 1] = objective;
        ++m;
    }
    if (m == 0) return false;
    int best = idx[0];
    float best_objective = obj[0];
    float score = scores[best];
    float competing = best_objective;
    for (int k = 0; k < m; ++k) {
        int d = idx[k] - best;
        if (d > 1 || d < -1) {
            competing = obj[k];
            break;
        }
    }
    float margin = fmaxf(best_objective - competing, 0.0f);
    float improvement = has_baseline ? score - baseline : 0.0f;
    float score_floor = fmaxf(minimum_score - 0.03f, MINIMUM_REGULARIZED_SCORE);
    float required_margin = seeded ? minimum_margin * 0.6f : minimum_margin;
    bool improves_global = !has_baseline || improvement >= minimum_improvement * 0.5f;
    bool supported = score >= score_floor && improves_global &&
                     (margin >= required_margin || improvement >= minimum_improvement);
    if (!supported) return false;
    float score_confidence = clampf_r((score - score_floor) / fmaxf(1.0f - score_floor, 1.0e-3f), 0.0f, 1.0f);
    float margin_confidence = clampf_r(margin / fmaxf(required_margin, 1.0e-3f), 0.0f, 1.0f);
    out_depth = depths[best];
    out_confidence = clampf_r(0.30f + 0.45f * score_confidence + 0.25f * margin_confidence, 0.0f, 1.0f);
    out_improvement = improvement;
    return true;
}

// best_depth_candidate: last maximum of the objective; -1 for None.
__device__ inline int best_candidate(const double *depths, const float *scores, int n, double far_depth,
                                     double near_depth) {
    double far_inverse = 1.0 / far_depth;
    double inverse_range = 1.0 / near_depth - far_inverse;
    int best = -1;
    float best_objective = 0.0f;
    for (int i = 0; i < n; ++i) {
        if (scores[i] != scores[i]) continue;
        double near_fraction = clampd_r((1.0 / depths[i] - far_inverse) / inverse_range, 0.0, 1.0);
        float objective = scores[i] - NEAR_DEPTH_PRIOR * (float)near_fraction;
        if (best < 0 || !(total_key(objective) < total_key(best_objective))) {
            best = i;
            best_objective = objective;
        }
    }
    return best;
}

struct DirectShared {
    RefPatch patch;
    double cand[MAX_DIRECT_CANDIDATES];
    float agg[MAX_DIRECT_CANDIDATES + 1];  // [0] baseline, [1 + c] candidates; NaN = None
    int n_cand, seeded, wide, first, last, tested;
    double depth;
    float confidence, improvement;
    int has;
};

// Score items (c, v) for c in [-1, n) over candidates cand[first..first+n)
// at the staged radius; aggregate into agg[0..n]. Block-cooperative.
__device__ inline void direct_scores(const DirectParams &p, const NodeSmem &s, DirectShared &d, float *item_scores,
                                     int first, int n, int radius) {
    const int V = p.n_targets;
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    for (int item = threadIdx.x; item < (n + 1) * V; item += blockDim.x) {
        int c = item / V - 1, v = item % V;
        float score = NAN;
        const ViewGeom &g = s.geom[v];
        double ddx = 0.0, ddy = 0.0;
        bool ok = g.gc_ok;
        if (ok && c >= 0) ok = depth_delta(s.cams[1 + v], g, d.cand[first + c], ddx, ddy);
        if (ok && d.patch.ok && g.taps_ok) {
            float sc;
            if (zncc_score(p.views[p.targets[v]].luma, s.gq + v * taps, s.w, s.wr, d.patch, taps, ddx, ddy, sc))
                score = sc;
        }
        item_scores[item] = score;
    }
    __syncthreads();
    for (int c = threadIdx.x; c <= n; c += blockDim.x) {
        float sc[MAX_VIEWS];
        for (int v = 0; v < V; ++v) sc[v] = item_scores[c * V + v];
        float a;
        d.agg[c] = aggregate_scores(sc, V, p.minimum_support, p.best_view_count, a) ? a : NAN;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(128) direct_depth_kernel(DirectParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ DirectShared d;
    __shared__ float item_scores[(MAX_DIRECT_CANDIDATES + 1) * MAX_VIEWS];
    const int node = blockIdx.x;
    const int column = node % p.columns, row = node / p.columns;
    const int V = p.n_targets;
    const int taps_wide = (2 * p.wide_radius + 1) * (2 * p.wide_radius + 1);
    const int taps_max = taps_wide > (2 * p.radius + 1) * (2 * p.radius + 1) ? taps_wide
                                                                              : (2 * p.radius + 1) * (2 * p.radius + 1);
    NodeSmem s = carve_node_smem(smem_raw, V, taps_max);
    const double cx = (double)(column * p.step), cy = (double)(row * p.step);

    load_cameras(s.cams, p.views, p.reference, p.targets, V);
    if (threadIdx.x == 0) {
        // nearest_coarse_depth (depth.rs:1062-1076)
        int cc = sat_index_d(clampd_r(round(cx / (double)p.coarse_step), 0.0, (double)(p.coarse_columns - 1)),
                             p.coarse_columns - 1);
        int cr = sat_index_d(clampd_r(round(cy / (double)p.coarse_step), 0.0, (double)(p.coarse_rows - 1)),
                             p.coarse_rows - 1);
        int ci = cr * p.coarse_columns + cc;
        d.seeded = p.coarse.has[ci];
        // direct_depth_candidates (depth.rs:1078-1107)
        if (d.seeded) {
            double seed = p.coarse.depth[ci];
            double far_inverse = 1.0 / p.far_depth, near_inverse = 1.0 / p.near_depth;
            int n = 0;
            for (int offset = -6; offset <= 6; ++offset) {
                double inv = clampd_r(1.0 / seed + (double)offset * p.inverse_step * 0.5, far_inverse, near_inverse);
                double depth = 1.0 / inv;
                if (n == 0 || fabs(1.0 / d.cand[n - 1] - 1.0 / depth) > p.inverse_step * 0.1) d.cand[n++] = depth;
            }
            d.n_cand = n;
        } else {
            for (int i = 0; i < 32; ++i) d.cand[i] = p.unseeded[i];
            d.n_cand = 32;
        }
        d.wide = 0;
    }
    __syncthreads();
    stage_node(s, d.patch, p.views, p.reference, p.targets, V, cx, cy, p.radius, p.spatial, true);
    direct_scores(p, s, d, item_scores, 0, d.n_cand, p.radius);
    if (threadIdx.x == 0) {
        int n = d.n_cand;
        bool tested = d.agg[0] == d.agg[0];
        for (int c = 0; c < n; ++c) tested |= d.agg[1 + c] == d.agg[1 + c];
        d.tested = tested;
        d.has = select_direct(d.cand, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0], d.seeded, p.far_depth,
                              p.near_depth, p.minimum_score, p.minimum_margin, p.minimum_improvement, d.depth,
                              d.confidence, d.improvement);
        if (!d.has) {
            int best = best_candidate(d.cand, d.agg + 1, n, p.far_depth, p.near_depth);
            if (best >= 0 && d.agg[1 + best] == d.agg[1 + best] && d.agg[1 + best] >= MINIMUM_REGULARIZED_SCORE) {
                d.wide = 1;
                d.first = best >= 3 ? best - 3 : 0;
                d.last = best + 3 < n - 1 ? best + 3 : n - 1;
            }
        }
    }
    __syncthreads();
    if (d.wide) {
        stage_node(s, d.patch, p.views, p.reference, p.targets, V, cx, cy, p.wide_radius, p.spatial_wide, false);
        int n = d.last - d.first + 1;
        direct_scores(p, s, d, item_scores, d.first, n, p.wide_radius);
        if (threadIdx.x == 0)
            d.has = select_direct(d.cand + d.first, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0], d.seeded,
                                  p.far_depth, p.near_depth, p.minimum_score, p.minimum_margin,
                                  p.minimum_improvement, d.depth, d.confidence, d.improvement);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        p.out.has[node] = d.has;
        p.out.depth[node] = d.has ? d.depth : NAN;
        p.out.confidence[node] = d.has ? d.confidence : 0.0f;
        p.out.improvement[node] = d.has ? d.improvement : 0.0f;
        p.out.regularized[node] = 0;
        p.tested[node] = d.tested;
        p.guidance[node] = d.patch.centre;  // reference_guidance: the centre sample or 0
    }
}

}  // namespace chiaro
