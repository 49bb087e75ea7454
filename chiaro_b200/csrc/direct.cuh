// direct.cuh — measure_direct_depths (crates/chiaro-fusion/src/depth.rs:715-876)
// with nearest_coarse_depth (1062-1076), direct_depth_candidates (1078-1107),
// select_direct_depth (1109-1165) and best_depth_candidate (1167-1185).
//
// A warp per fine-grid node, several nodes per CTA. The candidate list is built
// serially (its deduplication depends on the previous entry); the baseline and
// candidate scores are independent (candidate, view) ZNCC items spread over the
// warp; the selection follows the reference. Nodes that need the wide-radius
// retry go to a list that a second kernel processes with its larger patch.
#pragma once

#include "cost.cuh"
#include "select.cuh"

namespace chiaro {

constexpr int MAX_DIRECT_CANDIDATES = 32;

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

// ---- warp-per-node direct pass ---------------------------------------------------
struct DirectParams {
    const DevView *views;
    int reference, n_targets;
    int targets[MAX_VIEWS];
    int columns, rows, step;                           // fine grid
    Field coarse;                                      // SGM seed field
    int coarse_columns, coarse_rows, coarse_step;
    double inverse_step, near_depth, far_depth;
    const double *unseeded;                            // 32 candidates, far to near
    const GeomRec *geometry;                           // [node][target] of the fine grid
    int radius, wide_radius;
    const float *spatial, *spatial_wide;
    float minimum_score, minimum_margin, minimum_improvement;
    int minimum_support, best_view_count;
    int nodes_per_cta;
    Field out;
    float *guidance;
    uint8_t *tested;
    int *wide_count;                                   // wide-retry list length
    int4 *wide_list;                                   // (node, first, last, seeded)
};

// Per-warp shared memory of the direct pass for V targets and T taps.
struct DirectSlot {
    float *r, *w, *wr;   // [T]
    double2 *gh;         // [V][T] g/2 (fast path)
    TapBox *box;         // [V]
    double *cand;        // [32]
    float *items;        // [33][V]
    float *agg;          // [33]: [0] baseline, [1 + c] candidates
};

__host__ __device__ inline size_t direct_slot_bytes(int V, int taps) {
    return align16(3 * taps * sizeof(float)) + align16((size_t)V * taps * sizeof(double2)) +
           align16(V * sizeof(TapBox)) +
           align16(MAX_DIRECT_CANDIDATES * sizeof(double)) +
           align16((size_t)(MAX_DIRECT_CANDIDATES + 1) * V * sizeof(float)) +
           align16((MAX_DIRECT_CANDIDATES + 1) * sizeof(float));
}

__device__ inline DirectSlot carve_direct_slot(unsigned char *base, int V, int taps) {
    DirectSlot d;
    size_t o = 0;
    d.r = reinterpret_cast<float *>(base);
    d.w = d.r + taps;
    d.wr = d.w + taps;
    o += align16(3 * taps * sizeof(float));
    d.gh = reinterpret_cast<double2 *>(base + o);
    o += align16((size_t)V * taps * sizeof(double2));
    d.box = reinterpret_cast<TapBox *>(base + o);
    o += align16(V * sizeof(TapBox));
    d.cand = reinterpret_cast<double *>(base + o);
    o += align16(MAX_DIRECT_CANDIDATES * sizeof(double));
    d.items = reinterpret_cast<float *>(base + o);
    o += align16((size_t)(MAX_DIRECT_CANDIDATES + 1) * V * sizeof(float));
    d.agg = reinterpret_cast<float *>(base + o);
    return d;
}

// nearest_coarse_depth (depth.rs:1062-1076) and direct_depth_candidates
// (depth.rs:1078-1107); returns the candidate count, sets *seeded.
__device__ inline int direct_candidates(const DirectParams &p, double cx, double cy, double *cand, int *seeded) {
    int cc = sat_index_d(clampd_r(round(cx / (double)p.coarse_step), 0.0, (double)(p.coarse_columns - 1)),
                         p.coarse_columns - 1);
    int cr = sat_index_d(clampd_r(round(cy / (double)p.coarse_step), 0.0, (double)(p.coarse_rows - 1)),
                         p.coarse_rows - 1);
    int ci = cr * p.coarse_columns + cc;
    *seeded = p.coarse.has[ci];
    if (!*seeded) {
        for (int i = 0; i < 32; ++i) cand[i] = p.unseeded[i];
        return 32;
    }
    double seed = p.coarse.depth[ci];
    double far_inverse = 1.0 / p.far_depth, near_inverse = 1.0 / p.near_depth;
    int n = 0;
    for (int offset = -6; offset <= 6; ++offset) {
        double inv = clampd_r(1.0 / seed + (double)offset * p.inverse_step * 0.5, far_inverse, near_inverse);
        double depth = 1.0 / inv;
        if (n == 0 || fabs(1.0 / cand[n - 1] - 1.0 / depth) > p.inverse_step * 0.1) cand[n++] = depth;
    }
    return n;
}

// Warp-cooperative: reference patch (r, w, wr and the sums) and every target's
// tap positions for one node at `radius`; geometry from the records.
__device__ inline void warp_stage_node(const DirectParams &p, const DirectSlot &d, RefPatch &patch, ViewGeom *geom,
                                       double cx, double cy, int radius, const float *spatial, const GeomRec *recs) {
    const int lane = threadIdx.x & 31;
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    const int V = p.n_targets;
    const DevView &rv = p.views[p.reference];
    float centre = 0.0f;
    bool centre_ok = plane_sample(rv.luma, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
    if (lane == 0) {
        patch.ok = centre_ok;
        patch.centre = centre;
    }
    if (lane < V) {
        if (recs) geom_from_rec(recs[lane], camera_origin(rv.cam), geom[lane]);
        geom[lane].taps_ok = 1;
    }
    __syncwarp();
    for (int t = lane; t < taps; t += 32) {
        int dx, dy;
        tap_offset(t, radius, dx, dy);
        double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
        float value = 0.0f;
        if (!plane_sample(rv.luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value)) patch.ok = 0;
        float weight = spatial[t] * exp_f32(-1.2f * fabsf(value - centre));
        d.r[t] = value;
        d.w[t] = weight;
        d.wr[t] = weight * value;
        for (int v = 0; v < V; ++v) {
            float qx = 0.0f, qy = 0.0f;
            if (!warp_map(p.views[p.targets[v]].warp, (float)px, (float)py, qx, qy)) geom[v].taps_ok = 0;
            d.gh[v * taps + t] = make_double2((double)qx * 0.5, (double)qy * 0.5);
        }
    }
    __syncwarp();
    for (int v = 0; v < V; ++v) {
        TapBox b = warp_tap_box(d.gh + v * taps, taps);
        if (lane == 0) d.box[v] = b;
    }
    if (lane < 3) {
        float sum = 0.0f;
        if (lane == 0)
            for (int t = 0; t < taps; ++t) sum += d.w[t];
        else if (lane == 1)
            for (int t = 0; t < taps; ++t) sum += d.wr[t];
        else
            for (int t = 0; t < taps; ++t) sum += d.wr[t] * d.r[t];
        if (lane == 0) patch.count = sum;
        if (lane == 1) patch.sum_r = sum;
        if (lane == 2) patch.sum_rr = sum;
    }
    __syncwarp();
    if (lane == 0) patch.ref_energy = patch.sum_rr - patch.sum_r * patch.sum_r / patch.count;
    __syncwarp();
}

// Warp-cooperative scores of the baseline and candidates cand[0..n) over all
// targets, aggregated into d.agg[0..n]. NaN = None.
__device__ inline void warp_direct_scores(const DirectParams &p, const DirectSlot &d, const RefPatch &patch,
                                          const ViewGeom *geom, const double *cand, int n, int radius) {
    const int lane = threadIdx.x & 31;
    const int V = p.n_targets;
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    for (int item = lane; item < (n + 1) * V; item += 32) {
        int c = item / V - 1, v = item % V;
        float score = NAN;
        const ViewGeom &g = geom[v];
        double ddx = 0.0, ddy = 0.0;
        bool ok = g.gc_ok;
        if (ok && c >= 0) ok = depth_delta(p.views[p.targets[v]].cam, g, cand[c], ddx, ddy);
        if (ok && patch.ok && g.taps_ok) {
            const DevView &tv = p.views[p.targets[v]];
            float sc;
            if (zncc_any(TargetRef{tv.luma, tv.pairs}, d.gh + v * taps, d.box[v], d.w, d.wr, patch, taps, ddx, ddy,
                         sc))
                score = sc;
        }
        d.items[item] = score;
    }
    __syncwarp();
    for (int c = lane; c <= n; c += 32) {
        float sc[MAX_VIEWS];
        for (int v = 0; v < V; ++v) sc[v] = d.items[c * V + v];
        float a;
        d.agg[c] = aggregate_scores(sc, V, p.minimum_support, p.best_view_count, a) ? a : NAN;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(256) direct_depth_kernel(DirectParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patches[8];
    __shared__ ViewGeom geoms[8][MAX_VIEWS];
    __shared__ int n_cand[8], seeded_s[8];
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int node = blockIdx.x * p.nodes_per_cta + slot;
    if (slot >= p.nodes_per_cta || node >= p.columns * p.rows) return;  // whole warps
    const int V = p.n_targets;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    DirectSlot d = carve_direct_slot(smem_raw + (size_t)slot * direct_slot_bytes(V, taps), V, taps);
    RefPatch &patch = patches[slot];
    const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
    if (lane == 0) n_cand[slot] = direct_candidates(p, cx, cy, d.cand, &seeded_s[slot]);
    warp_stage_node(p, d, patch, geoms[slot], cx, cy, p.radius, p.spatial, p.geometry + (size_t)node * V);
    const int n = n_cand[slot];
    warp_direct_scores(p, d, patch, geoms[slot], d.cand, n, p.radius);
    if (lane != 0) return;
    bool tested = d.agg[0] == d.agg[0];
    for (int c = 0; c < n; ++c) tested |= d.agg[1 + c] == d.agg[1 + c];
    double depth = 0.0;
    float confidence = 0.0f, improvement = 0.0f;
    bool has = select_direct(d.cand, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0], seeded_s[slot], p.far_depth,
                             p.near_depth, p.minimum_score, p.minimum_margin, p.minimum_improvement, depth,
                             confidence, improvement);
    p.tested[node] = tested;
    p.guidance[node] = patch.centre;  // reference_guidance (depth.rs:1824-1832)
    p.out.has[node] = has;
    p.out.depth[node] = has ? depth : NAN;
    p.out.confidence[node] = has ? confidence : 0.0f;
    p.out.improvement[node] = has ? improvement : 0.0f;
    p.out.regularized[node] = 0;
    if (!has) {
        int best = best_candidate(d.cand, d.agg + 1, n, p.far_depth, p.near_depth);
        if (best >= 0 && d.agg[1 + best] == d.agg[1 + best] && d.agg[1 + best] >= MINIMUM_REGULARIZED_SCORE) {
            int first = best >= 3 ? best - 3 : 0;
            int last = best + 3 < n - 1 ? best + 3 : n - 1;
            int k = atomicAdd(p.wide_count, 1);
            p.wide_list[k] = make_int4(node, first, last, seeded_s[slot]);
        }
    }
}

// The wide-radius retry (depth.rs:803-846) for the listed nodes; a warp per
// entry, persistent over the list.
__global__ void __launch_bounds__(128) direct_wide_kernel(DirectParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patches[4];
    __shared__ ViewGeom geoms[4][MAX_VIEWS];
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int V = p.n_targets;
    const int taps = (2 * p.wide_radius + 1) * (2 * p.wide_radius + 1);
    DirectSlot d = carve_direct_slot(smem_raw + (size_t)slot * direct_slot_bytes(V, taps), V, taps);
    RefPatch &patch = patches[slot];
    const int count = *p.wide_count;
    for (int e = blockIdx.x * 4 + slot; e < count; e += gridDim.x * 4) {
        int4 entry = p.wide_list[e];
        const int node = entry.x, first = entry.y, last = entry.z;
        const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
        if (lane == 0) {
            int seeded;
            direct_candidates(p, cx, cy, d.cand, &seeded);
        }
        __syncwarp();
        warp_stage_node(p, d, patch, geoms[slot], cx, cy, p.wide_radius, p.spatial_wide,
                        p.geometry + (size_t)node * V);
        const int n = last - first + 1;
        warp_direct_scores(p, d, patch, geoms[slot], d.cand + first, n, p.wide_radius);
        if (lane == 0) {
            double depth = 0.0;
            float confidence = 0.0f, improvement = 0.0f;
            bool has = select_direct(d.cand + first, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0], entry.w != 0,
                                     p.far_depth, p.near_depth, p.minimum_score, p.minimum_margin,
                                     p.minimum_improvement, depth, confidence, improvement);
            if (has) {
                p.out.has[node] = 1;
                p.out.depth[node] = depth;
                p.out.confidence[node] = confidence;
                p.out.improvement[node] = improvement;
            }
        }
        __syncwarp();
    }
}

}  // namespace chiaro
