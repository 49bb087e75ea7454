// direct.cuh — measure_direct_depths (crates/chiaro-fusion/src/depth.rs:715-876)
// with nearest_coarse_depth (1062-1076), direct_depth_candidates (1078-1107),
// select_direct_depth (1109-1165) and best_depth_candidate (1167-1185).
//
// A warp per fine-grid node, as many nodes per CTA as keep the most warps
// resident. The thirteen seeded candidates are computed one per lane and
// deduplicated by a uniform scan; the baseline and candidate scores are
// independent (candidate, view) ZNCC items, listed fast-path first and spread
// over the warp; the selection replaces the reference's sort by warp
// reductions. Nodes that need the wide-radius retry go to a list that a second
// kernel processes with its larger patch.
#pragma once

#include "cost.cuh"
#include "select.cuh"

namespace chiaro {

constexpr int MAX_DIRECT_CANDIDATES = 32;
constexpr int KEY_NONE = -2147483647 - 1;  // below every total_key of a non-NaN float

// select_direct_depth (depth.rs:1109-1165) and best_depth_candidate
// (depth.rs:1167-1185) over (depth, score) pairs, score NaN = None, computed by
// a whole warp: lane c < n holds candidate c's objective. The reference sorts
// the objectives stably in descending total order; its head is the first
// maximum, and its first entry more than one index away from the head has the
// largest objective among those entries, so two warp max-reductions replace
// the sort. best_depth_candidate keeps the last maximum (`best_last`, -1 for
// None). Every lane returns the same result.
__device__ inline bool warp_select_direct(const double *depths, const float *scores, int n, bool has_baseline,
                                          float baseline, bool seeded, double far_depth, double near_depth,
                                          float minimum_score, float minimum_margin, float minimum_improvement,
                                          double &out_depth, float &out_confidence, float &out_improvement,
                                          int &best_last) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double far_inverse = 1.0 / far_depth;
    double inverse_range = 1.0 / near_depth - far_inverse;
    bool valid = false;
    float objective = 0.0f;
    if (lane < n) {
        float s = scores[lane];
        valid = !(s != s);
        if (valid) {
            double near_fraction = clampd_r((1.0 / depths[lane] - far_inverse) / inverse_range, 0.0, 1.0);
            objective = s - NEAR_DEPTH_PRIOR * (float)near_fraction;
        }
    }
    best_last = -1;
    if (!__ballot_sync(full, valid)) return false;
    const int key = valid ? total_key(objective) : KEY_NONE;
    const int top = __reduce_max_sync(full, key);
    const unsigned at_top = __ballot_sync(full, valid && key == top);
    const int best = __ffs(at_top) - 1;
    best_last = 31 - __clz(at_top);
    const float best_objective = __shfl_sync(full, objective, best);
    const bool away = valid && (lane - best > 1 || lane - best < -1);
    const unsigned away_mask = __ballot_sync(full, away);
    float competing = best_objective;
    if (away_mask) {
        const int away_top = __reduce_max_sync(full, away ? key : KEY_NONE);
        const int c = __ffs(__ballot_sync(full, away && key == away_top)) - 1;
        competing = __shfl_sync(full, objective, c);
    }
    float score = scores[best];
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
    TapLattice lattice;                                // of the fine grid, or planes == nullptr
    const RefPatch *patches;                           // [node] reference patch at `radius`, or nullptr
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

// Per-warp shared memory of the direct pass for V targets and T taps; TapT
// is the tap-position storage (double2 g/2 or float2 g).
template <typename TapT>
struct DirectSlot {
    float *rr;             // [T] (w r) r
    float2 *wt;            // [T] (w, w r)
    ViewGeom *geom;        // [V]
    TapT *gh;              // [V][T] tap positions
    TapBox *box;           // [V]
    double *cand;          // [32]
    float *items;          // [33][V]
    float *agg;            // [33]: [0] baseline, [1 + c] candidates
    unsigned short *list;  // [33][V] scored items: fast path from the front, exact path from the back
};

template <typename TapT>
__host__ __device__ inline size_t direct_slot_bytes(int V, int taps) {
    return align16(taps * sizeof(float)) + align16(taps * sizeof(float2)) + align16(V * sizeof(ViewGeom)) +
           align16((size_t)V * taps * sizeof(TapT)) + align16(V * sizeof(TapBox)) +
           align16(MAX_DIRECT_CANDIDATES * sizeof(double)) +
           align16((size_t)(MAX_DIRECT_CANDIDATES + 1) * V * sizeof(float)) +
           align16((MAX_DIRECT_CANDIDATES + 1) * sizeof(float)) +
           align16((size_t)(MAX_DIRECT_CANDIDATES + 1) * V * sizeof(unsigned short));
}

template <typename TapT>
__device__ inline DirectSlot<TapT> carve_direct_slot(unsigned char *base, int V, int taps) {
    DirectSlot<TapT> d;
    size_t o = 0;
    d.rr = reinterpret_cast<float *>(base);
    o += align16(taps * sizeof(float));
    d.wt = reinterpret_cast<float2 *>(base + o);
    o += align16(taps * sizeof(float2));
    d.geom = reinterpret_cast<ViewGeom *>(base + o);
    o += align16(V * sizeof(ViewGeom));
    d.gh = reinterpret_cast<TapT *>(base + o);
    o += align16((size_t)V * taps * sizeof(TapT));
    d.box = reinterpret_cast<TapBox *>(base + o);
    o += align16(V * sizeof(TapBox));
    d.cand = reinterpret_cast<double *>(base + o);
    o += align16(MAX_DIRECT_CANDIDATES * sizeof(double));
    d.items = reinterpret_cast<float *>(base + o);
    o += align16((size_t)(MAX_DIRECT_CANDIDATES + 1) * V * sizeof(float));
    d.agg = reinterpret_cast<float *>(base + o);
    o += align16((MAX_DIRECT_CANDIDATES + 1) * sizeof(float));
    d.list = reinterpret_cast<unsigned short *>(base + o);
    return d;
}

// nearest_coarse_depth (depth.rs:1062-1076) and direct_depth_candidates
// (depth.rs:1078-1107) by a whole warp; returns the candidate count (every
// lane) and sets `seeded`. Lane k < 13 computes offset k - 6's depth and its
// inverse; the deduplication against the last kept entry is a uniform scan of
// those inverses (1 / cand[n - 1] is the kept entry's inverse, computed the
// same way), then the kept depths are written in order.
__device__ inline int warp_direct_candidates(const DirectParams &p, double cx, double cy, double *cand,
                                             int &seeded) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int cc = sat_index_d(clampd_r(round(cx / (double)p.coarse_step), 0.0, (double)(p.coarse_columns - 1)),
                         p.coarse_columns - 1);
    int cr = sat_index_d(clampd_r(round(cy / (double)p.coarse_step), 0.0, (double)(p.coarse_rows - 1)),
                         p.coarse_rows - 1);
    int ci = cr * p.coarse_columns + cc;
    seeded = p.coarse.has[ci];
    if (!seeded) {
        cand[lane] = p.unseeded[lane];  // 32 candidates
        return 32;
    }
    double seed = p.coarse.depth[ci];
    double far_inverse = 1.0 / p.far_depth, near_inverse = 1.0 / p.near_depth;
    double depth = 0.0, inverse = 0.0;
    if (lane < 13) {
        double inv = clampd_r(1.0 / seed + (double)(lane - 6) * p.inverse_step * 0.5, far_inverse, near_inverse);
        depth = 1.0 / inv;
        inverse = 1.0 / depth;
    }
    unsigned kept = 1u;
    double last = __shfl_sync(full, inverse, 0);
    for (int k = 1; k < 13; ++k) {
        double current = __shfl_sync(full, inverse, k);
        if (fabs(last - current) > p.inverse_step * 0.1) {
            kept |= 1u << k;
            last = current;
        }
    }
    if (lane < 13 && ((kept >> lane) & 1u)) cand[__popc(kept & ((1u << lane) - 1u))] = depth;
    return __popc(kept);
}

// Warp-cooperative: reference patch and every target's tap positions for one
// node at `radius` (warp_stage_patch); geometry from the records.
template <typename TapT>
__device__ inline void warp_stage_node(const DirectParams &p, const DirectSlot<TapT> &d, RefPatch &patch, double cx,
                                       double cy, int radius, const float *spatial, const GeomRec *recs,
                                       const RefPatch *pre) {
    const int lane = threadIdx.x & 31;
    const int V = p.n_targets;
    const unsigned undefined = warp_stage_patch(p.views, p.reference, p.targets, V, cx, cy, radius, spatial, d.rr,
                                                d.wt, d.gh, d.box, patch, p.lattice, pre);
    if (lane < V) {
        geom_from_rec(recs[lane], camera_origin(p.views[p.reference].cam), d.geom[lane]);
        d.geom[lane].taps_ok = ((undefined >> lane) & 1u) ? 0 : 1;
    }
    __syncwarp();
}

// Warp-cooperative listing of the baseline and candidates cand[0..n) over all
// targets. Item i is (candidate i / V - 1, target i % V), candidate -1 being the
// baseline. It settles which items reach the correlation and whether their taps
// are all inside (the fast path), sets the others' scores to None and lists the
// scored ones: fast from the front of d.list, exact from the back of its
// (n + 1) V entries. Every lane returns the two counts.
template <typename TapT>
__device__ inline void warp_direct_list(const DirectParams &p, const DirectSlot<TapT> &d, const RefPatch &patch,
                                        const double *cand, int n, int &n_fast, int &n_exact) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int V = p.n_targets;
    const int total = (n + 1) * V;
    const ViewGeom *geom = d.geom;
    n_fast = 0;
    n_exact = 0;
    for (int base = 0; base < total; base += 32) {
        const int item = base + lane;
        bool scored = false, fast = false;
        if (item < total) {
            const int c = item / V - 1, v = item - (item / V) * V;
            const ViewGeom &g = geom[v];
            double ddx = 0.0, ddy = 0.0;
            bool ok = g.gc_ok;
            if (ok && c >= 0) ok = depth_delta(p.views[p.targets[v]].cam, g, cand[c], ddx, ddy);
            scored = ok && patch.ok && g.taps_ok;
            if (scored) {
                const PlaneRef &plane = p.views[p.targets[v]].luma;
                fast = taps_inside(d.box[v], ddx * 0.5, ddy * 0.5, plane.width, plane.height);
            } else {
                d.items[item] = NAN;
            }
        }
        const unsigned fast_mask = __ballot_sync(full, scored && fast);
        const unsigned exact_mask = __ballot_sync(full, scored && !fast);
        if (scored && fast) d.list[n_fast + __popc(fast_mask & below)] = (unsigned short)item;
        if (scored && !fast) d.list[total - 1 - (n_exact + __popc(exact_mask & below))] = (unsigned short)item;
        n_fast += __popc(fast_mask);
        n_exact += __popc(exact_mask);
    }
}

// The correlation of one listed item (warp_direct_list) into d.items; one thread.
template <typename TapT>
__device__ __forceinline__ void direct_item_score(const DirectParams &p, const DirectSlot<TapT> &d,
                                                  const RefPatch &patch, const double *cand, int item, int taps) {
    const int V = p.n_targets;
    const int c = item / V - 1, v = item - (item / V) * V;
    const DevView &tv = p.views[p.targets[v]];
    double ddx = 0.0, ddy = 0.0;
    if (c >= 0) depth_delta(tv.cam, d.geom[v], cand[c], ddx, ddy);
    float score = NAN, sc;
    if (zncc_any(TargetRef{tv.luma, tv.quads}, d.gh + v * taps, d.box[v], d.wt, patch, taps, ddx, ddy, sc))
        score = sc;
    d.items[item] = score;
}

// aggregate (depth.rs:1761-1770) of the baseline and candidates over the targets into
// d.agg[0..n]; the warp of the node.
template <typename TapT>
__device__ inline void warp_direct_aggregate(const DirectParams &p, const DirectSlot<TapT> &d, int n) {
    const int V = p.n_targets;
    for (int c = threadIdx.x & 31; c <= n; c += 32) {
        float sc[MAX_VIEWS];
        for (int v = 0; v < V; ++v) sc[v] = d.items[c * V + v];
        float a;
        d.agg[c] = aggregate_scores(sc, V, p.minimum_support, p.best_view_count, a) ? a : NAN;
    }
    __syncwarp();
}

// Warp-cooperative scores of the baseline and candidates cand[0..n) over all
// targets, aggregated into d.agg[0..n] (NaN = None): the node's list, scored by
// its own warp.
template <typename TapT>
__device__ inline void warp_direct_scores(const DirectParams &p, const DirectSlot<TapT> &d, const RefPatch &patch,
                                          const double *cand, int n, int radius) {
    const int lane = threadIdx.x & 31;
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    const int total = (n + 1) * p.n_targets;
    int n_fast, n_exact;
    warp_direct_list(p, d, patch, cand, n, n_fast, n_exact);
    __syncwarp();
    const int listed = n_fast + n_exact;
    for (int j = lane; j < listed; j += 32)
        direct_item_score(p, d, patch, cand, j < n_fast ? d.list[j] : d.list[total - 1 - (j - n_fast)], taps);
    __syncwarp();
    warp_direct_aggregate(p, d, n);
}

// A warp per fine node; the CTA holds nodes_per_cta nodes. Each warp lists its
// node's items; the CTA then scores the pooled lists (every node's fast items,
// then every node's exact items), so the lanes of all warps stay busy up to the
// pool's last round instead of each node's; each warp then selects its node.
__global__ void __launch_bounds__(256) direct_depth_kernel(DirectParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patches[8];
    __shared__ int pool[8][3];  // per node: fast count, exact count, list length
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nodes = blockDim.x >> 5;  // == p.nodes_per_cta
    const int node = blockIdx.x * p.nodes_per_cta + slot;
    const bool active = node < p.columns * p.rows;  // whole warps
    const int V = p.n_targets;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const size_t slot_bytes = direct_slot_bytes<float2>(V, taps);
    DirectSlot<float2> d = carve_direct_slot<float2>(smem_raw + (size_t)slot * slot_bytes, V, taps);
    RefPatch &patch = patches[slot];
    const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
    int seeded = 0, n = 0, n_fast = 0, n_exact = 0;
    if (active) {
        n = warp_direct_candidates(p, cx, cy, d.cand, seeded);
        warp_stage_node(p, d, patch, cx, cy, p.radius, p.spatial, p.geometry + (size_t)node * V,
                        p.patches ? p.patches + node : nullptr);
        warp_direct_list(p, d, patch, d.cand, n, n_fast, n_exact);
    }
    if (lane == 0) {
        pool[slot][0] = n_fast;
        pool[slot][1] = n_exact;
        pool[slot][2] = (n + 1) * V;
    }
    __syncthreads();
    int fast_total = 0, pooled = 0;
    for (int k = 0; k < nodes; ++k) {
        fast_total += pool[k][0];
        pooled += pool[k][0] + pool[k][1];
    }
    for (int j = threadIdx.x; j < pooled; j += blockDim.x) {
        // node k and the position of pooled entry j in its list
        int k = 0, at = j;
        if (j < fast_total) {
            while (at >= pool[k][0]) at -= pool[k++][0];
        } else {
            at -= fast_total;
            while (at >= pool[k][1]) at -= pool[k++][1];
            at = pool[k][2] - 1 - at;
        }
        const DirectSlot<float2> dk = carve_direct_slot<float2>(smem_raw + (size_t)k * slot_bytes, V, taps);
        direct_item_score(p, dk, patches[k], dk.cand, dk.list[at], taps);
    }
    __syncthreads();
    if (!active) return;
    warp_direct_aggregate(p, d, n);
    bool seen = false;
    for (int c = lane; c <= n; c += 32) seen |= d.agg[c] == d.agg[c];
    const bool tested = __any_sync(0xffffffffu, seen);
    double depth = 0.0;
    float confidence = 0.0f, improvement = 0.0f;
    int best;
    const bool has = warp_select_direct(d.cand, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0], seeded, p.far_depth,
                                        p.near_depth, p.minimum_score, p.minimum_margin, p.minimum_improvement,
                                        depth, confidence, improvement, best);
    if (lane != 0) return;
    p.tested[node] = tested;
    p.guidance[node] = patch.centre;  // reference_guidance (depth.rs:1824-1832)
    p.out.has[node] = has;
    p.out.depth[node] = has ? depth : NAN;
    p.out.confidence[node] = has ? confidence : 0.0f;
    p.out.improvement[node] = has ? improvement : 0.0f;
    p.out.regularized[node] = 0;
    if (!has && best >= 0 && d.agg[1 + best] == d.agg[1 + best] && d.agg[1 + best] >= MINIMUM_REGULARIZED_SCORE) {
        int first = best >= 3 ? best - 3 : 0;
        int last = best + 3 < n - 1 ? best + 3 : n - 1;
        int k = atomicAdd(p.wide_count, 1);
        p.wide_list[k] = make_int4(node, first, last, seeded);
    }
}

// The wide-radius retry (depth.rs:803-846) for the listed nodes; a warp per
// entry, persistent over the list. Its 225-tap positions are kept as f32 g,
// which halves their shared memory and lets more warps stay resident.
__global__ void __launch_bounds__(256) direct_wide_kernel(DirectParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patches[8];
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    const int V = p.n_targets;
    const int taps = (2 * p.wide_radius + 1) * (2 * p.wide_radius + 1);
    DirectSlot<float2> d =
        carve_direct_slot<float2>(smem_raw + (size_t)slot * direct_slot_bytes<float2>(V, taps), V, taps);
    RefPatch &patch = patches[slot];
    const int count = *p.wide_count;
    for (int e = blockIdx.x * warps + slot; e < count; e += gridDim.x * warps) {
        int4 entry = p.wide_list[e];
        const int node = entry.x, first = entry.y, last = entry.z;
        const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
        int seeded;
        warp_direct_candidates(p, cx, cy, d.cand, seeded);
        warp_stage_node(p, d, patch, cx, cy, p.wide_radius, p.spatial_wide, p.geometry + (size_t)node * V, nullptr);
        const int n = last - first + 1;
        warp_direct_scores(p, d, patch, d.cand + first, n, p.wide_radius);
        double depth = 0.0;
        float confidence = 0.0f, improvement = 0.0f;
        int best;
        const bool has = warp_select_direct(d.cand + first, d.agg + 1, n, d.agg[0] == d.agg[0], d.agg[0],
                                            entry.w != 0, p.far_depth, p.near_depth, p.minimum_score,
                                            p.minimum_margin, p.minimum_improvement, depth, confidence,
                                            improvement, best);
        if (has && lane == 0) {
            p.out.has[node] = 1;
            p.out.depth[node] = depth;
            p.out.confidence[node] = confidence;
            p.out.improvement[node] = improvement;
        }
        __syncwarp();
    }
}

}  // namespace chiaro
