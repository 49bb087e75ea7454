// cost.cuh — build_cost_volume (crates/chiaro-fusion/src/depth.rs:1187-1277).
//
// One CTA per coarse node. The CTA stages the node's reference patch, every
// target's tap positions and the label-independent geometry in shared memory,
// then each thread evaluates one depth label across all targets, aggregates
// the views (depth.rs:1761-1770) and writes the label-minor score and cost rows
// (node-major [N][D], as the reference lays them out).
#pragma once

#include "zncc.cuh"

namespace chiaro {

struct CostParams {
    const DevView *views;       // all modules
    int reference;              // reference module
    int n_targets;              // scored modules (accepted, calibrated, not the reference)
    int targets[MAX_VIEWS];
    int columns, rows, step;    // coarse grid
    int labels;                 // D = planes + 1
    const double *label_depth;  // [D], label 0 unused (the global warp)
    const float *spatial;       // [(2r+1)^2] spatial weights
    const GeomRec *geometry;    // [node][target]
    int radius;
    int minimum_support, best_view_count;
    float *scores, *costs, *guidance;
    uint8_t *tested;
};

// Dynamic shared memory of a node CTA: cameras, view geometry, reference
// patch arrays and per-view tap positions.
struct NodeSmem {
    DevCamera *cams;  // [0] reference, [1 + v] targets
    ViewGeom *geom;   // [V]
    TapBox *box;      // [V]
    float *r, *w, *wr;  // [T]
    double2 *gh;      // [V][T] g/2 of the tap positions
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) / 16 * 16; }

__host__ __device__ inline size_t node_smem_bytes(int V, int taps) {
    return align16((V + 1) * sizeof(DevCamera)) + align16(V * sizeof(ViewGeom)) + align16(V * sizeof(TapBox)) +
           align16(3 * taps * sizeof(float)) + (size_t)V * taps * sizeof(double2);
}

__device__ inline NodeSmem carve_node_smem(unsigned char *base, int V, int taps) {
    NodeSmem s;
    size_t o = 0;
    s.cams = reinterpret_cast<DevCamera *>(base + o);
    o += align16((V + 1) * sizeof(DevCamera));
    s.geom = reinterpret_cast<ViewGeom *>(base + o);
    o += align16(V * sizeof(ViewGeom));
    s.box = reinterpret_cast<TapBox *>(base + o);
    o += align16(V * sizeof(TapBox));
    s.r = reinterpret_cast<float *>(base + o);
    s.w = s.r + taps;
    s.wr = s.w + taps;
    o += align16(3 * taps * sizeof(float));
    s.gh = reinterpret_cast<double2 *>(base + o);
    return s;
}

// Copy the reference camera and the target cameras into shared memory.
__device__ inline void load_cameras(DevCamera *cams, const DevView *views, int reference, const int *targets, int V) {
    const int words = sizeof(DevCamera) / 8;
    for (int i = threadIdx.x; i < (V + 1) * words; i += blockDim.x) {
        int c = i / words, k = i % words;
        const DevCamera &src = c == 0 ? views[reference].cam : views[targets[c - 1]].cam;
        reinterpret_cast<uint64_t *>(&cams[c])[k] = reinterpret_cast<const uint64_t *>(&src)[k];
    }
}

// Stage reference patch, tap positions and (from the precomputed records
// `recs[0..V)`, when given) the view geometry for the node at (cx, cy) at the
// given radius. Without records the geometry already in s.geom is kept and
// only taps_ok is recomputed. Ends with __syncthreads().
__device__ inline void stage_node(const NodeSmem &s, RefPatch &patch, const DevView *views, int reference,
                                  const int *targets, int V, double cx, double cy, int radius, const float *spatial,
                                  const GeomRec *recs) {
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    for (int v = threadIdx.x; v < V; v += blockDim.x) {
        if (recs) geom_from_rec(recs[v], camera_origin(s.cams[0]), s.geom[v]);
        s.geom[v].taps_ok = 1;
    }
    ref_patch_setup(views[reference].luma, cx, cy, radius, spatial, s.r, s.w, s.wr, patch);
    for (int v = 0; v < V; ++v)
        tap_positions(views[targets[v]].warp, cx, cy, radius, s.gh + v * taps, s.geom[v]);
    __syncthreads();
    // one warp per view computes its tap box
    for (int v = threadIdx.x >> 5; v < V; v += blockDim.x >> 5) {
        TapBox b = warp_tap_box(s.gh + v * taps, taps);
        if ((threadIdx.x & 31) == 0) s.box[v] = b;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) cost_volume_kernel(CostParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patch;
    const int node = blockIdx.x;
    const int column = node % p.columns, row = node / p.columns;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const int V = p.n_targets;
    NodeSmem s = carve_node_smem(smem_raw, V, taps);
    const double cx = (double)(column * p.step), cy = (double)(row * p.step);

    load_cameras(s.cams, p.views, p.reference, p.targets, V);
    __syncthreads();
    stage_node(s, patch, p.views, p.reference, p.targets, V, cx, cy, p.radius, p.spatial,
               p.geometry + (size_t)node * V);

    int any_finite = 0;
    for (int label = threadIdx.x; label < p.labels; label += blockDim.x) {
        float sc[MAX_VIEWS];
        for (int v = 0; v < V; ++v) {
            sc[v] = NAN;
            const ViewGeom &g = s.geom[v];
            double ddx = 0.0, ddy = 0.0;
            if (!g.gc_ok) continue;
            if (label > 0 && !depth_delta(s.cams[1 + v], g, p.label_depth[label], ddx, ddy)) continue;
            if (!patch.ok || !g.taps_ok) continue;
            const DevView &tv = p.views[p.targets[v]];
            float score;
            if (zncc_any(TargetRef{tv.luma, tv.pairs}, s.gh + v * taps, s.box[v], s.w, s.wr, patch, taps, ddx, ddy,
                         score))
                sc[v] = score;
        }
        float agg;
        float score = aggregate_scores(sc, V, p.minimum_support, p.best_view_count, agg) ? agg : NAN;
        float cost;
        if (isfinite(score)) {
            any_finite = 1;
            float near_prior = label == 0 ? 0.0f : NEAR_DEPTH_PRIOR * (float)(label - 1) / (float)(p.labels - 2);
            cost = clampf_r(1.0f - score, 0.0f, 2.0f) + near_prior;
        } else {
            cost = MISSING_COST;
        }
        size_t o = (size_t)node * p.labels + label;
        p.scores[o] = score;
        p.costs[o] = cost;
    }
    // tested: any finite score; p.tested starts zeroed, one store per warp that saw one
    if (__ballot_sync(0xffffffffu, any_finite) && (threadIdx.x & 31) == 0) p.tested[node] = 1;
    if (threadIdx.x == 0) p.guidance[node] = patch.centre;  // reference_guidance (depth.rs:1824-1832)
}

}  // namespace chiaro
