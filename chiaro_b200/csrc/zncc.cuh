// zncc.cuh — the bilateral-weighted ZNCC of warped_patch_zncc
// (crates/chiaro-fusion/src/depth.rs:1772-1822) split into its
// hypothesis-independent and hypothesis-dependent parts, plus the per-view
// geometry of score_one_view / map_at_depth (depth.rs:1593-1627, 1738-1759).
//
// For one node the reference samples, per tap, the reference value r_i, the
// weight w_i = spatial_i * exp(-1.2 |r_i - centre|) and the global-warp
// position g_i of every target; only the target samples depend on the depth
// hypothesis. The reference-only sums (sum w, sum w r, sum w r r) are
// sequential sums over the taps in the reference's order, so computing them
// once per node gives the same bits as recomputing them per hypothesis. The
// three target sums keep their own sequential order in zncc_score().
#pragma once

#include "common.cuh"

namespace chiaro {

struct RefPatch {
    float count, sum_r, sum_rr;
    float ref_energy;  // sum_rr - sum_r * sum_r / count  (depth.rs:1818)
    float centre;      // centre reference sample
    int ok;            // centre and every reference tap sampled
};

// Per (node, target view) geometry, label-independent.
struct ViewGeom {
    double ox, oy, oz, dx, dy, dz;  // reference ray through the corrected reference pixel
    float gcx, gcy;                 // global warp at the node centre
    int gc_ok;                      // global.map(centre) is Some
    int ray_ok;                     // corrected reference pixel is Some
    int taps_ok;                    // global.map is Some at every tap
    int pad;
};

__device__ __forceinline__ void tap_offset(int t, int radius, int &dx, int &dy) {
    int side = 2 * radius + 1;
    dy = t / side - radius;
    dx = t % side - radius;
}

// Reference patch of the node at (cx, cy): r[], w[], wr[] and the sums.
// Block-cooperative; ends with __syncthreads().
__device__ void ref_patch_setup(const PlaneRef &ref, double cx, double cy, int radius, const float *spatial,
                                float *r, float *w, float *wr, RefPatch &patch) {
    int taps = (2 * radius + 1) * (2 * radius + 1);
    float centre = 0.0f;
    bool centre_ok = plane_sample(ref, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
    if (threadIdx.x == 0) {
        patch.ok = centre_ok ? 1 : 0;
        patch.centre = centre;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < taps; t += blockDim.x) {
        int dx, dy;
        tap_offset(t, radius, dx, dy);
        double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
        float rv = 0.0f;
        if (!plane_sample(ref, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), rv)) patch.ok = 0;
        float weight = spatial[t] * exp_f32(-1.2f * fabsf(rv - centre));
        r[t] = rv;
        w[t] = weight;
        wr[t] = weight * rv;
    }
    __syncthreads();
    // Three independent sequential sums: threads 0, 32 and 64 when the block
    // has three warps, otherwise all on thread 0.
    bool three = blockDim.x >= 96;
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int t = 0; t < taps; ++t) s += w[t];
        patch.count = s;
    }
    if ((three && threadIdx.x == 32) || (!three && threadIdx.x == 0)) {
        float s = 0.0f;
        for (int t = 0; t < taps; ++t) s += wr[t];
        patch.sum_r = s;
    }
    if ((three && threadIdx.x == 64) || (!three && threadIdx.x == 0)) {
        float s = 0.0f;
        for (int t = 0; t < taps; ++t) s += wr[t] * r[t];
        patch.sum_rr = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) patch.ref_energy = patch.sum_rr - patch.sum_r * patch.sum_r / patch.count;
    __syncthreads();
}

// Global-warp positions of every tap for one target warp; clears
// geom.taps_ok when one is undefined. Block-cooperative, no trailing sync.
__device__ void tap_positions(const WarpRef &warp, double cx, double cy, int radius, float2 *gq, ViewGeom &geom) {
    int taps = (2 * radius + 1) * (2 * radius + 1);
    for (int t = threadIdx.x; t < taps; t += blockDim.x) {
        int dx, dy;
        tap_offset(t, radius, dx, dy);
        double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
        float qx = 0.0f, qy = 0.0f;
        if (!warp_map(warp, (float)px, (float)py, qx, qy)) geom.taps_ok = 0;
        gq[t] = make_float2(qx, qy);
    }
}

// Label-independent geometry of map_at_depth for one (node, target); one thread.
__device__ void view_geometry(const DevCamera &rc, const DevCamera &tc, const WarpRef &warp, double cx, double cy,
                              ViewGeom &g) {
    float gx = 0.0f, gy = 0.0f;
    g.gc_ok = warp_map(warp, (float)cx, (float)cy, gx, gy) ? 1 : 0;
    g.gcx = gx;
    g.gcy = gy;
    g.ray_ok = 0;
    g.taps_ok = 1;
    if (!g.gc_ok) return;
    D3 o1, d1;
    pixel_to_ray(tc, (double)gx, (double)gy, o1, d1);
    double crx, cry;
    if (!project(rc, along(o1, d1, INFINITY_DEPTH), crx, cry)) return;
    D3 o2, d2;
    pixel_to_ray(rc, crx, cry, o2, d2);
    g.ox = o2.x;
    g.oy = o2.y;
    g.oz = o2.z;
    g.dx = d2.x;
    g.dy = d2.y;
    g.dz = d2.z;
    g.ray_ok = 1;
}

// Compact per (node, target) geometry kept in HBM between kernels. pixel_to_ray
// returns the camera centre as the origin for both pose kinds (geometry.rs:152-164),
// so only the direction varies per node. gcx is NaN when global.map(centre) is
// None, dx is NaN when the corrected reference pixel is None.
struct GeomRec {
    double dx, dy, dz;
    float gcx, gcy;
};

__device__ __forceinline__ D3 camera_origin(const DevCamera &c) {
    return c.pose_kind == 0 ? D3{c.center[0], c.center[1], c.center[2]}
                            : D3{c.virtual_center[0], c.virtual_center[1], c.virtual_center[2]};
}

__device__ __forceinline__ void geom_from_rec(const GeomRec &rec, const D3 &origin, ViewGeom &g) {
    g.gcx = rec.gcx;
    g.gcy = rec.gcy;
    g.gc_ok = !(rec.gcx != rec.gcx);
    g.ray_ok = g.gc_ok && !(rec.dx != rec.dx);
    g.ox = origin.x;
    g.oy = origin.y;
    g.oz = origin.z;
    g.dx = rec.dx;
    g.dy = rec.dy;
    g.dz = rec.dz;
    g.taps_ok = 1;
}

// One thread per (node, target) of a step-spaced grid: the label-independent
// part of map_at_depth (depth.rs:1745-1756).
struct GeometryParams {
    const DevView *views;
    int reference, n_targets;
    int targets[MAX_VIEWS];
    int columns, rows, step;
    GeomRec *out;  // [node][target]
};

__global__ void __launch_bounds__(128) view_geometry_kernel(GeometryParams p) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = (long)p.columns * p.rows * p.n_targets;
    if (i >= total) return;
    int v = (int)(i % p.n_targets);
    int node = (int)(i / p.n_targets);
    double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
    const DevView &tv = p.views[p.targets[v]];
    ViewGeom g;
    view_geometry(p.views[p.reference].cam, tv.cam, tv.warp, cx, cy, g);
    GeomRec rec;
    rec.gcx = g.gc_ok ? g.gcx : NAN;
    rec.gcy = g.gc_ok ? g.gcy : NAN;
    rec.dx = g.ray_ok ? g.dx : NAN;
    rec.dy = g.ray_ok ? g.dy : NAN;
    rec.dz = g.ray_ok ? g.dz : NAN;
    p.out[i] = rec;
}

// map_at_depth's last step and score_one_view's displacement check: the
// image displacement of a finite depth relative to the global centre. Returns
// false for None (depth.rs:1604-1614).
__device__ __forceinline__ bool depth_delta(const DevCamera &tc, const ViewGeom &g, double depth, double &ddx,
                                            double &ddy) {
    if (!g.gc_ok || !g.ray_ok) return false;
    double qx, qy;
    if (!project(tc, along({g.ox, g.oy, g.oz}, {g.dx, g.dy, g.dz}, depth), qx, qy)) return false;
    if (!(isfinite(qx) && isfinite(qy))) return false;
    ddx = qx - (double)g.gcx;
    ddy = qy - (double)g.gcy;
    return !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0);
}

// Hypothesis-dependent part of warped_patch_zncc: sample the target at every
// tap shifted by (ddx, ddy) and finish the correlation. False for None.
__device__ __forceinline__ bool zncc_score(const PlaneRef &target, const float2 *gq, const float *w, const float *wr,
                                           const RefPatch &patch, int taps, double ddx, double ddy, float &score) {
    float st = 0.0f, stt = 0.0f, srt = 0.0f;
    for (int t = 0; t < taps; ++t) {
        float2 g = gq[t];
        double qx = (double)g.x + ddx;
        double qy = (double)g.y + ddy;
        float tv;
        if (!plane_sample(target, (float)((qx - 0.5) * 0.5), (float)((qy - 0.5) * 0.5), tv)) return false;
        float wt = w[t] * tv;
        st += wt;
        stt += wt * tv;
        srt += wr[t] * tv;
    }
    float covariance = srt - patch.sum_r * st / patch.count;
    float target_energy = stt - st * st / patch.count;
    float denominator = sqrtf(fmaxf(patch.ref_energy, 0.0f) * fmaxf(target_energy, 0.0f));
    if (!(denominator > 1.0e-6f)) return false;
    score = clampf_r(covariance / denominator, -1.0f, 1.0f);
    return true;
}

// aggregate (depth.rs:1761-1770) over up to MAX_VIEWS scores (NaN = None).
__device__ __forceinline__ bool aggregate_scores(float *s, int n, int minimum_support, int best_view_count,
                                                 float &out) {
    // compact the Some values
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (!(s[i] != s[i])) s[m++] = s[i];
    if (m < minimum_support) return false;
    // stable insertion sort, descending by total order
    for (int i = 1; i < m; ++i) {
        float v = s[i];
        int j = i - 1;
        while (j >= 0 && total_key(s[j]) < total_key(v)) {
            s[j + 1] = s[j];
            --j;
        }
        s[j + 1] = v;
    }
    int k = best_view_count < m ? best_view_count : m;
    if (k < minimum_support) return false;
    float sum = -0.0f;
    for (int i = 0; i < k; ++i) sum += s[i];
    out = sum / (float)k;
    return true;
}

}  // namespace chiaro
