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

struct TapBox {
    double xmin, xmax, ymin, ymax;  // of g/2 over the taps
};

__device__ __forceinline__ void tap_offset(int t, int radius, int &dx, int &dy) {
    int side = 2 * radius + 1;
    dy = t / side - radius;
    dx = t % side - radius;
}

// The same with the row split by SmallDiv(2 radius + 1) (one multiply per tap).
__device__ __forceinline__ void tap_offset(int t, int radius, const SmallDiv &side, int &dx, int &dy) {
    const int row = side.quotient(t);
    dy = row - radius;
    dx = t - row * (int)side.d - radius;
}

// Tap positions are kept either as g/2 in f64 (double2: one 16-byte load per
// tap on the fast path) or as g in f32 (float2: half the shared memory, halved
// to f64 at use). g is f32 and halving is exact in f64, so both give the same
// bits everywhere.
__device__ __forceinline__ double2 tap_half(const double2 &v) { return v; }
__device__ __forceinline__ double2 tap_half(const float2 &v) {
    return make_double2((double)v.x * 0.5, (double)v.y * 0.5);
}
__device__ __forceinline__ float2 tap_g(const double2 &v) {
    return make_float2((float)(v.x * 2.0), (float)(v.y * 2.0));
}
__device__ __forceinline__ float2 tap_g(const float2 &v) { return v; }
__device__ __forceinline__ void store_tap(double2 &d, float qx, float qy) {
    d = make_double2((double)qx * 0.5, (double)qy * 0.5);
}
__device__ __forceinline__ void store_tap(float2 &d, float qx, float qy) { d = make_float2(qx, qy); }

// Bounding box of g/2 over one target's taps, computed by an aligned group of
// eight lanes (min and max are exact, so the reduction order does not matter).
// Every lane of the warp calls it; the groups reduce with shuffles.
template <typename TapT>
__device__ inline TapBox group8_tap_box(const TapT *gh, int taps) {
    const double2 g0 = tap_half(gh[0]);
    TapBox b{g0.x, g0.x, g0.y, g0.y};
    for (int t = threadIdx.x & 7; t < taps; t += 8) {
        const double2 g = tap_half(gh[t]);
        b.xmin = fmin(b.xmin, g.x);
        b.xmax = fmax(b.xmax, g.x);
        b.ymin = fmin(b.ymin, g.y);
        b.ymax = fmax(b.ymax, g.y);
    }
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {
        b.xmin = fmin(b.xmin, __shfl_xor_sync(0xffffffffu, b.xmin, off));
        b.xmax = fmax(b.xmax, __shfl_xor_sync(0xffffffffu, b.xmax, off));
        b.ymin = fmin(b.ymin, __shfl_xor_sync(0xffffffffu, b.ymin, off));
        b.ymax = fmax(b.ymax, __shfl_xor_sync(0xffffffffu, b.ymax, off));
    }
    return b;
}

// A sequential f32 sum in tap order of a[t * stride] (the reference's three
// patch sums add w, w r and (w r) r tap by tap).
__device__ inline float sequential_sum(const float *a, int stride, int taps) {
    float sum = 0.0f;
    for (int t = 0; t < taps; ++t) sum += a[t * stride];
    return sum;
}

// The same sum unrolled by nine (the same order of additions), for the cost volume, whose
// three lanes summing hold up the node's CTA.
__device__ inline float sequential_sum_unrolled(const float *a, int stride, int taps) {
    float sum = 0.0f;
#pragma unroll 9
    for (int t = 0; t < taps; ++t) sum += a[t * stride];
    return sum;
}

__device__ inline void store_reference_sum(RefPatch &patch, int which, float sum) {
    if (which == 0)
        patch.count = sum;
    else if (which == 1)
        patch.sum_r = sum;
    else
        patch.sum_rr = sum;
}

// Tap lattice. A node of a grid with an even step sits at even pixel coordinates and its
// taps lie 2 px apart, so every tap of every node is a point (px, py) of the even lattice.
// The reference sample and each target's global warp at a tap depend on (px, py) alone,
// so they are evaluated once per lattice point and call (tap_lattice_kernel) instead of
// once per node and tap; a node reads them back with plain loads. Plane 0 holds the
// reference sample (plane_sample's value, 1 if it is Some else 0; the value is 0 when
// None, as the staging's initial value), plane 1 + v target v's Warp::map (NaN for None).
// Point (i, j) is the pixel (2 (i - margin), 2 (j - margin)). planes == nullptr: none.
struct TapLattice {
    const float2 *planes;  // [(V + 1)][rows][columns]
    int columns, rows, margin;
    __device__ __forceinline__ size_t plane_size() const { return (size_t)columns * rows; }
    // the lattice point of the even pixel (cx, cy)
    __device__ __forceinline__ size_t index(double cx, double cy) const {
        return (size_t)((int)(cy * 0.5) + margin) * columns + ((int)(cx * 0.5) + margin);
    }
};

struct LatticeParams {
    const DevView *views;
    int reference, n_targets;
    int targets[MAX_VIEWS];
    int columns, rows, margin;
    float2 *out;
};

// A thread per lattice point: the reference sample and every target's global warp there,
// with the staging's own expressions (warp_stage_patch).
__global__ void __launch_bounds__(256) tap_lattice_kernel(LatticeParams p) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long size = (long)p.columns * p.rows;
    if (i >= size) return;
    const double px = (double)(2 * ((int)(i % p.columns) - p.margin));
    const double py = (double)(2 * ((int)(i / p.columns) - p.margin));
    float value = 0.0f;
    const bool ok =
        plane_sample(p.views[p.reference].luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value);
    p.out[i] = make_float2(value, ok ? 1.0f : 0.0f);
    for (int v = 0; v < p.n_targets; ++v) {
        float qx = 0.0f, qy = 0.0f;
        const bool defined = warp_map(p.views[p.targets[v]].warp, (float)px, (float)py, qx, qy);
        p.out[(size_t)(v + 1) * size + i] = defined ? make_float2(qx, qy) : make_float2(NAN, NAN);
    }
}

// Warp-cooperative staging of one node at (cx, cy) and `radius`: the
// reference patch ((w, w r) and (w r) r per tap, the three sums, the energy and the
// centre sample) and, for each target, g/2 of every tap and their box. Returns
// on every lane the mask of targets with a tap where the global warp is None
// (bit v); `patch` is written by lanes 0-2 and valid after the trailing
// __syncwarp(). `pre`: the node's patch from patch_sums_kernel at this radius, or
// nullptr; lane 0 copies it instead of the three lanes summing the taps.
template <typename TapT>
__device__ inline unsigned warp_stage_patch(const DevView *views, int reference, const int *targets, int V,
                                            double cx, double cy, int radius, const float *spatial, float *rr,
                                            float2 *wt, TapT *gh, TapBox *box, RefPatch &patch,
                                            const TapLattice &lattice, const RefPatch *pre) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int taps = (2 * radius + 1) * (2 * radius + 1);
    const DevView &rv = views[reference];
    float centre = 0.0f;
    bool centre_ok;
    const size_t at0 = lattice.planes ? lattice.index(cx, cy) : 0;
    if (lattice.planes) {
        const float2 c = __ldg(lattice.planes + at0);
        centre = c.x;
        centre_ok = c.y != 0.0f;
    } else {
        centre_ok = plane_sample(rv.luma, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
    }
    bool sampled = true;
    unsigned undefined = 0u;
    for (int t = lane; t < taps; t += 32) {
        int dx, dy;
        tap_offset(t, radius, dx, dy);
        float value = 0.0f;
        if (lattice.planes) {
            const size_t at = at0 + (ptrdiff_t)dy * lattice.columns + dx;
            const float2 r = __ldg(lattice.planes + at);
            value = r.x;
            sampled &= r.y != 0.0f;
            for (int v = 0; v < V; ++v) {
                const float2 q = __ldg(lattice.planes + (size_t)(v + 1) * lattice.plane_size() + at);
                if (q.x != q.x) undefined |= 1u << v;
                store_tap(gh[v * taps + t], q.x, q.y);
            }
        } else {
            double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
            sampled &= plane_sample(rv.luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value);
            for (int v = 0; v < V; ++v) {
                float qx = 0.0f, qy = 0.0f;
                if (!warp_map(views[targets[v]].warp, (float)px, (float)py, qx, qy)) undefined |= 1u << v;
                store_tap(gh[v * taps + t], qx, qy);
            }
        }
        float weight = spatial[t] * exp_f32(-1.2f * fabsf(value - centre));
        float weighted = weight * value;
        wt[t] = make_float2(weight, weighted);
        rr[t] = weighted * value;
    }
    undefined = __reduce_or_sync(full, undefined);
    sampled = __all_sync(full, sampled);
    __syncwarp();
    for (int vb = 0; vb < V; vb += 4) {  // eight lanes per target
        const int v = vb + (lane >> 3);
        TapBox b = group8_tap_box(gh + (v < V ? v : V - 1) * taps, taps);
        if ((lane & 7) == 0 && v < V) box[v] = b;
    }
    if (pre) {
        if (lane == 0) patch = *pre;
    } else {
        if (lane < 3)
            store_reference_sum(patch, lane,
                                lane == 2 ? sequential_sum(rr, 1, taps)
                                          : sequential_sum(reinterpret_cast<const float *>(wt) + lane, 2, taps));
        __syncwarp();
        if (lane == 0) {
            patch.centre = centre;
            patch.ok = centre_ok && sampled;
            patch.ref_energy = patch.sum_rr - patch.sum_r * patch.sum_r / patch.count;
        }
    }
    __syncwarp();
    return undefined;
}

// The reference patch of every node of a step-spaced grid at `radius`, a thread per node:
// what warp_stage_patch computes for it (the taps' weights w = spatial * exp(-1.2 |r -
// centre|), the sums of w, w r and (w r) r in tap order, the energy, the centre sample and
// whether the centre and every tap were sampled), with the same expressions in the same
// order, so the same bits. The direct pass and the decisions read it instead of summing 81
// or more taps in three lanes of a warp.
struct PatchParams {
    const DevView *views;
    int reference;
    int columns, rows, step, radius;
    const float *spatial;
    TapLattice lattice;  // of this grid, or planes == nullptr
    RefPatch *out;
};

__global__ void __launch_bounds__(256) patch_sums_kernel(PatchParams p) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)p.columns * p.rows) return;
    const double cx = (double)((int)(i % p.columns) * p.step), cy = (double)((int)(i / p.columns) * p.step);
    const DevView &rv = p.views[p.reference];
    const TapLattice &lattice = p.lattice;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    float centre = 0.0f;
    bool centre_ok;
    const size_t at0 = lattice.planes ? lattice.index(cx, cy) : 0;
    if (lattice.planes) {
        const float2 c = __ldg(lattice.planes + at0);
        centre = c.x;
        centre_ok = c.y != 0.0f;
    } else {
        centre_ok = plane_sample(rv.luma, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
    }
    bool sampled = true;
    float count = 0.0f, sum_r = 0.0f, sum_rr = 0.0f;
    for (int t = 0; t < taps; ++t) {
        int dx, dy;
        tap_offset(t, p.radius, dx, dy);
        float value = 0.0f;
        if (lattice.planes) {
            const float2 r = __ldg(lattice.planes + at0 + (ptrdiff_t)dy * lattice.columns + dx);
            value = r.x;
            sampled &= r.y != 0.0f;
        } else {
            double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
            sampled &= plane_sample(rv.luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value);
        }
        float weight = __ldg(p.spatial + t) * exp_f32(-1.2f * fabsf(value - centre));
        float weighted = weight * value;
        count += weight;
        sum_r += weighted;
        sum_rr += weighted * value;
    }
    RefPatch r;
    r.count = count;
    r.sum_r = sum_r;
    r.sum_rr = sum_rr;
    r.ref_energy = sum_rr - sum_r * sum_r / count;
    r.centre = centre;
    r.ok = centre_ok && sampled;
    p.out[i] = r;
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
template <typename TapT>
__device__ __forceinline__ bool zncc_score(const PlaneRef &target, const TapT *gh, const float2 *wt,
                                           const RefPatch &patch, int taps, double ddx, double ddy, float &score) {
    float st = 0.0f, stt = 0.0f, srt = 0.0f;
    for (int t = 0; t < taps; ++t) {
        const float2 g = tap_g(gh[t]);  // the tap's global-warp position
        double qx = (double)g.x + ddx;
        double qy = (double)g.y + ddy;
        float tv;
        if (!plane_sample(target, (float)((qx - 0.5) * 0.5), (float)((qy - 0.5) * 0.5), tv)) return false;
        const float2 weights = wt[t];
        float wv = weights.x * tv;
        st += wv;
        stt += wv * tv;
        srt += weights.y * tv;
    }
    float covariance = srt - patch.sum_r * st / patch.count;
    float target_energy = stt - st * st / patch.count;
    float denominator = sqrtf(fmaxf(patch.ref_energy, 0.0f) * fmaxf(target_energy, 0.0f));
    if (!(denominator > 1.0e-6f)) return false;
    score = clampf_r(covariance / denominator, -1.0f, 1.0f);
    return true;
}

// ---- fast path ---------------------------------------------------------------------
// The reference computes each target sample coordinate as
//   x = (f32)(((f64)g + d - 0.5) * 0.5)
// with two f64 roundings. Multiplying by 0.5 is exact and commutes with
// rounding, so the same bits come from x = (f32)((g/2 + d/2) - 0.25), where g/2
// is stored per tap (TapHalf) and d/2 is computed once per hypothesis. The
// coordinate is monotone in g, so the bounding box of the taps' g decides for
// every tap at once whether all samples fall strictly inside [0, w-1) x [0, h-1);
// inside, the reference's bounds checks and edge clamps cannot trigger and the
// bilinear fetch reads the four neighbours from a quad plane with one 16-byte
// load.

// Quad plane: the quad of (x, y) is (L[y][x], L[y][x1], L[y1][x], L[y1][x1]) with
// x1 = min(x + 1, w - 1) and y1 = min(y + 1, h - 1), pair-interleaved: the quads of rows
// 2k and 2k + 1 alternate, so (x, y) sits at (y >> 1) * stride + 2 x + (y & 1) with
// stride = 2 * roundup(w, 4), and each 128-byte line holds a 4 x 2 block of quads. The
// taps of neighbouring labels spread along the epipolar line in any direction; against
// row-major quads (8 x 1 per line) a 4 x 2 block keeps more of a quarter-warp's gathers
// in one line.
__host__ __device__ inline int quad_pair_stride(int width) { return 2 * ((width + 3) / 4 * 4); }

__device__ __forceinline__ size_t quad_index(int x, int y, int stride) {
    return (size_t)(y >> 1) * stride + 2 * x + (y & 1);
}

__global__ void quad_plane_kernel(const float *__restrict__ plane, int width, int height, int stride,
                                  float4 *quads) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)width * height) return;
    int x = (int)(i % width), y = (int)(i / width);
    long right = x + 1 < width ? 1 : 0, down = y + 1 < height ? width : 0;
    quads[quad_index(x, y, stride)] = make_float4(plane[i], plane[i + right], plane[i + down], plane[i + down + right]);
}

struct TargetRef {
    PlaneRef plane;
    const float4 *quads;  // quad plane
};

// True when every tap at displacement (hdx, hdy) = (ddx/2, ddy/2) samples
// strictly inside the plane.
__device__ __forceinline__ bool taps_inside(const TapBox &box, double hdx, double hdy, int width, int height) {
    float x0 = (float)((box.xmin + hdx) - 0.25), x1 = (float)((box.xmax + hdx) - 0.25);
    float y0 = (float)((box.ymin + hdy) - 0.25), y1 = (float)((box.ymax + hdy) - 0.25);
    // width, height < 2^22 (checked on the host), so inside also means < 2^22
    return x0 >= 0.0f && y0 >= 0.0f && x1 < (float)(width - 1) && y1 < (float)(height - 1);
}

// warped_patch_zncc's hypothesis-dependent part for taps known to be inside
// (see taps_inside). gh holds g/2 per tap.
template <typename TapT>
__device__ __forceinline__ float zncc_inside(const float4 *__restrict__ quads, int stride, const TapT *gh,
                                             const float2 *wt, const RefPatch &patch, int taps,
                                             double hdx, double hdy, bool &ok) {
    float st = 0.0f, stt = 0.0f, srt = 0.0f;
#pragma unroll 9
    for (int t = 0; t < taps; ++t) {
        const double2 g = tap_half(gh[t]);
        float x = (float)((g.x + hdx) - 0.25);
        float y = (float)((g.y + hdy) - 0.25);
        int ix, iy;
        float tx = floor_frac_small(x, ix), ty = floor_frac_small(y, iy);
        const float4 q = __ldg(quads + quad_index(ix, iy, stride));
        float top = q.x * (1.0f - tx) + q.y * tx;
        float bottom = q.z * (1.0f - tx) + q.w * tx;
        float tv = top * (1.0f - ty) + bottom * ty;
        const float2 weights = wt[t];
        float wv = weights.x * tv;
        st += wv;
        stt += wv * tv;
        srt += weights.y * tv;
    }
    float covariance = srt - patch.sum_r * st / patch.count;
    float target_energy = stt - st * st / patch.count;
    float denominator = sqrtf(fmaxf(patch.ref_energy, 0.0f) * fmaxf(target_energy, 0.0f));
    ok = denominator > 1.0e-6f;
    return clampf_r(covariance / denominator, -1.0f, 1.0f);
}

// Either path, bit-identical to warped_patch_zncc: fast when the box is inside,
// exact per-tap checks otherwise. gh: g/2 per tap.
template <typename TapT>
__device__ __forceinline__ bool zncc_any(const TargetRef &target, const TapT *gh, const TapBox &box, const float2 *wt, const RefPatch &patch,
                                         int taps, double ddx, double ddy, float &score) {
    double hdx = ddx * 0.5, hdy = ddy * 0.5;
    if (taps_inside(box, hdx, hdy, target.plane.width, target.plane.height)) {
        bool ok;
        score = zncc_inside(target.quads, quad_pair_stride(target.plane.width), gh, wt, patch, taps, hdx, hdy, ok);
        return ok;
    }
    return zncc_score(target.plane, gh, wt, patch, taps, ddx, ddy, score);
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
