// common.cuh — building blocks shared by every kernel of the depth stage.
//
// Everything here is compiled with -fmad=false (device) and
// -ffp-contract=off (host check build): the reference (Rust) never fuses
// a*b+c, so every product and sum rounds separately here too, in the
// reference's operand order. With that, each routine returns the same bits as
// the Rust function it restates (cited per routine). Functions are
// host+device so the CPU test build can check them directly.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define CH_HD __host__ __device__ __forceinline__
#else
#define CH_HD inline
#endif

#include "../../include/chiaro_depth.h"

namespace chiaro {

constexpr int MAX_VIEWS = 32;    // modules per call
constexpr int MAX_LABELS = 256;  // planes + 1
constexpr int MAX_RADIUS = 16;   // patch radius; the wide retry uses max(2r, 8)

// ---- constants of the reference (depth.rs:23-37) ----------------------------
constexpr double INFINITY_DEPTH = 1.0e8;
constexpr float MISSING_COST = 2.25f;
constexpr float SGM_SMALL_PENALTY = 0.06f;
constexpr float SGM_LARGE_PENALTY = 0.45f;
constexpr float SGM_DIRECTIONS = 8.0f;
constexpr float MINIMUM_REGULARIZED_SCORE = 0.30f;
constexpr float MAXIMUM_REGULARIZED_BASELINE_LOSS = 0.04f;
constexpr float NEAR_DEPTH_PRIOR = 0.10f;
constexpr float WARP_BOUNDARY_DELTA_PX = 2.0f;
constexpr float WARP_BOUNDARY_CONTRAST = 0.30f;
constexpr int MINIMUM_DIRECT_COMPONENT_NODES = 24;

// ---- bit casts -------------------------------------------------------------------
CH_HD uint32_t f2u(float v) { uint32_t u; memcpy(&u, &v, 4); return u; }
CH_HD uint64_t d2u(double v) { uint64_t u; memcpy(&u, &v, 8); return u; }
CH_HD double u2d(uint64_t u) { double v; memcpy(&v, &u, 8); return v; }

// ---- Rust scalar semantics -----------------------------------------------------
// (floor(f) as usize).min(hi) for floor values: NaN and negatives saturate to 0.
CH_HD int sat_index(float f, int hi) {
    if (!(f > 0.0f)) return 0;
    if (f >= (float)hi) return hi;
    return (int)f;
}
CH_HD int sat_index_d(double f, int hi) {
    if (!(f > 0.0)) return 0;
    if (f >= (double)hi) return hi;
    return (int)f;
}
CH_HD float clampf_r(float x, float lo, float hi) {  // f32::clamp
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
CH_HD double clampd_r(double x, double lo, double hi) {  // f64::clamp
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
CH_HD int32_t total_key(float v) {  // order of f32::total_cmp
    int32_t b = (int32_t)f2u(v);
    return b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1);
}
CH_HD float fmin_r(float a, float b) { return fminf(a, b); }  // f32::min (NaN-ignoring)
CH_HD float fmax_r(float a, float b) { return fmaxf(a, b); }  // f32::max

CH_HD double fma_d(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

// ---- exponentials --------------------------------------------------------------
// The reference's f32::exp / f64::exp call the platform libm. These restate the
// table-driven method of the ARM Optimized Routines (Szabolcs Nagy), which glibc
// ships as expf/exp: x = k ln2/N + r, 2^(k/N) from a table of N entries, a short
// polynomial in r, all in double. The tables are 2^(i/N) rounded to double
// (computed, not transcribed); the polynomial coefficients are the published
// minimax values. Both were checked for bit equality against the host libm over
// every argument the stage can produce (tests/test_exact_math.py).

// f32 exp: N = 32, cubic polynomial; exact for |x| < 88 and NaN/inf handled.
#define EXPF_TABLE_VALUES                                                                    \
    0x3ff0000000000000ULL, 0x3fefd9b0d3158574ULL, 0x3fefb5586cf9890fULL, 0x3fef9301d0125b51ULL, \
    0x3fef72b83c7d517bULL, 0x3fef54873168b9aaULL, 0x3fef387a6e756238ULL, 0x3fef1e9df51fdee1ULL, \
    0x3fef06fe0a31b715ULL, 0x3feef1a7373aa9cbULL, 0x3feedea64c123422ULL, 0x3feece086061892dULL, \
    0x3feebfdad5362a27ULL, 0x3feeb42b569d4f82ULL, 0x3feeab07dd485429ULL, 0x3feea47eb03a5585ULL, \
    0x3feea09e667f3bcdULL, 0x3fee9f75e8ec5f74ULL, 0x3feea11473eb0187ULL, 0x3feea589994cce13ULL, \
    0x3feeace5422aa0dbULL, 0x3feeb737b0cdc5e5ULL, 0x3feec49182a3f090ULL, 0x3feed503b23e255dULL, \
    0x3feee89f995ad3adULL, 0x3feeff76f2fb5e47ULL, 0x3fef199bdd85529cULL, 0x3fef3720dcef9069ULL, \
    0x3fef5818dcfba487ULL, 0x3fef7c97337b9b5fULL, 0x3fefa4afa2a490daULL, 0x3fefd0765b6e4540ULL
#include "exp_f64_table.inc"

#ifdef __CUDACC__
__device__ const uint64_t EXPF_TAB_DEVICE[32] = {EXPF_TABLE_VALUES};
__device__ const uint64_t EXP_F64_TAB_DEVICE[256] = {EXP_F64_TABLE_VALUES};
#endif
static const uint64_t EXPF_TAB_HOST[32] = {EXPF_TABLE_VALUES};
static const uint64_t EXP_F64_TAB_HOST[256] = {EXP_F64_TABLE_VALUES};

CH_HD uint64_t expf_table(unsigned i) {
#ifdef __CUDA_ARCH__
    return __ldg(reinterpret_cast<const unsigned long long *>(EXPF_TAB_DEVICE) + i);
#else
    return EXPF_TAB_HOST[i];
#endif
}
CH_HD uint64_t exp_f64_table(unsigned i) {
#ifdef __CUDA_ARCH__
    return __ldg(reinterpret_cast<const unsigned long long *>(EXP_F64_TAB_DEVICE) + i);
#else
    return EXP_F64_TAB_HOST[i];
#endif
}

CH_HD float exp_f32(float x) {
    const double inv_ln2_n = 0x1.71547652b82fep+0 * 32.0;
    const double shift = 0x1.8p+52;
    const double c0 = 0x1.c6af84b912394p-5 / 32.0 / 32.0 / 32.0;
    const double c1 = 0x1.ebfce50fac4f3p-3 / 32.0 / 32.0;
    const double c2 = 0x1.62e42ff0c52d6p-1 / 32.0;
    if (x != x) return x;
    if (x <= -0x1.9fe368p6f) return 0.0f;  // underflows to +0 like libm
    if (x > 0x1.62e42ep6f) return INFINITY;
    double xd = (double)x;
    double z = inv_ln2_n * xd;
    double kd = z + shift;
    uint64_t ki = d2u(kd);
    kd -= shift;
    double r = z - kd;
    uint64_t t = expf_table((unsigned)(ki % 32)) + (ki << 47);
    double s = u2d(t);
    double zz = c0 * r + c1;
    double r2 = r * r;
    double y = c2 * r + 1.0;
    y = zz * r2 + y;
    y = y * s;
    return (float)y;
}

// f64 exp: N = 128, table of (tail, 2^(i/N) - (i << 45)) pairs, quartic
// polynomial evaluated with fused multiply-adds as the x86-64 FMA build of libm
// does. Used on [-1.5, 0] (the local plane fit); NaN/inf handled.

CH_HD double exp_f64(double x) {
    const double inv_ln2_n = 0x1.71547652b82fep0 * 128.0;
    const double shift = 0x1.8p52;
    const double neg_ln2_hi_n = -0x1.62e42fefa0000p-8;
    const double neg_ln2_lo_n = -0x1.cf79abc9e3b3ap-47;
    const double c2 = 0x1.ffffffffffdbdp-2, c3 = 0x1.555555555543cp-3;
    const double c4 = 0x1.55555cf172b91p-5, c5 = 0x1.1111167a4d017p-7;
    if (x != x) return x;
    if (x < -700.0) return 0.0;
    if (x > 700.0) return INFINITY;
    double z = inv_ln2_n * x;
    double kd = z + shift;
    uint64_t ki = d2u(kd);
    kd -= shift;
    double r = x + kd * neg_ln2_hi_n + kd * neg_ln2_lo_n;
    uint64_t idx = 2 * (ki % 128);
    uint64_t top = ki << 45;
    double tail = u2d(exp_f64_table((unsigned)idx));
    uint64_t sbits = exp_f64_table((unsigned)idx + 1) + top;
    double r2 = r * r;
    double tmp = fma_d(r2 * r2, fma_d(r, c5, c4), fma_d(r2, fma_d(r, c3, c2), tail + r));
    double scale = u2d(sbits);
    return fma_d(scale, tmp, scale);
}

// floor(x) as an int and x - floor(x) for 0 <= x < 2^22 without a
// float-to-int conversion: r = floor(x) is an integer below 2^22, so r + 2^23
// is exact and holds r in its low mantissa bits; x - r is exact.
// floor(n / d) for 0 <= n, 1 <= d and n d < 2^32, with one multiply instead of an
// integer division: division by an invariant integer (Granlund and Montgomery, 1994)
// with m = ceil(2^32 / d). Writing m d = 2^32 + e with 0 <= e < d, n m / 2^32 =
// n / d + n e / (d 2^32), and n e < n d < 2^32 keeps the second term below 1 / d, so the
// high word of n m is the exact quotient. d = 1 keeps n (its m would be 2^32). Every use
// in the kernels has n, d < 2^16 (items below MAX_VIEWS * MAX_LABELS, taps below 65^2).
struct SmallDiv {
    uint32_t m, d;
    CH_HD explicit SmallDiv(int divisor)
        : m(divisor > 1 ? 0xFFFFFFFFu / (uint32_t)divisor + 1u : 0u), d((uint32_t)divisor) {}
    CH_HD int quotient(int n) const {
        return d > 1 ? (int)(((uint64_t)(uint32_t)n * m) >> 32) : n;
    }
};

// aggregate (depth.rs:1761-1770) of n <= N per-view scores s[i * stride] (NaN = None) in
// registers. The reference compacts the Some scores, sorts them descending by
// f32::total_cmp with a stable sort, needs at least minimum_support of them, and averages
// the first min(best_view_count, m) after adding them in that order from -0.0. Here a
// sorting network (Batcher's odd-even merge, N = 4 or 8) orders (key, score) pairs
// descending, a None taking a key below every score. Equal keys are bit-identical scores,
// so the sorted sequence, and with it the sum, is the reference's whatever the order the
// network leaves among equals.
template <int N>
CH_HD bool aggregate_small(const float *s, int stride, int n, int minimum_support, int best_view_count,
                           float &out) {
    static_assert(N == 4 || N == 8, "networks for 4 and 8 views");
    int32_t key[N];
    float val[N];
    int m = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const float x = i < n ? s[i * stride] : NAN;
        const bool some = !(x != x);
        m += some ? 1 : 0;
        key[i] = some ? total_key(x) : INT32_MIN;
        val[i] = x;
    }
    if (m < minimum_support) return false;
    constexpr int pairs = N == 4 ? 5 : 19;
    constexpr int net[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {1, 2}, {5, 6},
                                {0, 4}, {1, 5}, {2, 6}, {3, 7}, {2, 4}, {3, 5}, {1, 2}, {3, 4}, {5, 6}};
    constexpr int net4[5][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}};
#pragma unroll
    for (int c = 0; c < pairs; ++c) {
        const int a = N == 4 ? net4[c][0] : net[c][0], b = N == 4 ? net4[c][1] : net[c][1];
        const bool swap = key[a] < key[b];
        const int32_t ka = key[a];
        const float va = val[a];
        key[a] = swap ? key[b] : ka;
        val[a] = swap ? val[b] : va;
        key[b] = swap ? ka : key[b];
        val[b] = swap ? va : val[b];
    }
    const int k = best_view_count < m ? best_view_count : m;
    if (k < minimum_support) return false;
    float sum = -0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (i < k) sum += val[i];
    out = sum / (float)k;
    return true;
}

CH_HD float floor_frac_small(float x, int &ix) {
    const float r = floorf(x);
    ix = (int)(f2u(r + 8388608.0f) - 0x4B000000u);  // 2^23
    return x - r;
}

// ---- Plane::sample (image.rs:451-466) --------------------------------------------
struct PlaneRef {
    const float *data;
    int width, height;
};

CH_HD float plane_at(const PlaneRef &p, int x, int y) {
#ifdef __CUDA_ARCH__
    return __ldg(p.data + (size_t)y * p.width + x);
#else
    return p.data[(size_t)y * p.width + x];
#endif
}

// Returns false for None.
CH_HD bool plane_sample(const PlaneRef &p, float x, float y, float &out) {
    if (!(x >= 0.0f && y >= 0.0f && x <= (float)(p.width - 1) && y <= (float)(p.height - 1))) return false;
    float fx = floorf(x), fy = floorf(y);
    int x0 = (int)fx, y0 = (int)fy;
    int x1 = x0 + 1 < p.width - 1 ? x0 + 1 : p.width - 1;
    int y1 = y0 + 1 < p.height - 1 ? y0 + 1 : p.height - 1;
    float tx = x - fx;  // x - (x0 as f32); x0 == floor(x) exactly
    float ty = y - fy;
    float top = plane_at(p, x0, y0) * (1.0f - tx) + plane_at(p, x1, y0) * tx;
    float bottom = plane_at(p, x0, y1) * (1.0f - tx) + plane_at(p, x1, y1) * tx;
    out = top * (1.0f - ty) + bottom * ty;
    return true;
}

// ---- Warp::map (align.rs:84-111) ---------------------------------------------------
struct WarpRef {
    const float2 *points;
    int step, columns, rows;
};

CH_HD float2 warp_point(const WarpRef &w, int c, int r) {
#ifdef __CUDA_ARCH__
    return __ldg(w.points + (size_t)r * w.columns + c);
#else
    return w.points[(size_t)r * w.columns + c];
#endif
}

CH_HD bool warp_map(const WarpRef &w, float x, float y, float &qx, float &qy) {
    float fx = x / (float)w.step;
    float fy = y / (float)w.step;
    if (fx < 0.0f || fy < 0.0f) return false;
    int c0 = sat_index(floorf(fx), w.columns - 1);
    int r0 = sat_index(floorf(fy), w.rows - 1);
    int c1 = c0 + 1 < w.columns - 1 ? c0 + 1 : w.columns - 1;
    int r1 = r0 + 1 < w.rows - 1 ? r0 + 1 : w.rows - 1;
    float tx = fx - (float)c0;
    float ty = fy - (float)r0;
    float2 a = warp_point(w, c0, r0), b = warp_point(w, c1, r0), c = warp_point(w, c0, r1), d = warp_point(w, c1, r1);
    float top0 = a.x * (1.0f - tx) + b.x * tx;
    float bottom0 = c.x * (1.0f - tx) + d.x * tx;
    qx = top0 * (1.0f - ty) + bottom0 * ty;
    float top1 = a.y * (1.0f - tx) + b.y * tx;
    float bottom1 = c.y * (1.0f - tx) + d.y * tx;
    qy = top1 * (1.0f - ty) + bottom1 * ty;
    return !(qx != qx || qy != qy);
}

// ---- camera model (geometry.rs:139-240, math.rs) ------------------------------------
struct DevCamera {
    double k[9], k_inverse[9];
    double dist_center[2], dist_norm[2], dist_coeffs[5];
    double rotation_wc[9], rotation_cw[9], translation_wc[3], center[3];
    double real_cw[9], reflect[9], virtual_center[3];
    double oc[9];
    double width, height;
    int has_distortion, flip, pose_kind, oc_identity;
};

struct D3 {
    double x, y, z;
};

CH_HD double dot3(const double *m, D3 v) { return m[0] * v.x + m[1] * v.y + m[2] * v.z; }
CH_HD D3 mul_vec(const double *m, D3 v) { return {dot3(m, v), dot3(m + 3, v), dot3(m + 6, v)}; }
CH_HD D3 mul_vec_t(const double *m, D3 v) {  // transpose(m) * v
    return {m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
            m[2] * v.x + m[5] * v.y + m[8] * v.z};
}
CH_HD D3 normalize3(D3 a) {  // math.rs:39-42
    double n = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    if (n == 0.0) return a;
    double s = 1.0 / n;
    return {a.x * s, a.y * s, a.z * s};
}

CH_HD void distort_normalized(const double *c, double x, double y, double &ox, double &oy) {  // geometry.rs:313-323
    double k1 = c[0], k2 = c[1], p1 = c[2], p2 = c[3], k3 = c[4];
    double r2 = x * x + y * y;
    double radial = 1.0 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2;
    ox = x * radial + 2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x);
    oy = y * radial + p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y;
}

CH_HD void distort(const DevCamera &c, double px, double py, double &ox, double &oy) {  // geometry.rs:325-330
    double nx = (px - c.dist_center[0]) / c.dist_norm[0];
    double ny = (py - c.dist_center[1]) / c.dist_norm[1];
    double dx, dy;
    distort_normalized(c.dist_coeffs, nx, ny, dx, dy);
    ox = dx * c.dist_norm[0] + c.dist_center[0];
    oy = dy * c.dist_norm[1] + c.dist_center[1];
}

CH_HD void undistort(const DevCamera &c, double px, double py, double &ox, double &oy) {  // geometry.rs:334-353
    double obx = (px - c.dist_center[0]) / c.dist_norm[0];
    double oby = (py - c.dist_center[1]) / c.dist_norm[1];
    double ex = obx, ey = oby;
    for (int i = 0; i < 20; ++i) {
        double dx, dy;
        distort_normalized(c.dist_coeffs, ex, ey, dx, dy);
        double nx = ex + (obx - dx), ny = ey + (oby - dy);
        double delta = fmax(fabs(nx - ex), fabs(ny - ey));
        ex = nx;
        ey = ny;
        if (delta < 1e-12) break;
    }
    ox = ex * c.dist_norm[0] + c.dist_center[0];
    oy = ey * c.dist_norm[1] + c.dist_center[1];
}

CH_HD void reflect_image_axis(const DevCamera &c, double &x, double &y) {  // geometry.rs:129-136
    if (c.flip == 1)
        y = -y;
    else if (c.flip == 2)
        x = -x;
}

// pixel_to_ray (geometry.rs:139-166)
CH_HD void pixel_to_ray(const DevCamera &c, double px, double py, D3 &origin, D3 &direction) {
    double ix = px, iy = py;
    if (c.has_distortion) undistort(c, px, py, ix, iy);
    D3 d = normalize3(mul_vec(c.k_inverse, {ix, iy, 1.0}));
    if (c.flip != 0) {
        double x = d.x, y = d.y;
        reflect_image_axis(c, x, y);
        d = normalize3({x, y, d.z});
    }
    D3 world;
    if (c.pose_kind == 0) {
        origin = {c.center[0], c.center[1], c.center[2]};
        world = mul_vec(c.rotation_cw, d);
    } else {
        origin = {c.virtual_center[0], c.virtual_center[1], c.virtual_center[2]};
        world = mul_vec(c.reflect, mul_vec(c.real_cw, d));
    }
    direction = normalize3(mul_vec(c.oc, normalize3(world)));
}

// project (geometry.rs:172-231), bounded. Returns false for None.
CH_HD bool project(const DevCamera &c, D3 point, double &ox, double &oy) {
    if (!c.oc_identity) {
        D3 cen = c.pose_kind == 0 ? D3{c.center[0], c.center[1], c.center[2]}
                                  : D3{c.virtual_center[0], c.virtual_center[1], c.virtual_center[2]};
        D3 rel = mul_vec_t(c.oc, {point.x - cen.x, point.y - cen.y, point.z - cen.z});
        point = {cen.x + rel.x, cen.y + rel.y, cen.z + rel.z};
    }
    D3 cam;
    if (c.pose_kind == 0) {
        D3 m = mul_vec(c.rotation_wc, point);
        cam = {m.x + c.translation_wc[0], m.y + c.translation_wc[1], m.z + c.translation_wc[2]};
    } else {
        D3 s = {point.x - c.virtual_center[0], point.y - c.virtual_center[1], point.z - c.virtual_center[2]};
        cam = mul_vec_t(c.real_cw, mul_vec(c.reflect, s));
    }
    if (cam.z <= 0.0) return false;
    double nx = cam.x / cam.z, ny = cam.y / cam.z;
    reflect_image_axis(c, nx, ny);
    double ix = c.k[0] * nx + c.k[1] * ny + c.k[2];
    double iy = c.k[4] * ny + c.k[5];
    double mx = c.width * 0.5, my = c.height * 0.5;
    if (ix < -mx || iy < -my || ix > c.width + mx || iy > c.height + my) return false;
    if (c.has_distortion) {
        distort(c, ix, iy, ox, oy);
    } else {
        ox = ix;
        oy = iy;
    }
    return true;
}

// Ray-to-point at a depth along a unit direction: add(origin, scale(direction, depth)).
CH_HD D3 along(D3 origin, D3 direction, double depth) {
    return {origin.x + direction.x * depth, origin.y + direction.y * depth, origin.z + direction.z * depth};
}

// ---- device forms of the boundary types -------------------------------------------
struct DevView {
    PlaneRef luma;
    const float4 *quads;  // bilinear neighbourhood (quad) plane of the luminance (targets only)
    WarpRef warp;
    int width, height;
    int has_camera, accepted;
    DevCamera cam;
};

// DepthOptions fields read by kernels (depth.rs:39-67) plus derived values.
struct DevOptions {
    double near_depth, far_depth;
    double inverse_step;  // (1/near - 1/far) / (planes - 1), depth.rs:346-347
    float minimum_score, minimum_margin, minimum_improvement;
    int patch_radius, minimum_support, best_view_count, minimum_neighbour_support;
};

// Fill a DevCamera from the ABI struct (host side).
inline void camera_from_abi(const chiaro_camera &a, DevCamera &c) {
    memcpy(c.k, a.k, sizeof(c.k));
    memcpy(c.k_inverse, a.k_inverse, sizeof(c.k_inverse));
    for (int i = 0; i < 2; ++i) {
        c.dist_center[i] = a.distortion_center[i];
        c.dist_norm[i] = a.distortion_normalization[i];
    }
    for (int i = 0; i < 5; ++i) c.dist_coeffs[i] = a.distortion_coeffs[i];
    memcpy(c.rotation_wc, a.rotation_wc, sizeof(c.rotation_wc));
    memcpy(c.rotation_cw, a.rotation_cw, sizeof(c.rotation_cw));
    memcpy(c.translation_wc, a.translation_wc, sizeof(c.translation_wc));
    memcpy(c.center, a.center, sizeof(c.center));
    memcpy(c.real_cw, a.real_cw, sizeof(c.real_cw));
    memcpy(c.reflect, a.reflect, sizeof(c.reflect));
    memcpy(c.virtual_center, a.virtual_center, sizeof(c.virtual_center));
    memcpy(c.oc, a.orientation_correction, sizeof(c.oc));
    c.width = (double)a.width;
    c.height = (double)a.height;
    c.has_distortion = a.has_distortion != 0;
    c.flip = a.flip;
    c.pose_kind = a.pose_kind;
    static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    c.oc_identity = 1;
    for (int i = 0; i < 9; ++i)
        if (!(a.orientation_correction[i] == I[i])) c.oc_identity = 0;
}

}  // namespace chiaro
