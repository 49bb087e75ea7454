// chiaro_oracle.cpp — CPU ORACLE for the multi-view depth stage.
//
// TEST INFRASTRUCTURE ONLY. This file restates, in plain C++17, the Rust
// reference path of chiaro-fusion's depth stage so that the CUDA library can be
// checked against it and so that the reference's CPU cost can be timed on the
// same host. Only the tests, the smoke check and the benchmark's CPU-baseline
// leg load it; the product library never links or calls it.
//
// It follows, function by function:
//   crates/chiaro-fusion/src/depth.rs     (the stage, lines 312-1891)
//   crates/chiaro-fusion/src/image.rs     (Plane::sample 451-466, luminance_half 401-428)
//   crates/chiaro-fusion/src/align.rs     (Warp::map 84-111, magnification 133-143)
//   crates/chiaro-fusion/src/geometry.rs  (pixel_to_ray/project/map_from 140-274,
//                                          distort/undistort 298-360)
//   crates/chiaro-fusion/src/math.rs      (3x3 f64 algebra 1-139)
//
// Fidelity rules (each changes results if broken):
//   - compiled with -ffp-contract=off and without fast-math: Rust never fuses
//     a*b+c, so neither may this file;
//   - f32 expressions stay f32, f64 stay f64, in the reference's operand order;
//   - exp/expf/log come from the platform libm, which is what Rust's f64::exp /
//     f32::exp / f32::ln call on Linux;
//   - Iterator::min_by keeps the first minimum, max_by the last maximum,
//     sort_by is stable, f32::min/max ignore NaN, `as usize` saturates;
//   - f32 Sum starts from -0.0 (current Rust).
//
// The reference threads the cost build and the direct pass over row bands
// (depth.rs:1204-1206, 729-731); this oracle does the same with std::thread.
// SGM and the per-target loop are serial, as in the reference.

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <optional>
#include <string>
#include <thread>
#include <vector>

#include "../include/chiaro_depth.h"

namespace oracle {

using Vec2 = std::array<double, 2>;
using Vec3 = std::array<double, 3>;
using Mat3 = std::array<std::array<double, 3>, 3>;
using F2 = std::array<float, 2>;

// ---- constants (depth.rs:23-37) --------------------------------------------
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
constexpr size_t MINIMUM_DIRECT_COMPONENT_NODES = 24;

// ---- Rust scalar semantics ------------------------------------------------
static inline size_t sat_usize(double v) {  // `as usize` (saturating, NaN -> 0)
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551615.0) return SIZE_MAX;
    return (size_t)v;
}
static inline float fmin_r(float a, float b) { return std::fmin(a, b); }  // f32::min
static inline float fmax_r(float a, float b) { return std::fmax(a, b); }  // f32::max
static inline double dmax_r(double a, double b) { return std::fmax(a, b); }
static inline float fclamp(float x, float lo, float hi) {  // f32::clamp
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
static inline double dclamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// total_cmp keys: order of the IEEE bit pattern with the sign trick.
static inline int32_t total_key_f32(float v) {
    int32_t b;
    std::memcpy(&b, &v, 4);
    return b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1);
}
static inline int64_t total_key_f64(double v) {
    int64_t b;
    std::memcpy(&b, &v, 8);
    return b ^ (int64_t)(((uint64_t)(b >> 63)) >> 1);
}
static inline size_t div_ceil(size_t a, size_t b) { return (a + b - 1) / b; }
static inline size_t abs_diff(size_t a, size_t b) { return a > b ? a - b : b - a; }

// ---- math.rs --------------------------------------------------------------
static inline double dot(const Vec3 &a, const Vec3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline Vec3 add(const Vec3 &a, const Vec3 &b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
static inline Vec3 sub(const Vec3 &a, const Vec3 &b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static inline Vec3 scale(const Vec3 &a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
static inline double norm(const Vec3 &a) { return std::sqrt(dot(a, a)); }
static inline Vec3 normalize(const Vec3 &a) {  // math.rs:39-42
    double n = norm(a);
    return n == 0.0 ? a : scale(a, 1.0 / n);
}
static inline Vec3 mul_vec(const Mat3 &m, const Vec3 &v) { return {dot(m[0], v), dot(m[1], v), dot(m[2], v)}; }
static inline Mat3 transpose(const Mat3 &m) {
    return {{{m[0][0], m[1][0], m[2][0]}, {m[0][1], m[1][1], m[2][1]}, {m[0][2], m[1][2], m[2][2]}}};
}
static inline double determinant(const Mat3 &m) {  // math.rs:64-68
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}
static std::optional<Mat3> inverse(const Mat3 &m) {  // math.rs:70-95
    double det = determinant(m);
    if (std::fabs(det) < 1e-300) return std::nullopt;
    double inv_det = 1.0 / det;
    auto c = [&](int r0, int c0, int r1, int c1) { return m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0]; };
    Mat3 out = {{{c(1, 1, 2, 2) * inv_det, -c(0, 1, 2, 2) * inv_det, c(0, 1, 1, 2) * inv_det},
                 {-c(1, 0, 2, 2) * inv_det, c(0, 0, 2, 2) * inv_det, -c(0, 0, 1, 2) * inv_det},
                 {c(1, 0, 2, 1) * inv_det, -c(0, 0, 2, 1) * inv_det, c(0, 0, 1, 1) * inv_det}}};
    return out;
}
static Mat3 mat_from(const double *m) {
    return {{{m[0], m[1], m[2]}, {m[3], m[4], m[5]}, {m[6], m[7], m[8]}}};
}

// ---- geometry.rs ----------------------------------------------------------
struct Distortion {
    Vec2 center, normalization;
    double coeffs[5];
};

static inline Vec2 to_normalized(const Distortion &d, const Vec2 &p) {  // geometry.rs:298-303
    return {(p[0] - d.center[0]) / d.normalization[0], (p[1] - d.center[1]) / d.normalization[1]};
}
static inline Vec2 from_normalized(const Distortion &d, const Vec2 &n) {  // geometry.rs:305-310
    return {n[0] * d.normalization[0] + d.center[0], n[1] * d.normalization[1] + d.center[1]};
}
static inline Vec2 distort_normalized(const double *c, const Vec2 &xy) {  // geometry.rs:313-323
    double k1 = c[0], k2 = c[1], p1 = c[2], p2 = c[3], k3 = c[4];
    double x = xy[0], y = xy[1];
    double r2 = x * x + y * y;
    double radial = 1.0 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2;
    return {x * radial + 2.0 * p1 * x * y + p2 * (r2 + 2.0 * x * x),
            y * radial + p1 * (r2 + 2.0 * y * y) + 2.0 * p2 * x * y};
}
static inline Vec2 distort(const Distortion &d, const Vec2 &ideal) {  // geometry.rs:325-330
    return from_normalized(d, distort_normalized(d.coeffs, to_normalized(d, ideal)));
}
static inline Vec2 undistort(const Distortion &d, const Vec2 &pixel) {  // geometry.rs:334-353
    Vec2 observed = to_normalized(d, pixel);
    Vec2 estimate = observed;
    for (int i = 0; i < 20; ++i) {
        Vec2 distorted = distort_normalized(d.coeffs, estimate);
        Vec2 next = {estimate[0] + (observed[0] - distorted[0]), estimate[1] + (observed[1] - distorted[1])};
        double delta = dmax_r(std::fabs(next[0] - estimate[0]), std::fabs(next[1] - estimate[1]));
        estimate = next;
        if (delta < 1e-12) break;
    }
    return from_normalized(d, estimate);
}

struct Ray {
    Vec3 origin, direction;
};

struct Camera {  // ResolvedCamera (geometry.rs:31-62)
    size_t width, height;
    Mat3 k, k_inverse;
    bool has_distortion;
    Distortion distortion;
    int flip;  // 0 none, 1 Some(true), 2 Some(false)
    int pose;  // 0 canonical, 1 mirror
    Mat3 rotation_wc, rotation_cw;
    Vec3 translation_wc, center_c;
    Mat3 real_cw, reflect;
    Vec3 virtual_center;
    Mat3 orientation_correction;
    bool oc_identity;

    explicit Camera(const chiaro_camera &c) {
        width = (size_t)c.width;
        height = (size_t)c.height;
        k = mat_from(c.k);
        k_inverse = mat_from(c.k_inverse);
        has_distortion = c.has_distortion != 0;
        distortion.center = {c.distortion_center[0], c.distortion_center[1]};
        distortion.normalization = {c.distortion_normalization[0], c.distortion_normalization[1]};
        for (int i = 0; i < 5; ++i) distortion.coeffs[i] = c.distortion_coeffs[i];
        flip = c.flip;
        pose = c.pose_kind;
        rotation_wc = mat_from(c.rotation_wc);
        rotation_cw = mat_from(c.rotation_cw);
        translation_wc = {c.translation_wc[0], c.translation_wc[1], c.translation_wc[2]};
        center_c = {c.center[0], c.center[1], c.center[2]};
        real_cw = mat_from(c.real_cw);
        reflect = mat_from(c.reflect);
        virtual_center = {c.virtual_center[0], c.virtual_center[1], c.virtual_center[2]};
        orientation_correction = mat_from(c.orientation_correction);
        static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        oc_identity = true;
        for (int i = 0; i < 9; ++i)
            if (!(c.orientation_correction[i] == I[i])) oc_identity = false;
    }

    Vec3 center() const { return pose == 0 ? center_c : virtual_center; }  // geometry.rs:121-126

    Vec2 reflect_image_axis(const Vec2 &n) const {  // geometry.rs:129-136
        if (flip == 1) return {n[0], -n[1]};
        if (flip == 2) return {-n[0], n[1]};
        return n;
    }

    Ray pixel_to_ray(const Vec2 &pixel) const {  // geometry.rs:139-166
        Vec2 ideal = has_distortion ? undistort(distortion, pixel) : pixel;
        Vec3 direction = normalize(mul_vec(k_inverse, {ideal[0], ideal[1], 1.0}));
        if (flip != 0) {
            Vec2 xy = reflect_image_axis({direction[0], direction[1]});
            direction = normalize({xy[0], xy[1], direction[2]});
        }
        Vec3 origin, world;
        if (pose == 0) {
            origin = center_c;
            world = mul_vec(rotation_cw, direction);
        } else {
            origin = virtual_center;
            world = mul_vec(reflect, mul_vec(real_cw, direction));
        }
        return {origin, normalize(mul_vec(orientation_correction, normalize(world)))};
    }

    std::optional<Vec2> project(Vec3 point) const {  // geometry.rs:172-231, bounded
        if (!oc_identity) {
            Vec3 c = center();
            point = add(c, mul_vec(transpose(orientation_correction), sub(point, c)));
        }
        Vec3 camera;
        if (pose == 0)
            camera = add(mul_vec(rotation_wc, point), translation_wc);
        else
            camera = mul_vec(transpose(real_cw), mul_vec(reflect, sub(point, virtual_center)));
        if (camera[2] <= 0.0) return std::nullopt;
        Vec2 normalized = reflect_image_axis({camera[0] / camera[2], camera[1] / camera[2]});
        Vec2 ideal = {k[0][0] * normalized[0] + k[0][1] * normalized[1] + k[0][2], k[1][1] * normalized[1] + k[1][2]};
        double margin_x = (double)width * 0.5;
        double margin_y = (double)height * 0.5;
        if (ideal[0] < -margin_x || ideal[1] < -margin_y || ideal[0] > (double)width + margin_x ||
            ideal[1] > (double)height + margin_y)
            return std::nullopt;
        return has_distortion ? distort(distortion, ideal) : ideal;
    }

    // self = target; geometry.rs:237-240
    std::optional<Vec2> map_from(const Camera &reference, const Vec2 &pixel, double depth) const {
        Ray ray = reference.pixel_to_ray(pixel);
        return project(add(ray.origin, scale(ray.direction, depth)));
    }
};

// ---- image.rs: Plane ------------------------------------------------------
struct Plane {
    size_t width = 0, height = 0;
    const float *data = nullptr;
    float at(size_t x, size_t y) const { return data[y * width + x]; }
    std::optional<float> sample(float x, float y) const {  // image.rs:451-466
        if (!(x >= 0.0f && y >= 0.0f && x <= (float)(width - 1) && y <= (float)(height - 1))) return std::nullopt;
        size_t x0 = sat_usize(std::floor(x));
        size_t y0 = sat_usize(std::floor(y));
        size_t x1 = std::min(x0 + 1, width - 1);
        size_t y1 = std::min(y0 + 1, height - 1);
        float tx = x - (float)x0;
        float ty = y - (float)y0;
        float top = at(x0, y0) * (1.0f - tx) + at(x1, y0) * tx;
        float bottom = at(x0, y1) * (1.0f - tx) + at(x1, y1) * tx;
        return top * (1.0f - ty) + bottom * ty;
    }
};

// ---- align.rs: Warp -------------------------------------------------------
struct Warp {
    size_t step = 0, columns = 0, rows = 0;
    const float *points = nullptr;  // 2*columns*rows
    F2 p(size_t c, size_t r) const { return {points[2 * (r * columns + c)], points[2 * (r * columns + c) + 1]}; }
    std::optional<F2> map(float x, float y) const {  // align.rs:84-111
        float fx = x / (float)step;
        float fy = y / (float)step;
        if (fx < 0.0f || fy < 0.0f) return std::nullopt;
        size_t c0 = std::min(sat_usize(std::floor(fx)), columns - 1);
        size_t r0 = std::min(sat_usize(std::floor(fy)), rows - 1);
        size_t c1 = std::min(c0 + 1, columns - 1);
        size_t r1 = std::min(r0 + 1, rows - 1);
        float tx = fx - (float)c0;
        float ty = fy - (float)r0;
        F2 a = p(c0, r0), b = p(c1, r0), c = p(c0, r1), d = p(c1, r1);
        F2 out;
        for (int k = 0; k < 2; ++k) {
            float top = a[k] * (1.0f - tx) + b[k] * tx;
            float bottom = c[k] * (1.0f - tx) + d[k] * tx;
            out[k] = top * (1.0f - ty) + bottom * ty;
        }
        if (std::isnan(out[0]) || std::isnan(out[1])) return std::nullopt;
        return out;
    }
};

// ---- depth.rs -------------------------------------------------------------
struct Options {  // DepthOptions (depth.rs:39-67)
    bool enabled;
    size_t grid_step;
    double near_depth, far_depth;
    size_t planes, patch_radius, minimum_support, best_view_count;
    float minimum_score, minimum_margin, minimum_improvement;
    size_t minimum_neighbour_support, completion_iterations;
    explicit Options(const chiaro_depth_options &o) {
        enabled = o.enabled != 0;
        grid_step = (size_t)o.grid_step;
        near_depth = o.near_depth;
        far_depth = o.far_depth;
        planes = (size_t)o.planes;
        patch_radius = (size_t)o.patch_radius;
        minimum_support = (size_t)o.minimum_support;
        best_view_count = (size_t)o.best_view_count;
        minimum_score = o.minimum_score;
        minimum_margin = o.minimum_margin;
        minimum_improvement = o.minimum_improvement;
        minimum_neighbour_support = (size_t)o.minimum_neighbour_support;
        completion_iterations = (size_t)o.completion_iterations;
    }
};

static void default_options(chiaro_depth_options *o) {  // depth.rs:69-91
    std::memset(o, 0, sizeof(*o));
    o->enabled = 1;
    o->grid_step = 8;
    o->near_depth = 500.0;
    o->far_depth = 10000000.0;
    o->planes = 96;
    o->patch_radius = 4;
    o->minimum_support = 2;
    o->best_view_count = 3;
    o->minimum_score = 0.45f;
    o->minimum_margin = 0.01f;
    o->minimum_improvement = 0.01f;
    o->minimum_neighbour_support = 2;
    o->completion_iterations = 0;
}

static bool valid_options(const Options &o) {  // depth.rs:1879-1891
    return o.enabled && o.grid_step > 0 && std::isfinite(o.near_depth) && std::isfinite(o.far_depth) &&
           o.near_depth > 0.0 && o.far_depth > o.near_depth && o.planes >= 3 && o.patch_radius > 0 &&
           o.minimum_support > 0 && o.best_view_count >= o.minimum_support && o.minimum_neighbour_support > 0;
}

struct NodeDepth {  // depth.rs:248-254
    double depth;
    float confidence;
    float improvement;
    bool regularized;
};
using Field = std::vector<std::optional<NodeDepth>>;

struct Input {  // AlignInput + ModuleAlignment for one module
    Plane luminance;
    size_t width, height;
    std::optional<Camera> camera;
    bool accepted;
    Warp warp;
};

static std::vector<double> inverse_depth_samples(double near_d, double far_d, size_t count) {  // depth.rs:1834-1843
    double near_inverse = 1.0 / near_d;
    double far_inverse = 1.0 / far_d;
    std::vector<double> out(count);
    for (size_t index = 0; index < count; ++index) {
        double weight = (double)index / (double)(count - 1);
        out[index] = 1.0 / (near_inverse * (1.0 - weight) + far_inverse * weight);
    }
    return out;
}

// warped_patch_zncc (depth.rs:1772-1822)
static std::optional<float> warped_patch_zncc(const Plane &reference, const Plane &target, const Warp &global,
                                              const Vec2 &centre, const Vec2 &delta, size_t radius) {
    auto centre_reference =
        reference.sample((float)((centre[0] - 0.5) * 0.5), (float)((centre[1] - 0.5) * 0.5));
    if (!centre_reference) return std::nullopt;
    float sigma = fmax_r((float)radius * 0.75f, 1.0f);
    float count = 0.0f, sum_reference = 0.0f, sum_target = 0.0f, sum_reference_sq = 0.0f, sum_target_sq = 0.0f,
          sum_product = 0.0f;
    long r = (long)radius;
    for (long dy = -r; dy <= r; ++dy) {
        for (long dx = -r; dx <= r; ++dx) {
            Vec2 p = {centre[0] + (double)dx * 2.0, centre[1] + (double)dy * 2.0};
            auto reference_value = reference.sample((float)((p[0] - 0.5) * 0.5), (float)((p[1] - 0.5) * 0.5));
            if (!reference_value) return std::nullopt;
            auto global_q = global.map((float)p[0], (float)p[1]);
            if (!global_q) return std::nullopt;
            Vec2 q = {(double)(*global_q)[0] + delta[0], (double)(*global_q)[1] + delta[1]};
            auto target_value = target.sample((float)((q[0] - 0.5) * 0.5), (float)((q[1] - 0.5) * 0.5));
            if (!target_value) return std::nullopt;
            float distance_sq = (float)(dx * dx + dy * dy);
            float spatial = std::exp(-distance_sq / (2.0f * sigma * sigma));
            float range = std::exp(-1.2f * std::fabs(*reference_value - *centre_reference));
            float weight = spatial * range;
            float rv = *reference_value, tv = *target_value;
            count += weight;
            sum_reference += weight * rv;
            sum_target += weight * tv;
            sum_reference_sq += weight * rv * rv;
            sum_target_sq += weight * tv * tv;
            sum_product += weight * rv * tv;
        }
    }
    float covariance = sum_product - sum_reference * sum_target / count;
    float reference_energy = sum_reference_sq - sum_reference * sum_reference / count;
    float target_energy = sum_target_sq - sum_target * sum_target / count;
    float denominator = std::sqrt(fmax_r(reference_energy, 0.0f) * fmax_r(target_energy, 0.0f));
    if (denominator > 1.0e-6f) return fclamp(covariance / denominator, -1.0f, 1.0f);
    return std::nullopt;
}

// map_at_depth (depth.rs:1738-1759)
static std::optional<Vec2> map_at_depth(const Camera &reference_camera, const Camera &target_camera,
                                        const Warp &global, const Vec2 &pixel, double depth) {
    auto global_q = global.map((float)pixel[0], (float)pixel[1]);
    if (!global_q) return std::nullopt;
    auto corrected_reference =
        reference_camera.map_from(target_camera, {(double)(*global_q)[0], (double)(*global_q)[1]}, INFINITY_DEPTH);
    if (!corrected_reference) return std::nullopt;
    auto q = target_camera.map_from(reference_camera, *corrected_reference, depth);
    if (!q) return std::nullopt;
    if (std::isfinite((*q)[0]) && std::isfinite((*q)[1])) return q;
    return std::nullopt;
}

// score_one_view (depth.rs:1593-1627)
static std::optional<float> score_one_view(const Input &reference, const Input &target, const Warp &global,
                                           const Vec2 &centre, std::optional<double> depth, size_t patch_radius) {
    if (!reference.camera || !target.camera) return std::nullopt;
    auto global_centre = global.map((float)centre[0], (float)centre[1]);
    if (!global_centre) return std::nullopt;
    Vec2 mapped_centre;
    if (depth) {
        auto m = map_at_depth(*reference.camera, *target.camera, global, centre, *depth);
        if (!m) return std::nullopt;
        mapped_centre = *m;
    } else {
        mapped_centre = {(double)(*global_centre)[0], (double)(*global_centre)[1]};
    }
    Vec2 delta = {mapped_centre[0] - (double)(*global_centre)[0], mapped_centre[1] - (double)(*global_centre)[1]};
    if (std::fabs(delta[0]) > 128.0 || std::fabs(delta[1]) > 128.0) return std::nullopt;
    return warped_patch_zncc(reference.luminance, target.luminance, global, centre, delta, patch_radius);
}

// score_views (depth.rs:1566-1591)
static std::vector<float> score_views(const std::vector<Input> &inputs, size_t reference_index, const Vec2 &centre,
                                      std::optional<double> depth, size_t patch_radius) {
    std::vector<float> out;
    for (size_t index = 0; index < inputs.size(); ++index) {
        if (index == reference_index || !inputs[index].accepted || !inputs[index].camera) continue;
        auto s = score_one_view(inputs[reference_index], inputs[index], inputs[index].warp, centre, depth,
                                patch_radius);
        if (s) out.push_back(*s);
    }
    return out;
}

// aggregate (depth.rs:1761-1770)
static std::optional<float> aggregate(const std::vector<float> &scores, const Options &options) {
    if (scores.size() < options.minimum_support) return std::nullopt;
    std::vector<float> values = scores;
    std::stable_sort(values.begin(), values.end(),
                     [](float l, float r) { return total_key_f32(r) < total_key_f32(l); });
    values.resize(std::min(options.best_view_count, values.size()));
    if (values.size() >= options.minimum_support) {
        float sum = -0.0f;
        for (float v : values) sum += v;
        return sum / (float)values.size();
    }
    return std::nullopt;
}

// reference_guidance (depth.rs:1824-1832)
static float reference_guidance(const Input &reference, const Vec2 &pixel) {
    auto s = reference.luminance.sample((float)((pixel[0] - 0.5) * 0.5), (float)((pixel[1] - 0.5) * 0.5));
    return s ? *s : 0.0f;
}

static size_t worker_count_for(size_t rows, int threads) {
    size_t automatic = threads > 0 ? (size_t)threads : std::max<size_t>(1, std::thread::hardware_concurrency());
    return std::min(std::max<size_t>(automatic, 1), std::max<size_t>(rows, 1));
}

// Run fn(first_row, last_row) over row bands like thread::scope in the reference.
static void for_row_bands(size_t rows, int threads, const std::function<void(size_t, size_t)> &fn) {
    size_t worker_count = worker_count_for(rows, threads);
    size_t rows_per_worker = div_ceil(rows, worker_count);
    std::vector<std::thread> handles;
    for (size_t first_row = 0; first_row < rows; first_row += rows_per_worker) {
        size_t last_row = std::min(first_row + rows_per_worker, rows);
        handles.emplace_back(fn, first_row, last_row);
    }
    for (auto &h : handles) h.join();
}

struct CostVolume {  // depth.rs:291-299
    std::vector<std::optional<double>> labels;
    std::vector<float> scores, costs, guidance;
    std::vector<uint8_t> tested;
};

// build_cost_volume (depth.rs:1187-1277)
// row_mask (optional, one byte per row) restricts the work to the marked rows; the
// rows are still split into the reference's worker bands, so a mask that marks rows
// in every band keeps every worker busy (the benchmark's bounded samples).
static CostVolume build_cost_volume(const std::vector<Input> &inputs, size_t reference_index, size_t columns,
                                    size_t rows, size_t step, const Options &options, int threads,
                                    const uint8_t *row_mask = nullptr) {
    auto finite_depths = inverse_depth_samples(options.near_depth, options.far_depth, options.planes);
    std::reverse(finite_depths.begin(), finite_depths.end());
    CostVolume v;
    v.labels.push_back(std::nullopt);
    for (double d : finite_depths) v.labels.push_back(d);
    size_t label_count = v.labels.size();
    size_t node_count = columns * rows;
    v.scores.assign(node_count * label_count, 0.0f);
    v.costs.assign(node_count * label_count, 0.0f);
    v.guidance.assign(node_count, 0.0f);
    v.tested.assign(node_count, 0);
    for_row_bands(rows, threads, [&](size_t first_row, size_t last_row) {
        for (size_t row = first_row; row < last_row; ++row) {
            if (row_mask && !row_mask[row]) continue;
            for (size_t column = 0; column < columns; ++column) {
                size_t node = row * columns + column;
                Vec2 p = {(double)(column * step), (double)(row * step)};
                v.guidance[node] = reference_guidance(inputs[reference_index], p);
                bool node_tested = false;
                for (size_t label = 0; label < label_count; ++label) {
                    auto views = score_views(inputs, reference_index, p, v.labels[label], options.patch_radius);
                    auto agg = aggregate(views, options);
                    float score = agg ? *agg : NAN;
                    node_tested |= std::isfinite(score);
                    v.scores[node * label_count + label] = score;
                    float cost;
                    if (std::isfinite(score)) {
                        float near_prior = label == 0 ? 0.0f
                                                      : NEAR_DEPTH_PRIOR * (float)(label - 1) /
                                                            (float)(label_count - 2);
                        cost = fclamp(1.0f - score, 0.0f, 2.0f) + near_prior;
                    } else {
                        cost = MISSING_COST;
                    }
                    v.costs[node * label_count + label] = cost;
                }
                v.tested[node] = node_tested;
            }
        }
    });
    return v;
}

// accumulate_path (depth.rs:1340-1383)
static void accumulate_path(const float *data, const float *guidance, float *output, size_t labels,
                            const std::vector<size_t> &path, std::vector<float> &previous,
                            std::vector<float> &current) {
    for (size_t path_index = 0; path_index < path.size(); ++path_index) {
        size_t node = path[path_index];
        size_t offset = node * labels;
        if (path_index == 0) {
            for (size_t l = 0; l < labels; ++l) previous[l] = data[offset + l];
            for (size_t l = 0; l < labels; ++l) output[offset + l] += previous[l];
            continue;
        }
        size_t previous_node = path[path_index - 1];
        float edge = std::fabs(guidance[node] - guidance[previous_node]);
        float edge_scale = 1.0f / (1.0f + 4.0f * edge);
        float p1 = SGM_SMALL_PENALTY * fmax_r(edge_scale, 0.35f);
        float p2 = SGM_LARGE_PENALTY * fmax_r(edge_scale, 0.12f);
        float minimum_previous = INFINITY;
        for (size_t l = 0; l < labels; ++l) minimum_previous = fmin_r(minimum_previous, previous[l]);
        for (size_t l = 0; l < labels; ++l) {
            float same = previous[l];
            float lower = l > 0 ? previous[l - 1] + p1 : INFINITY;
            float higher = l + 1 < labels ? previous[l + 1] + p1 : INFINITY;
            float jump = minimum_previous + p2;
            current[l] = data[offset + l] + fmin_r(fmin_r(fmin_r(same, lower), higher), jump) - minimum_previous;
            output[offset + l] += current[l];
        }
        std::swap(previous, current);
    }
}

// diagonal_paths (depth.rs:1313-1338)
static std::vector<std::vector<size_t>> diagonal_paths(size_t columns, size_t rows, bool mirrored) {
    std::vector<std::vector<size_t>> paths;
    for (size_t start_column = 0; start_column < columns; ++start_column) {
        std::vector<size_t> path;
        long column = (long)start_column;
        size_t row = 0;
        while (column >= 0 && column < (long)columns && row < rows) {
            path.push_back(row * columns + (size_t)column);
            column += mirrored ? -1 : 1;
            row += 1;
        }
        paths.push_back(path);
    }
    for (size_t start_row = 1; start_row < rows; ++start_row) {
        std::vector<size_t> path;
        long column = mirrored ? (long)columns - 1 : 0;
        size_t row = start_row;
        while (column >= 0 && column < (long)columns && row < rows) {
            path.push_back(row * columns + (size_t)column);
            column += mirrored ? -1 : 1;
            row += 1;
        }
        paths.push_back(path);
    }
    return paths;
}

// semi_global_costs (depth.rs:1279-1311)
static std::vector<float> semi_global_costs(const float *data, const float *guidance, size_t columns, size_t rows,
                                            size_t labels) {
    std::vector<float> output(columns * rows * labels, 0.0f);
    std::vector<float> previous(labels), current(labels);
    std::vector<size_t> forward, reverse;
    for (size_t row = 0; row < rows; ++row) {
        forward.clear();
        for (size_t column = 0; column < columns; ++column) forward.push_back(row * columns + column);
        reverse.assign(forward.rbegin(), forward.rend());
        accumulate_path(data, guidance, output.data(), labels, forward, previous, current);
        accumulate_path(data, guidance, output.data(), labels, reverse, previous, current);
    }
    for (size_t column = 0; column < columns; ++column) {
        forward.clear();
        for (size_t row = 0; row < rows; ++row) forward.push_back(row * columns + column);
        reverse.assign(forward.rbegin(), forward.rend());
        accumulate_path(data, guidance, output.data(), labels, forward, previous, current);
        accumulate_path(data, guidance, output.data(), labels, reverse, previous, current);
    }
    auto down_right = diagonal_paths(columns, rows, false);
    auto down_left = diagonal_paths(columns, rows, true);
    for (int family = 0; family < 2; ++family) {
        const auto &paths = family == 0 ? down_right : down_left;
        for (const auto &path : paths) {
            accumulate_path(data, guidance, output.data(), labels, path, previous, current);
            reverse.assign(path.rbegin(), path.rend());
            accumulate_path(data, guidance, output.data(), labels, reverse, previous, current);
        }
    }
    return output;
}

// sublabel_depth (depth.rs:1469-1488)
static double sublabel_depth(const std::vector<std::optional<double>> &labels, const float *costs,
                             size_t best_label) {
    double centre_depth = *labels[best_label];
    if (best_label <= 1 || best_label + 1 >= labels.size()) return centre_depth;
    float left = costs[best_label - 1], centre = costs[best_label], right = costs[best_label + 1];
    float curvature = left - 2.0f * centre + right;
    if (!std::isfinite(curvature) || curvature <= 1.0e-6f) return centre_depth;
    double offset = (double)fclamp(0.5f * (left - right) / curvature, -0.75f, 0.75f);
    double lower_inverse = 1.0 / *labels[best_label - 1];
    double upper_inverse = 1.0 / *labels[best_label + 1];
    double inverse_step = (upper_inverse - lower_inverse) * 0.5;
    return 1.0 / (1.0 / centre_depth + offset * inverse_step);
}

// select_depths (depth.rs:1385-1467)
static void select_depths(const std::vector<std::optional<double>> &labels_v, const float *scores,
                          const uint8_t *tested, size_t n_nodes, const float *regularised, const Options &options,
                          Field &field, std::vector<uint8_t> &fillable) {
    size_t labels = labels_v.size();
    field.assign(n_nodes, std::nullopt);
    fillable.assign(n_nodes, 0);
    for (size_t node = 0; node < n_nodes; ++node) {
        if (!tested[node]) continue;
        size_t offset = node * labels;
        if (labels < 2) continue;
        size_t best_label = 1;
        float best_cost = regularised[offset + 1];
        for (size_t label = 2; label < labels; ++label) {  // min_by keeps the first minimum
            float c = regularised[offset + label];
            if (total_key_f32(c) < total_key_f32(best_cost)) {
                best_cost = c;
                best_label = label;
            }
        }
        double depth = sublabel_depth(labels_v, regularised + offset, best_label);
        float score = scores[offset + best_label];
        if (!std::isfinite(score) || score < MINIMUM_REGULARIZED_SCORE) {
            fillable[node] = 1;
            continue;
        }
        bool have_competing = false;
        float competing = 0.0f;
        for (size_t label = 1; label < labels; ++label) {
            if (abs_diff(label, best_label) <= 2) continue;
            float c = regularised[offset + label];
            if (!have_competing || total_key_f32(c) < total_key_f32(competing)) {
                competing = c;
                have_competing = true;
            }
        }
        if (!have_competing) competing = best_cost;
        float margin = fmax_r((competing - best_cost) / SGM_DIRECTIONS, 0.0f);
        float baseline = scores[offset];
        float improvement = std::isfinite(baseline) ? score - baseline : 0.0f;
        if (std::isfinite(baseline) && improvement < -MAXIMUM_REGULARIZED_BASELINE_LOSS) continue;
        bool measured = score >= options.minimum_score && improvement >= options.minimum_improvement * 0.5f &&
                        (margin >= options.minimum_margin || improvement >= options.minimum_improvement);
        float score_confidence =
            fclamp((score - options.minimum_score) / fmax_r(1.0f - options.minimum_score, 1.0e-3f), 0.0f, 1.0f);
        float margin_confidence = fclamp(margin / fmax_r(options.minimum_margin, 1.0e-3f), 0.0f, 1.0f);
        float improvement_confidence =
            fclamp(improvement / fmax_r(options.minimum_improvement, 1.0e-3f), 0.0f, 1.0f);
        float confidence =
            measured ? fclamp(0.30f + 0.45f * score_confidence + 0.25f * margin_confidence, 0.0f, 1.0f)
                     : fclamp(0.10f + 0.25f * score_confidence + 0.15f * margin_confidence +
                                  0.10f * improvement_confidence,
                              0.10f, 0.55f);
        field[node] = NodeDepth{depth, confidence, improvement, !measured};
    }
}

// complete_depth_field (depth.rs:1490-1564)
static void complete_depth_field(Field &field, const float *guidance, const uint8_t *fillable, size_t columns,
                                 size_t rows, const Options &options) {
    for (size_t it = 0; it < options.completion_iterations; ++it) {
        Field previous = field;
        bool changed = false;
        for (size_t row = 0; row < rows; ++row) {
            for (size_t column = 0; column < columns; ++column) {
                size_t index = row * columns + column;
                if (previous[index] || !fillable[index]) continue;
                std::vector<std::pair<double, float>> candidates;
                for (int dy = -1; dy <= 1; ++dy) {
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0) continue;
                        long x = (long)column + dx, y = (long)row + dy;
                        if (x < 0 || y < 0 || x >= (long)columns || y >= (long)rows) continue;
                        size_t ni = (size_t)y * columns + (size_t)x;
                        if (!previous[ni]) continue;
                        const NodeDepth &neighbour = *previous[ni];
                        float edge = std::fabs(guidance[index] - guidance[ni]);
                        if (edge > 0.35f) continue;
                        float spatial = (dx != 0 && dy != 0) ? 0.707f : 1.0f;
                        float weight = neighbour.confidence * spatial * std::exp(-3.0f * edge);
                        if (weight >= 0.05f) candidates.push_back({1.0 / neighbour.depth, weight});
                    }
                }
                if (candidates.size() < options.minimum_neighbour_support) continue;
                std::stable_sort(candidates.begin(), candidates.end(), [](const auto &l, const auto &r) {
                    return total_key_f64(l.first) < total_key_f64(r.first);
                });
                float total_weight = -0.0f;
                for (auto &c : candidates) total_weight += c.second;
                float accumulated = 0.0f;
                bool found = false;
                double inverse_depth = 0.0;
                for (auto &c : candidates) {
                    accumulated += c.second;
                    if (accumulated >= total_weight * 0.5f) {
                        inverse_depth = c.first;
                        found = true;
                        break;
                    }
                }
                if (!found) inverse_depth = candidates[candidates.size() / 2].first;
                float maxw = 0.0f;
                for (auto &c : candidates) maxw = fmax_r(maxw, c.second);
                float confidence = fclamp(maxw * 0.92f, 0.15f, 0.75f);
                field[index] = NodeDepth{1.0 / inverse_depth, confidence, 0.0f, true};
                changed = true;
            }
        }
        if (!changed) break;
    }
}

// nearest_coarse_depth (depth.rs:1062-1076)
static std::optional<NodeDepth> nearest_coarse_depth(const Field &coarse, size_t columns, size_t rows, size_t step,
                                                     const Vec2 &pixel) {
    size_t column = sat_usize(dclamp(std::round(pixel[0] / (double)step), 0.0, (double)(columns - 1)));
    size_t row = sat_usize(dclamp(std::round(pixel[1] / (double)step), 0.0, (double)(rows - 1)));
    return coarse[row * columns + column];
}

// direct_depth_candidates (depth.rs:1078-1107)
static std::vector<double> direct_depth_candidates(std::optional<double> seed, double inverse_step,
                                                   const Options &options) {
    double far_inverse = 1.0 / options.far_depth;
    double near_inverse = 1.0 / options.near_depth;
    std::vector<double> depths;
    if (seed) {
        for (int offset = -6; offset <= 6; ++offset) {
            double inv = dclamp(1.0 / *seed + (double)offset * inverse_step * 0.5, far_inverse, near_inverse);
            double depth = 1.0 / inv;
            if (depths.empty() || std::fabs(1.0 / depths.back() - 1.0 / depth) > inverse_step * 0.1)
                depths.push_back(depth);
        }
    } else {
        depths = inverse_depth_samples(options.near_depth, options.far_depth, 32);
        std::reverse(depths.begin(), depths.end());
    }
    return depths;
}

// select_direct_depth (depth.rs:1109-1165)
static std::optional<NodeDepth> select_direct_depth(const double *depths, const std::optional<float> *scores,
                                                    size_t n, std::optional<float> baseline, bool seeded,
                                                    const Options &options) {
    double far_inverse = 1.0 / options.far_depth;
    double inverse_range = 1.0 / options.near_depth - far_inverse;
    struct Ranked {
        size_t index;
        double depth;
        float score, objective;
    };
    std::vector<Ranked> ranked;
    for (size_t index = 0; index < n; ++index) {
        if (!scores[index]) continue;
        float score = *scores[index];
        double near_fraction = dclamp((1.0 / depths[index] - far_inverse) / inverse_range, 0.0, 1.0);
        float objective = score - NEAR_DEPTH_PRIOR * (float)near_fraction;
        ranked.push_back({index, depths[index], score, objective});
    }
    std::stable_sort(ranked.begin(), ranked.end(), [](const Ranked &l, const Ranked &r) {
        return total_key_f32(r.objective) < total_key_f32(l.objective);
    });
    if (ranked.empty()) return std::nullopt;
    const Ranked best = ranked.front();
    float competing = best.objective;
    for (const auto &c : ranked)
        if (abs_diff(c.index, best.index) > 1) {
            competing = c.objective;
            break;
        }
    float margin = fmax_r(best.objective - competing, 0.0f);
    float improvement = baseline ? best.score - *baseline : 0.0f;
    float score_floor = fmax_r(options.minimum_score - 0.03f, MINIMUM_REGULARIZED_SCORE);
    float required_margin = seeded ? options.minimum_margin * 0.6f : options.minimum_margin;
    bool improves_global = !baseline || improvement >= options.minimum_improvement * 0.5f;
    bool supported = best.score >= score_floor && improves_global &&
                     (margin >= required_margin || improvement >= options.minimum_improvement);
    if (!supported) return std::nullopt;
    float score_confidence =
        fclamp((best.score - score_floor) / fmax_r(1.0f - score_floor, 1.0e-3f), 0.0f, 1.0f);
    float margin_confidence = fclamp(margin / fmax_r(required_margin, 1.0e-3f), 0.0f, 1.0f);
    return NodeDepth{best.depth, fclamp(0.30f + 0.45f * score_confidence + 0.25f * margin_confidence, 0.0f, 1.0f),
                     improvement, false};
}

// best_depth_candidate (depth.rs:1167-1185): max_by keeps the last maximum
static std::optional<size_t> best_depth_candidate(const double *depths, const std::optional<float> *scores,
                                                  size_t n, const Options &options) {
    double far_inverse = 1.0 / options.far_depth;
    double inverse_range = 1.0 / options.near_depth - far_inverse;
    std::optional<size_t> best;
    float best_objective = 0.0f;
    for (size_t index = 0; index < n; ++index) {
        if (!scores[index]) continue;
        double near_fraction = dclamp((1.0 / depths[index] - far_inverse) / inverse_range, 0.0, 1.0);
        float objective = *scores[index] - NEAR_DEPTH_PRIOR * (float)near_fraction;
        if (!best || !(total_key_f32(objective) < total_key_f32(best_objective))) {
            best = index;
            best_objective = objective;
        }
    }
    return best;
}

struct DirectField {  // depth.rs:301-308
    size_t columns, rows, step;
    Field nodes;
    std::vector<float> guidance;
    std::vector<uint8_t> tested;
};

// measure_direct_depths (depth.rs:715-876)
static DirectField measure_direct_depths(const std::vector<Input> &inputs, size_t reference_index,
                                         const Field &coarse, size_t coarse_columns, size_t coarse_rows,
                                         size_t coarse_step, double inverse_step, const Options &options,
                                         int threads, const uint8_t *row_mask = nullptr) {
    DirectField out;
    out.step = std::max<size_t>(coarse_step / 2, 4);
    out.columns = div_ceil(inputs[reference_index].width, out.step) + 1;
    out.rows = div_ceil(inputs[reference_index].height, out.step) + 1;
    size_t columns = out.columns, rows = out.rows, step = out.step;
    out.nodes.assign(columns * rows, std::nullopt);
    out.guidance.assign(columns * rows, 0.0f);
    out.tested.assign(columns * rows, 0);
    size_t direct_radius = std::max<size_t>(options.patch_radius, 3);
    size_t wide_radius = std::max<size_t>(options.patch_radius * 2, 8);
    for_row_bands(rows, threads, [&](size_t first_row, size_t last_row) {
        for (size_t row = first_row; row < last_row; ++row) {
            if (row_mask && !row_mask[row]) continue;
            for (size_t column = 0; column < columns; ++column) {
                size_t index = row * columns + column;
                Vec2 p = {(double)(column * step), (double)(row * step)};
                out.guidance[index] = reference_guidance(inputs[reference_index], p);
                auto seed = nearest_coarse_depth(coarse, coarse_columns, coarse_rows, coarse_step, p);
                auto candidates =
                    direct_depth_candidates(seed ? std::optional<double>(seed->depth) : std::nullopt, inverse_step,
                                            options);
                auto baseline =
                    aggregate(score_views(inputs, reference_index, p, std::nullopt, direct_radius), options);
                std::vector<std::optional<float>> scores;
                for (double depth : candidates)
                    scores.push_back(aggregate(score_views(inputs, reference_index, p, depth, direct_radius), options));
                bool node_tested = baseline.has_value();
                for (auto &s : scores) node_tested |= s.has_value();
                auto selected = select_direct_depth(candidates.data(), scores.data(), candidates.size(), baseline,
                                                    seed.has_value(), options);
                if (!selected) {
                    auto best = best_depth_candidate(candidates.data(), scores.data(), candidates.size(), options);
                    if (best && scores[*best] && *scores[*best] >= MINIMUM_REGULARIZED_SCORE) {
                        size_t first = *best >= 3 ? *best - 3 : 0;
                        size_t last = std::min(*best + 3, candidates.size() - 1);
                        auto wide_baseline =
                            aggregate(score_views(inputs, reference_index, p, std::nullopt, wide_radius), options);
                        std::vector<std::optional<float>> wide_scores;
                        for (size_t i = first; i <= last; ++i)
                            wide_scores.push_back(aggregate(
                                score_views(inputs, reference_index, p, candidates[i], wide_radius), options));
                        selected = select_direct_depth(candidates.data() + first, wide_scores.data(),
                                                       last - first + 1, wide_baseline, seed.has_value(), options);
                    }
                }
                out.nodes[index] = selected;
                out.tested[index] = node_tested;
            }
        }
    });
    return out;
}

// reject_isolated_direct_depths (depth.rs:881-924)
static void reject_isolated_direct_depths(Field &field, const float *guidance, size_t columns, size_t rows,
                                          double inverse_tolerance) {
    Field source = field;
    for (size_t row = 0; row < rows; ++row) {
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            if (!source[index]) continue;
            const NodeDepth node = *source[index];
            double inv = 1.0 / node.depth;
            size_t agreeing = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    long x = (long)column + dx, y = (long)row + dy;
                    if (x < 0 || y < 0 || x >= (long)columns || y >= (long)rows) continue;
                    size_t ni = (size_t)y * columns + (size_t)x;
                    if (!source[ni]) continue;
                    float image_edge = std::fabs(guidance[index] - guidance[ni]);
                    if (image_edge <= 0.6f && std::fabs(1.0 / source[ni]->depth - inv) <= inverse_tolerance)
                        agreeing += 1;
                }
            size_t minimum = node.confidence >= 0.75f ? 1 : 2;
            if (agreeing < minimum) field[index] = std::nullopt;
        }
    }
}

// reject_small_direct_components (depth.rs:933-989)
static void reject_small_direct_components(Field &field, const float *guidance, size_t columns, size_t rows,
                                           double inverse_tolerance, size_t minimum_nodes) {
    if (minimum_nodes <= 1) return;
    Field source = field;
    std::vector<uint8_t> visited(source.size(), 0);
    std::vector<size_t> pending, component;
    for (size_t seed = 0; seed < source.size(); ++seed) {
        if (visited[seed] || !source[seed]) continue;
        visited[seed] = 1;
        pending.assign(1, seed);
        component.clear();
        while (!pending.empty()) {
            size_t index = pending.back();
            pending.pop_back();
            component.push_back(index);
            size_t column = index % columns, row = index / columns;
            double inv = 1.0 / source[index]->depth;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    long x = (long)column + dx, y = (long)row + dy;
                    if (x < 0 || y < 0 || x >= (long)columns || y >= (long)rows) continue;
                    size_t neighbour = (size_t)y * columns + (size_t)x;
                    if (visited[neighbour]) continue;
                    if (!source[neighbour]) continue;
                    float image_edge = std::fabs(guidance[index] - guidance[neighbour]);
                    double inverse_difference = std::fabs(1.0 / source[neighbour]->depth - inv);
                    if (image_edge <= 0.6f && inverse_difference <= inverse_tolerance) {
                        visited[neighbour] = 1;
                        pending.push_back(neighbour);
                    }
                }
        }
        if (component.size() < minimum_nodes)
            for (size_t index : component) field[index] = std::nullopt;
    }
}

// fit_local_depth_planes (depth.rs:995-1060)
static void fit_local_depth_planes(Field &field, const float *guidance, size_t columns, size_t rows,
                                   double inverse_tolerance) {
    Field source = field;
    for (size_t row = 0; row < rows; ++row) {
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            if (!source[index]) continue;
            NodeDepth node = *source[index];
            double centre_inverse = 1.0 / node.depth;
            double normal[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            double rhs[3] = {0, 0, 0};
            size_t support = 0;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    long x = (long)column + dx, y = (long)row + dy;
                    if (x < 0 || y < 0 || x >= (long)columns || y >= (long)rows) continue;
                    size_t ni = (size_t)y * columns + (size_t)x;
                    if (!source[ni]) continue;
                    double inv = 1.0 / source[ni]->depth;
                    float image_edge = std::fabs(guidance[index] - guidance[ni]);
                    if (image_edge > 0.6f || std::fabs(inv - centre_inverse) > inverse_tolerance) continue;
                    double spatial = std::exp((double)(-(dx * dx + dy * dy)) / 6.0);
                    double weight = (double)source[ni]->confidence * spatial * std::exp(-2.5 * (double)image_edge);
                    double basis[3] = {1.0, (double)dx, (double)dy};
                    for (int r = 0; r < 3; ++r) {
                        rhs[r] += weight * basis[r] * inv;
                        for (int c = 0; c < 3; ++c) normal[r][c] += weight * basis[r] * basis[c];
                    }
                    support += 1;
                }
            if (support < 6) continue;
            Mat3 n = {{{normal[0][0], normal[0][1], normal[0][2]},
                       {normal[1][0], normal[1][1], normal[1][2]},
                       {normal[2][0], normal[2][1], normal[2][2]}}};
            auto m = inverse(n);
            if (!m) continue;
            double inv = dot((*m)[0], {rhs[0], rhs[1], rhs[2]});
            if (!(std::isfinite(inv) && inv > 0.0)) continue;
            double maximum_adjustment = inverse_tolerance * 0.25;
            inv = dclamp(inv, centre_inverse - maximum_adjustment, centre_inverse + maximum_adjustment);
            node.depth = 1.0 / inv;
            field[index] = node;
        }
    }
}

// NodeWarp (depth.rs:256-271)
struct NodeWarp {
    int kind = CHIARO_NW_UNDEFINED;
    F2 global = {0, 0}, point = {0, 0};
    float confidence = 0.0f;
    bool measured = false;
};

// warp_decisions_agree (depth.rs:682-712)
static bool warp_decisions_agree(int kind, const NodeWarp &centre, const NodeWarp &neighbour) {
    if (kind == 0 && centre.kind == CHIARO_NW_REFINED && neighbour.kind == CHIARO_NW_REFINED) {
        F2 cd = {centre.point[0] - centre.global[0], centre.point[1] - centre.global[1]};
        F2 nd = {neighbour.point[0] - neighbour.global[0], neighbour.point[1] - neighbour.global[1]};
        float dx = cd[0] - nd[0], dy = cd[1] - nd[1];
        return dx * dx + dy * dy <= 9.0f;
    }
    if (kind == 1 && centre.kind == CHIARO_NW_OCCLUDED && neighbour.kind == CHIARO_NW_OCCLUDED) return true;
    return false;
}

// enforce_warp_consensus (depth.rs:582-618)
static void enforce_warp_consensus(std::vector<NodeWarp> &decisions, size_t columns, size_t rows) {
    std::vector<NodeWarp> source = decisions;
    for (size_t row = 0; row < rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            int kind;
            size_t minimum_neighbours;
            const NodeWarp &s = source[index];
            if (s.kind == CHIARO_NW_REFINED) {
                kind = 0;
                minimum_neighbours = s.measured ? 2 : 4;
            } else if (s.kind == CHIARO_NW_OCCLUDED) {
                kind = 1;
                minimum_neighbours = s.measured ? 3 : 5;
            } else {
                continue;
            }
            size_t neighbours = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    long x = (long)column + dx, y = (long)row + dy;
                    if (x < 0 || y < 0 || x >= (long)columns || y >= (long)rows) continue;
                    neighbours += warp_decisions_agree(kind, s, source[(size_t)y * columns + (size_t)x]) ? 1 : 0;
                }
            if (neighbours < minimum_neighbours) {
                NodeWarp g;
                g.kind = CHIARO_NW_GLOBAL;
                g.global = s.global;
                g.point = s.global;
                decisions[index] = g;
            }
        }
}

// warp_mapping (depth.rs:674-680)
static bool warp_mapping(const NodeWarp &d, F2 &global, F2 &point) {
    if (d.kind == CHIARO_NW_GLOBAL) {
        global = d.global;
        point = d.global;
        return true;
    }
    if (d.kind == CHIARO_NW_REFINED) {
        global = d.global;
        point = d.point;
        return true;
    }
    return false;
}

// suppress_warp_boundaries (depth.rs:620-672)
static void suppress_warp_boundaries(std::vector<NodeWarp> &decisions, const float *guidance, size_t columns,
                                     size_t rows) {
    std::vector<NodeWarp> source = decisions;
    std::vector<uint8_t> boundary(decisions.size(), 0);
    for (size_t row = 0; row < rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            F2 global, point;
            if (!warp_mapping(source[index], global, point)) continue;
            F2 delta = {point[0] - global[0], point[1] - global[1]};
            const size_t nbr[2][2] = {{column + 1, row}, {column, row + 1}};
            for (int k = 0; k < 2; ++k) {
                size_t x = nbr[k][0], y = nbr[k][1];
                if (x >= columns || y >= rows) continue;
                size_t ni = y * columns + x;
                F2 ng, np;
                if (!warp_mapping(source[ni], ng, np)) continue;
                F2 nd = {np[0] - ng[0], np[1] - ng[1]};
                F2 diff = {delta[0] - nd[0], delta[1] - nd[1]};
                bool mapping_edge =
                    diff[0] * diff[0] + diff[1] * diff[1] > WARP_BOUNDARY_DELTA_PX * WARP_BOUNDARY_DELTA_PX;
                bool image_edge = std::fabs(guidance[index] - guidance[ni]) > WARP_BOUNDARY_CONTRAST;
                if (mapping_edge && image_edge) {
                    boundary[index] = 1;
                    boundary[ni] = 1;
                }
            }
        }
    for (size_t index = 0; index < boundary.size(); ++index) {
        if (!boundary[index]) continue;
        F2 global, point;
        if (!warp_mapping(source[index], global, point)) continue;
        NodeWarp b;
        b.kind = CHIARO_NW_BOUNDARY;
        b.global = global;
        decisions[index] = b;
    }
}

// score_one_view_at_point (depth.rs:1710-1736)
static std::optional<float> score_one_view_at_point(const Input &reference, const Input &target, const Warp &global,
                                                    const Vec2 &centre, const F2 &global_point, const F2 &point,
                                                    size_t patch_radius) {
    Vec2 delta = {(double)(point[0] - global_point[0]), (double)(point[1] - global_point[1])};
    if (std::fabs(delta[0]) > 128.0 || std::fabs(delta[1]) > 128.0) return std::nullopt;
    return warped_patch_zncc(reference.luminance, target.luminance, global, centre, delta, patch_radius);
}

struct ViewRefinement {
    float score;
    F2 point;
};

// refine_one_view (depth.rs:1634-1708)
static std::optional<ViewRefinement> refine_one_view(const Input &reference, const Input &target,
                                                     const Warp &global, const Vec2 &centre, double shared_depth,
                                                     double inverse_step, const Options &options) {
    if (!reference.camera || !target.camera) return std::nullopt;
    auto global_point = global.map((float)centre[0], (float)centre[1]);
    if (!global_point) return std::nullopt;
    double min_inverse = 1.0 / options.far_depth;
    double max_inverse = 1.0 / options.near_depth;
    double shared_inverse = 1.0 / shared_depth;
    bool have_best = false;
    float best_objective = 0.0f, best_score = 0.0f;
    F2 best_point = {0, 0};
    const double offsets[5] = {-1.0, -0.5, 0.0, 0.5, 1.0};
    for (double label_offset : offsets) {
        double inv = dclamp(shared_inverse + label_offset * inverse_step, min_inverse, max_inverse);
        auto point64 = map_at_depth(*reference.camera, *target.camera, global, centre, 1.0 / inv);
        if (!point64) return std::nullopt;
        F2 point = {(float)(*point64)[0], (float)(*point64)[1]};
        auto score =
            score_one_view_at_point(reference, target, global, centre, *global_point, point, options.patch_radius);
        if (!score) return std::nullopt;
        float objective = *score - (float)std::fabs(label_offset) * 0.002f;
        if (!have_best || objective > best_objective) {
            have_best = true;
            best_objective = objective;
            best_score = *score;
            best_point = point;
        }
    }
    F2 depth_point = best_point;
    float b0 = best_score, b1 = best_score;
    F2 b2 = depth_point;
    const float shifts[3] = {-1.5f, 0.0f, 1.5f};
    for (float dy : shifts)
        for (float dx : shifts) {
            if (dx == 0.0f && dy == 0.0f) continue;
            F2 point = {depth_point[0] + dx, depth_point[1] + dy};
            auto score =
                score_one_view_at_point(reference, target, global, centre, *global_point, point, options.patch_radius);
            if (!score) return std::nullopt;
            float residual_sq = dx * dx + dy * dy;
            float objective = *score - residual_sq * 0.002f;
            if (objective > b0) {
                b0 = objective;
                b1 = *score;
                b2 = point;
            }
        }
    return ViewRefinement{b1, b2};
}

static float fraction(size_t count, size_t total) { return total == 0 ? 0.0f : (float)count / (float)total; }

struct Result {
    size_t columns, rows, step;
    Field field;
    std::vector<uint8_t> tested;
};

// Per-target decisions for one target (depth.rs:427-489), returning the
// filtered decision list.
// row_of (optional) gives the raster row index of each grid row, for a grid of
// sampled rows stacked together.
static std::vector<NodeWarp> target_decisions(const std::vector<Input> &inputs, size_t reference_index,
                                              size_t target_index, const Field &field, const float *guidance,
                                              size_t columns, size_t rows, size_t step, double inverse_step,
                                              const Options &options, const size_t *row_of = nullptr) {
    const Input &reference = inputs[reference_index];
    const Warp &global = inputs[target_index].warp;
    std::vector<NodeWarp> decisions(columns * rows);
    for (size_t row = 0; row < rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            Vec2 p = {(double)(column * step), (double)((row_of ? row_of[row] : row) * step)};
            NodeWarp &d = decisions[index];
            auto global_q = global.map((float)p[0], (float)p[1]);
            if (!global_q) {
                d.kind = CHIARO_NW_UNDEFINED;
                continue;
            }
            if (!field[index]) {
                d.kind = CHIARO_NW_GLOBAL;
                d.global = *global_q;
                d.point = *global_q;
                continue;
            }
            const NodeDepth node = *field[index];
            auto selected =
                refine_one_view(reference, inputs[target_index], global, p, node.depth, inverse_step, options);
            auto baseline =
                score_one_view(reference, inputs[target_index], global, p, std::nullopt, options.patch_radius);
            bool supported = selected && selected->score >= options.minimum_score &&
                             (!baseline || selected->score + 0.01f >= *baseline);
            bool contradicted = selected && baseline && selected->score + 0.12f < *baseline;
            if (contradicted) {
                d.kind = CHIARO_NW_OCCLUDED;
                d.global = *global_q;
                d.measured = !node.regularized;
            } else if (supported) {
                d.kind = CHIARO_NW_REFINED;
                d.global = *global_q;
                d.point = selected->point;
                d.confidence = node.regularized ? node.confidence * 0.6f : 0.5f + 0.5f * node.confidence;
                d.measured = !node.regularized;
            } else {
                d.kind = CHIARO_NW_GLOBAL;
                d.global = *global_q;
                d.point = *global_q;
            }
        }
    enforce_warp_consensus(decisions, columns, rows);
    suppress_warp_boundaries(decisions, guidance, columns, rows);
    return decisions;
}

static std::vector<Input> make_inputs(const chiaro_view *views, size_t n_views) {
    std::vector<Input> inputs(n_views);
    for (size_t i = 0; i < n_views; ++i) {
        const chiaro_view &v = views[i];
        inputs[i].luminance.width = (size_t)v.luma_width;
        inputs[i].luminance.height = (size_t)v.luma_height;
        inputs[i].luminance.data = v.luminance;
        inputs[i].width = (size_t)v.width;
        inputs[i].height = (size_t)v.height;
        if (v.has_camera) inputs[i].camera.emplace(v.camera);
        inputs[i].accepted = v.accepted != 0;
        inputs[i].warp.step = (size_t)v.warp.step;
        inputs[i].warp.columns = (size_t)v.warp.columns;
        inputs[i].warp.rows = (size_t)v.warp.rows;
        inputs[i].warp.points = v.warp.points;
    }
    return inputs;
}

static void field_to_arrays(const Field &f, uint8_t *has, double *depth, float *confidence, float *improvement,
                            uint8_t *regularized) {
    for (size_t i = 0; i < f.size(); ++i) {
        if (has) has[i] = f[i].has_value();
        if (depth) depth[i] = f[i] ? f[i]->depth : NAN;
        if (confidence) confidence[i] = f[i] ? f[i]->confidence : 0.0f;
        if (improvement) improvement[i] = f[i] ? f[i]->improvement : 0.0f;
        if (regularized) regularized[i] = f[i] ? f[i]->regularized : 0;
    }
}

static Field arrays_to_field(size_t n, const uint8_t *has, const double *depth, const float *confidence,
                             const float *improvement, const uint8_t *regularized) {
    Field f(n);
    for (size_t i = 0; i < n; ++i)
        if (has[i])
            f[i] = NodeDepth{depth[i], confidence ? confidence[i] : 0.0f, improvement ? improvement[i] : 0.0f,
                             regularized ? regularized[i] != 0 : false};
    return f;
}

// refine_multiview_depth (depth.rs:312-580)
static int refine_multiview_depth(const chiaro_view *views, size_t n_views, size_t reference_index,
                                  const chiaro_depth_options *opt, chiaro_warp *refined, chiaro_depth_report *reports,
                                  chiaro_depth_map *out_map, const chiaro_depth_debug *debug, int threads) {
    Options options(*opt);
    if (!valid_options(options) || reference_index >= n_views || !views[reference_index].has_camera)
        return CHIARO_INVALID;
    auto inputs = make_inputs(views, n_views);
    const Input &reference = inputs[reference_index];
    size_t coarse_step = std::max<size_t>(options.grid_step, 4);
    size_t coarse_columns = div_ceil(reference.width, coarse_step) + 1;
    size_t coarse_rows = div_ceil(reference.height, coarse_step) + 1;
    CostVolume volume =
        build_cost_volume(inputs, reference_index, coarse_columns, coarse_rows, coarse_step, options, threads);
    size_t nl = volume.labels.size(), nn = coarse_columns * coarse_rows;
    std::vector<float> regularised =
        semi_global_costs(volume.costs.data(), volume.guidance.data(), coarse_columns, coarse_rows, nl);
    Field coarse_field;
    std::vector<uint8_t> fillable;
    select_depths(volume.labels, volume.scores.data(), volume.tested.data(), nn, regularised.data(), options,
                  coarse_field, fillable);
    double inverse_step = (1.0 / options.near_depth - 1.0 / options.far_depth) / (double)(options.planes - 1);
    if (options.completion_iterations > 0)
        complete_depth_field(coarse_field, volume.guidance.data(), fillable.data(), coarse_columns, coarse_rows,
                             options);
    if (debug) {
        if (debug->coarse_scores) std::memcpy(debug->coarse_scores, volume.scores.data(), nn * nl * 4);
        if (debug->coarse_costs) std::memcpy(debug->coarse_costs, volume.costs.data(), nn * nl * 4);
        if (debug->coarse_guidance) std::memcpy(debug->coarse_guidance, volume.guidance.data(), nn * 4);
        if (debug->coarse_tested) std::memcpy(debug->coarse_tested, volume.tested.data(), nn);
        if (debug->regularised) std::memcpy(debug->regularised, regularised.data(), nn * nl * 4);
        field_to_arrays(coarse_field, debug->coarse_has, debug->coarse_depth, debug->coarse_confidence,
                        debug->coarse_improvement, debug->coarse_regularized);
        if (debug->coarse_fillable) std::memcpy(debug->coarse_fillable, fillable.data(), nn);
    }
    regularised.clear();
    regularised.shrink_to_fit();

    DirectField direct = measure_direct_depths(inputs, reference_index, coarse_field, coarse_columns, coarse_rows,
                                               coarse_step, inverse_step, options, threads);
    size_t columns = direct.columns, rows = direct.rows, step = direct.step, m = columns * rows;
    Field &field = direct.nodes;
    if (debug) {
        field_to_arrays(field, debug->direct_has, debug->direct_depth, debug->direct_confidence,
                        debug->direct_improvement, debug->direct_regularized);
        if (debug->direct_guidance) std::memcpy(debug->direct_guidance, direct.guidance.data(), m * 4);
        if (debug->direct_tested) std::memcpy(debug->direct_tested, direct.tested.data(), m);
    }
    reject_isolated_direct_depths(field, direct.guidance.data(), columns, rows, inverse_step * 2.5);
    if (debug && debug->isolated_has)
        for (size_t i = 0; i < m; ++i) debug->isolated_has[i] = field[i].has_value();
    reject_small_direct_components(field, direct.guidance.data(), columns, rows, inverse_step * 2.5,
                                   MINIMUM_DIRECT_COMPONENT_NODES);
    if (debug && debug->component_has)
        for (size_t i = 0; i < m; ++i) debug->component_has[i] = field[i].has_value();
    fit_local_depth_planes(field, direct.guidance.data(), columns, rows, inverse_step * 4.0);
    if (debug && debug->fitted_depth)
        for (size_t i = 0; i < m; ++i) debug->fitted_depth[i] = field[i] ? field[i]->depth : NAN;

    size_t tested_nodes = 0, measured_nodes = 0, regularized_nodes = 0;
    std::vector<double> selected_depths;
    std::vector<float> improvements;
    for (size_t i = 0; i < m; ++i) {
        tested_nodes += direct.tested[i] ? 1 : 0;
        if (!field[i]) continue;
        selected_depths.push_back(field[i]->depth);
        if (field[i]->regularized)
            regularized_nodes += 1;
        else {
            measured_nodes += 1;
            improvements.push_back(field[i]->improvement);
        }
    }
    size_t fallback_nodes =
        tested_nodes >= measured_nodes + regularized_nodes ? tested_nodes - (measured_nodes + regularized_nodes) : 0;
    std::stable_sort(selected_depths.begin(), selected_depths.end(),
                     [](double l, double r) { return total_key_f64(l) < total_key_f64(r); });
    std::stable_sort(improvements.begin(), improvements.end(),
                     [](float l, float r) { return total_key_f32(l) < total_key_f32(r); });

    for (size_t target_index = 0; target_index < n_views; ++target_index) {
        if (reports) reports[target_index].present = 0;
        if (target_index == reference_index || !inputs[target_index].accepted || !inputs[target_index].camera)
            continue;
        auto decisions = target_decisions(inputs, reference_index, target_index, field, direct.guidance.data(),
                                          columns, rows, step, inverse_step, options);
        size_t refined_nodes = 0, occluded_nodes = 0, boundary_nodes = 0;
        if (debug && debug->decision_kind)
            for (size_t i = 0; i < m; ++i) debug->decision_kind[target_index * m + i] = (uint8_t)decisions[i].kind;
        if (refined) {
            chiaro_warp &w = refined[target_index];
            if (w.capacity < m || !w.points || !w.confidence) return CHIARO_ERR_CAPACITY;
            w.step = step;
            w.columns = columns;
            w.rows = rows;
            for (size_t i = 0; i < m; ++i) {
                const NodeWarp &d = decisions[i];
                float px = 0, py = 0, c = 0;
                switch (d.kind) {
                    case CHIARO_NW_UNDEFINED: px = py = NAN; c = 0.0f; break;
                    case CHIARO_NW_GLOBAL: px = d.global[0]; py = d.global[1]; c = 1.0f; break;
                    case CHIARO_NW_REFINED: px = d.point[0]; py = d.point[1]; c = d.confidence; break;
                    case CHIARO_NW_OCCLUDED:
                    case CHIARO_NW_BOUNDARY: px = d.global[0]; py = d.global[1]; c = 0.0f; break;
                }
                w.points[2 * i] = px;
                w.points[2 * i + 1] = py;
                w.confidence[i] = c;
            }
        }
        for (size_t i = 0; i < m; ++i) {
            refined_nodes += decisions[i].kind == CHIARO_NW_REFINED;
            occluded_nodes += decisions[i].kind == CHIARO_NW_OCCLUDED;
            boundary_nodes += decisions[i].kind == CHIARO_NW_BOUNDARY;
        }
        if (reports) {
            chiaro_depth_report &r = reports[target_index];
            r.present = 1;
            r.tested_nodes = tested_nodes;
            r.measured_nodes = measured_nodes;
            r.regularized_nodes = regularized_nodes;
            r.fallback_nodes = fallback_nodes;
            r.refined_nodes = refined_nodes;
            r.occluded_nodes = occluded_nodes;
            r.boundary_nodes = boundary_nodes;
            r.reconstructed_fraction = fraction(measured_nodes + regularized_nodes, tested_nodes);
            r.refined_fraction = fraction(refined_nodes, tested_nodes);
            r.occluded_fraction = fraction(occluded_nodes, tested_nodes);
            r.has_median_depth = !selected_depths.empty();
            r.median_depth = selected_depths.empty() ? 0.0 : selected_depths[selected_depths.size() / 2];
            r.has_median_score_improvement = !improvements.empty();
            r.median_score_improvement = improvements.empty() ? 0.0f : improvements[improvements.size() / 2];
        }
    }
    if (out_map) {
        if (out_map->capacity < m || !out_map->depth || !out_map->confidence || !out_map->provenance)
            return CHIARO_ERR_CAPACITY;
        out_map->columns = columns;
        out_map->rows = rows;
        out_map->step = step;
        out_map->near_depth = options.near_depth;
        out_map->far_depth = options.far_depth;
        for (size_t i = 0; i < m; ++i) {
            if (field[i]) {
                out_map->depth[i] = field[i]->depth;
                out_map->confidence[i] = field[i]->confidence;
                out_map->provenance[i] = field[i]->regularized ? CHIARO_REGULARIZED : CHIARO_MEASURED;
            } else if (direct.tested[i]) {
                out_map->depth[i] = NAN;
                out_map->confidence[i] = 1.0f;
                out_map->provenance[i] = CHIARO_GLOBAL;
            } else {
                out_map->depth[i] = NAN;
                out_map->confidence[i] = 0.0f;
                out_map->provenance[i] = CHIARO_UNSUPPORTED;
            }
        }
    }
    return CHIARO_OK;
}

// DenseDepthMap::diagnostic_samples (depth.rs:200-222) and helpers
static uint16_t round_u16(double v) {  // f64::round() as u16 (saturating)
    double r = std::round(v);
    if (!(r > 0.0)) return 0;
    if (r >= 65535.0) return 65535;
    return (uint16_t)r;
}
static void scale_color(const uint16_t c[3], double s, uint16_t out[3]) {  // depth.rs:1857-1859
    for (int i = 0; i < 3; ++i) out[i] = round_u16((double)c[i] * s);
}
static void depth_color(double normalized, uint16_t out[3]) {  // depth.rs:1861-1877
    static const double stops[5][3] = {
        {0.0, 0.1, 0.7}, {0.0, 0.9, 1.0}, {0.0, 1.0, 0.2}, {1.0, 0.9, 0.0}, {1.0, 0.0, 0.0}};
    double position = dclamp(normalized, 0.0, 1.0) * 4.0;
    size_t lower = std::min<size_t>(sat_usize(std::floor(position)), 4);
    size_t upper = std::min<size_t>(lower + 1, 4);
    double fr = position - (double)lower;
    for (int ch = 0; ch < 3; ++ch)
        out[ch] = round_u16((stops[lower][ch] * (1.0 - fr) + stops[upper][ch] * fr) * 65535.0);
}

}  // namespace oracle

// ---------------------------------------------------------------------------
// C entry points (test infrastructure).
// ---------------------------------------------------------------------------
using namespace oracle;

extern "C" {

void oracle_options_default(chiaro_depth_options *o) { default_options(o); }
int oracle_options_valid(const chiaro_depth_options *o) { return valid_options(Options(*o)) ? 1 : 0; }

int oracle_refine_multiview_depth(const chiaro_view *views, size_t n_views, size_t reference_index,
                                  const chiaro_depth_options *options, chiaro_warp *refined,
                                  chiaro_depth_report *reports, chiaro_depth_map *out_map,
                                  const chiaro_depth_debug *debug, int threads) {
    return refine_multiview_depth(views, n_views, reference_index, options, refined, reports, out_map, debug,
                                  threads);
}

void oracle_inverse_depth_samples(double near_d, double far_d, size_t count, double *out) {
    auto v = inverse_depth_samples(near_d, far_d, count);
    std::memcpy(out, v.data(), count * sizeof(double));
}

// labels: NaN = None.
double oracle_sublabel_depth(const double *labels, size_t n, const float *costs, size_t best) {
    std::vector<std::optional<double>> l(n);
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(labels[i])) l[i] = labels[i];
    return sublabel_depth(l, costs, best);
}

int oracle_aggregate(const float *scores, size_t n, const chiaro_depth_options *opt, float *out) {
    auto r = aggregate(std::vector<float>(scores, scores + n), Options(*opt));
    if (r) *out = *r;
    return r.has_value();
}

void oracle_semi_global_costs(const float *data, const float *guidance, size_t columns, size_t rows, size_t labels,
                              float *out) {
    auto v = semi_global_costs(data, guidance, columns, rows, labels);
    std::memcpy(out, v.data(), v.size() * 4);
}

// Flattened diagonal paths: indices and per-path lengths; returns path count.
size_t oracle_diagonal_paths(size_t columns, size_t rows, int mirrored, size_t *indices, size_t *lengths) {
    auto paths = diagonal_paths(columns, rows, mirrored != 0);
    size_t k = 0;
    for (size_t i = 0; i < paths.size(); ++i) {
        lengths[i] = paths[i].size();
        for (size_t v : paths[i]) indices[k++] = v;
    }
    return paths.size();
}

void oracle_select_depths(const double *labels, size_t n_labels, const float *scores, const float *regularised,
                          const uint8_t *tested, size_t n_nodes, const chiaro_depth_options *opt, uint8_t *has,
                          double *depth, float *confidence, float *improvement, uint8_t *regularized,
                          uint8_t *fillable) {
    std::vector<std::optional<double>> l(n_labels);
    for (size_t i = 0; i < n_labels; ++i)
        if (!std::isnan(labels[i])) l[i] = labels[i];
    Field f;
    std::vector<uint8_t> fill;
    select_depths(l, scores, tested, n_nodes, regularised, Options(*opt), f, fill);
    field_to_arrays(f, has, depth, confidence, improvement, regularized);
    std::memcpy(fillable, fill.data(), n_nodes);
}

void oracle_complete_depth_field(uint8_t *has, double *depth, float *confidence, float *improvement,
                                 uint8_t *regularized, const float *guidance, const uint8_t *fillable,
                                 size_t columns, size_t rows, const chiaro_depth_options *opt) {
    size_t n = columns * rows;
    Field f = arrays_to_field(n, has, depth, confidence, improvement, regularized);
    complete_depth_field(f, guidance, fillable, columns, rows, Options(*opt));
    field_to_arrays(f, has, depth, confidence, improvement, regularized);
}

void oracle_reject_isolated(uint8_t *has, const double *depth, const float *confidence, const float *guidance,
                            size_t columns, size_t rows, double tol) {
    size_t n = columns * rows;
    Field f = arrays_to_field(n, has, depth, confidence, nullptr, nullptr);
    reject_isolated_direct_depths(f, guidance, columns, rows, tol);
    for (size_t i = 0; i < n; ++i) has[i] = f[i].has_value();
}

void oracle_reject_small_components(uint8_t *has, const double *depth, const float *guidance, size_t columns,
                                    size_t rows, double tol, size_t minimum_nodes) {
    size_t n = columns * rows;
    Field f = arrays_to_field(n, has, depth, nullptr, nullptr, nullptr);
    reject_small_direct_components(f, guidance, columns, rows, tol, minimum_nodes);
    for (size_t i = 0; i < n; ++i) has[i] = f[i].has_value();
}

void oracle_fit_local_planes(const uint8_t *has, double *depth, const float *confidence, const float *guidance,
                             size_t columns, size_t rows, double tol) {
    size_t n = columns * rows;
    Field f = arrays_to_field(n, has, depth, confidence, nullptr, nullptr);
    fit_local_depth_planes(f, guidance, columns, rows, tol);
    for (size_t i = 0; i < n; ++i)
        if (f[i]) depth[i] = f[i]->depth;
}

// scores: NaN = None. has_baseline selects Some(baseline). Returns 1 when Some.
int oracle_select_direct_depth(const double *depths, const float *scores, size_t n, int has_baseline,
                               float baseline, int seeded, const chiaro_depth_options *opt, double *out_depth,
                               float *out_confidence, float *out_improvement) {
    std::vector<std::optional<float>> s(n);
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(scores[i])) s[i] = scores[i];
    auto r = select_direct_depth(depths, s.data(), n, has_baseline ? std::optional<float>(baseline) : std::nullopt,
                                 seeded != 0, Options(*opt));
    if (!r) return 0;
    *out_depth = r->depth;
    *out_confidence = r->confidence;
    *out_improvement = r->improvement;
    return 1;
}

// Returns index or -1 (None).
long oracle_best_depth_candidate(const double *depths, const float *scores, size_t n,
                                 const chiaro_depth_options *opt) {
    std::vector<std::optional<float>> s(n);
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(scores[i])) s[i] = scores[i];
    auto r = best_depth_candidate(depths, s.data(), n, Options(*opt));
    return r ? (long)*r : -1;
}

static std::vector<NodeWarp> decisions_from(size_t n, const uint8_t *kind, const float *global, const float *point,
                                            const uint8_t *measured) {
    std::vector<NodeWarp> d(n);
    for (size_t i = 0; i < n; ++i) {
        d[i].kind = kind[i];
        d[i].global = {global[2 * i], global[2 * i + 1]};
        d[i].point = {point[2 * i], point[2 * i + 1]};
        d[i].measured = measured[i] != 0;
    }
    return d;
}

int oracle_warp_decisions_agree(int kind, int c_kind, const float *c_global, const float *c_point, int n_kind,
                                const float *n_global, const float *n_point) {
    NodeWarp c, n;
    c.kind = c_kind;
    c.global = {c_global[0], c_global[1]};
    c.point = {c_point[0], c_point[1]};
    n.kind = n_kind;
    n.global = {n_global[0], n_global[1]};
    n.point = {n_point[0], n_point[1]};
    return warp_decisions_agree(kind, c, n) ? 1 : 0;
}

void oracle_warp_decisions_filter(uint8_t *kind, float *global, float *point, const uint8_t *measured,
                                  const float *guidance, size_t columns, size_t rows, int consensus,
                                  int boundaries) {
    size_t n = columns * rows;
    auto d = decisions_from(n, kind, global, point, measured);
    if (consensus) enforce_warp_consensus(d, columns, rows);
    if (boundaries) suppress_warp_boundaries(d, guidance, columns, rows);
    for (size_t i = 0; i < n; ++i) {
        kind[i] = (uint8_t)d[i].kind;
        global[2 * i] = d[i].global[0];
        global[2 * i + 1] = d[i].global[1];
        point[2 * i] = d[i].point[0];
        point[2 * i + 1] = d[i].point[1];
    }
}

// diagnostic_samples (depth.rs:200-222): depth_out[n], provenance_out[3n].
void oracle_diagnostic_samples(const chiaro_depth_map *map, uint16_t *depth_out, uint16_t *provenance_out) {
    double near_inverse = 1.0 / map->near_depth, far_inverse = 1.0 / map->far_depth;
    double range = dmax_r(near_inverse - far_inverse, 2.2250738585072014e-308);
    size_t n = map->columns * map->rows;
    for (size_t i = 0; i < n; ++i) {
        bool has = map->provenance[i] == CHIARO_MEASURED || map->provenance[i] == CHIARO_REGULARIZED;
        uint16_t encoded = 0;
        if (has) {
            double normalized = dclamp((1.0 / map->depth[i] - far_inverse) / range, 0.0, 1.0);
            encoded = (uint16_t)(1 + round_u16(normalized * 65534.0));
        }
        depth_out[i] = encoded;
        double confidence = (double)(0.35f + 0.65f * fclamp(map->confidence[i], 0.0f, 1.0f));
        uint16_t color[3] = {0, 0, 0};
        static const uint16_t green[3] = {0, 65535, 0}, amber[3] = {65535, 32768, 0};
        switch (map->provenance[i]) {
            case CHIARO_UNSUPPORTED: break;
            case CHIARO_GLOBAL: color[2] = 32768; break;
            case CHIARO_MEASURED: scale_color(green, confidence, color); break;
            case CHIARO_REGULARIZED: scale_color(amber, confidence, color); break;
        }
        for (int c = 0; c < 3; ++c) provenance_out[3 * i + c] = color[c];
    }
}

// visualization_samples (depth.rs:224-245): out[3n].
void oracle_visualization_samples(const chiaro_depth_map *map, uint16_t *out) {
    double log_range = std::log(map->far_depth / map->near_depth);
    size_t n = map->columns * map->rows;
    for (size_t i = 0; i < n; ++i) {
        bool has = map->provenance[i] == CHIARO_MEASURED || map->provenance[i] == CHIARO_REGULARIZED;
        uint16_t color[3] = {0, 0, 0};
        if (has) {
            double normalized =
                dclamp((std::log(map->far_depth) - std::log(map->depth[i])) / log_range, 0.0, 1.0);
            double confidence = 0.45 + 0.55 * (double)fclamp(map->confidence[i], 0.0f, 1.0f);
            uint16_t base[3];
            depth_color(normalized, base);
            scale_color(base, confidence, color);
        } else if (map->provenance[i] == CHIARO_GLOBAL) {
            color[2] = 12000;
        }
        for (int c = 0; c < 3; ++c) out[3 * i + c] = color[c];
    }
}

// geometry.rs helpers for the distortion round-trip and camera fixtures.
void oracle_distort(const chiaro_camera *cam, const double *in, double *out) {
    Camera c(*cam);
    auto v = distort(c.distortion, {in[0], in[1]});
    out[0] = v[0];
    out[1] = v[1];
}
void oracle_undistort(const chiaro_camera *cam, const double *in, double *out) {
    Camera c(*cam);
    auto v = undistort(c.distortion, {in[0], in[1]});
    out[0] = v[0];
    out[1] = v[1];
}
void oracle_pixel_to_ray(const chiaro_camera *cam, const double *pixel, double *origin, double *direction) {
    Camera c(*cam);
    Ray r = c.pixel_to_ray({pixel[0], pixel[1]});
    for (int i = 0; i < 3; ++i) {
        origin[i] = r.origin[i];
        direction[i] = r.direction[i];
    }
}
int oracle_project(const chiaro_camera *cam, const double *point, double *out) {
    Camera c(*cam);
    auto v = c.project({point[0], point[1], point[2]});
    if (!v) return 0;
    out[0] = (*v)[0];
    out[1] = (*v)[1];
    return 1;
}
int oracle_map_from(const chiaro_camera *target, const chiaro_camera *reference, const double *pixel, double depth,
                    double *out) {
    Camera t(*target), r(*reference);
    auto v = t.map_from(r, {pixel[0], pixel[1]}, depth);
    if (!v) return 0;
    out[0] = (*v)[0];
    out[1] = (*v)[1];
    return 1;
}

int oracle_warp_map(const chiaro_warp *w, float x, float y, float *out) {
    Warp warp;
    warp.step = (size_t)w->step;
    warp.columns = (size_t)w->columns;
    warp.rows = (size_t)w->rows;
    warp.points = w->points;
    auto v = warp.map(x, y);
    if (!v) return 0;
    out[0] = (*v)[0];
    out[1] = (*v)[1];
    return 1;
}

// Warp::magnification (align.rs:133-143); returns 0 for None.
int oracle_warp_magnification(const chiaro_warp *w, float x, float y, float *out) {
    Warp warp;
    warp.step = (size_t)w->step;
    warp.columns = (size_t)w->columns;
    warp.rows = (size_t)w->rows;
    warp.points = w->points;
    float h = (float)warp.step;
    auto a = warp.map(x, y), b = warp.map(x + h, y), c = warp.map(x, y + h);
    if (!a || !b || !c) return 0;
    // powi(2) lowers to a single multiplication
    float bx = (*b)[0] - (*a)[0], by = (*b)[1] - (*a)[1], cx = (*c)[0] - (*a)[0], cy = (*c)[1] - (*a)[1];
    float dx = std::sqrt(bx * bx + by * by) / h;
    float dy = std::sqrt(cx * cx + cy * cy) / h;
    *out = fmax_r(std::sqrt(dx * dy), 1e-6f);
    return 1;
}

float oracle_plane_sample(const float *data, size_t width, size_t height, float x, float y, int *ok) {
    Plane p;
    p.width = width;
    p.height = height;
    p.data = data;
    auto v = p.sample(x, y);
    *ok = v.has_value();
    return v ? *v : 0.0f;
}

// One view's ZNCC score through score_one_view (depth.rs:1593-1627); depth NaN = None.
int oracle_score_one_view(const chiaro_view *views, size_t n_views, size_t reference_index, size_t target_index,
                          double cx, double cy, double depth, size_t radius, float *out) {
    auto inputs = make_inputs(views, n_views);
    auto r = score_one_view(inputs[reference_index], inputs[target_index], inputs[target_index].warp, {cx, cy},
                            std::isnan(depth) ? std::nullopt : std::optional<double>(depth), radius);
    if (!r) return 0;
    *out = *r;
    return 1;
}

// Stage-level: build_cost_volume (depth.rs:1187-1277), restricted to rows
// [row_begin, row_end) when asked (the benchmark times a bounded sample).
int oracle_build_cost_volume(const chiaro_view *views, size_t n_views, size_t reference_index,
                             const chiaro_depth_options *opt, size_t row_begin, size_t row_end, float *scores,
                             float *costs, float *guidance, uint8_t *tested, int threads) {
    Options options(*opt);
    if (!valid_options(options) || reference_index >= n_views || !views[reference_index].has_camera)
        return CHIARO_INVALID;
    auto inputs = make_inputs(views, n_views);
    size_t step = std::max<size_t>(options.grid_step, 4);
    size_t columns = div_ceil(inputs[reference_index].width, step) + 1;
    size_t rows = div_ceil(inputs[reference_index].height, step) + 1;
    row_end = std::min(row_end, rows);
    std::vector<uint8_t> mask(rows, 0);
    for (size_t row = row_begin; row < row_end; ++row) mask[row] = 1;
    auto v = build_cost_volume(inputs, reference_index, columns, rows, step, options, threads, mask.data());
    size_t nl = v.labels.size();
    for (size_t row = row_begin; row < row_end; ++row)
        for (size_t column = 0; column < columns; ++column) {
            size_t node = row * columns + column;
            if (scores) std::memcpy(scores + node * nl, v.scores.data() + node * nl, nl * 4);
            if (costs) std::memcpy(costs + node * nl, v.costs.data() + node * nl, nl * 4);
            if (guidance) guidance[node] = v.guidance[node];
            if (tested) tested[node] = v.tested[node];
        }
    return CHIARO_OK;
}

// Stage-level: measure_direct_depths (depth.rs:715-876) given a coarse field,
// restricted to rows [row_begin, row_end).
int oracle_measure_direct_depths(const chiaro_view *views, size_t n_views, size_t reference_index,
                                 const chiaro_depth_options *opt, const uint8_t *coarse_has,
                                 const double *coarse_depth, const float *coarse_confidence,
                                 const float *coarse_improvement, const uint8_t *coarse_regularized,
                                 size_t row_begin, size_t row_end, uint8_t *has, double *depth, float *confidence,
                                 float *improvement, float *guidance, uint8_t *tested, int threads) {
    Options options(*opt);
    if (!valid_options(options) || reference_index >= n_views || !views[reference_index].has_camera)
        return CHIARO_INVALID;
    auto inputs = make_inputs(views, n_views);
    size_t cstep = std::max<size_t>(options.grid_step, 4);
    size_t cc = div_ceil(inputs[reference_index].width, cstep) + 1;
    size_t cr = div_ceil(inputs[reference_index].height, cstep) + 1;
    Field coarse =
        arrays_to_field(cc * cr, coarse_has, coarse_depth, coarse_confidence, coarse_improvement, coarse_regularized);
    double inverse_step = (1.0 / options.near_depth - 1.0 / options.far_depth) / (double)(options.planes - 1);
    size_t fine_step = std::max<size_t>(cstep / 2, 4);
    size_t fine_rows = div_ceil(inputs[reference_index].height, fine_step) + 1;
    row_end = std::min(row_end, fine_rows);
    std::vector<uint8_t> mask(fine_rows, 0);
    for (size_t row = row_begin; row < row_end; ++row) mask[row] = 1;
    auto d = measure_direct_depths(inputs, reference_index, coarse, cc, cr, cstep, inverse_step, options, threads,
                                   mask.data());
    for (size_t row = row_begin; row < row_end; ++row)
        for (size_t column = 0; column < d.columns; ++column) {
            size_t i = row * d.columns + column;
            if (has) has[i] = d.nodes[i].has_value();
            if (depth) depth[i] = d.nodes[i] ? d.nodes[i]->depth : NAN;
            if (confidence) confidence[i] = d.nodes[i] ? d.nodes[i]->confidence : 0.0f;
            if (improvement) improvement[i] = d.nodes[i] ? d.nodes[i]->improvement : 0.0f;
            if (guidance) guidance[i] = d.guidance[i];
            if (tested) tested[i] = d.tested[i];
        }
    return CHIARO_OK;
}

// Stage-level: one target's decisions (depth.rs:427-489) with consensus and
// boundary suppression, over the fine rows [row_begin, row_end) only (the
// band is treated as its own grid). Serial, like the reference's loop.
// field arrays and guidance are the full fine grid; kind_out is band-sized.
int oracle_target_decisions(const chiaro_view *views, size_t n_views, size_t reference_index, size_t target_index,
                            const chiaro_depth_options *opt, const uint8_t *has, const double *depth,
                            const float *confidence, const uint8_t *regularized, const float *guidance,
                            size_t row_begin, size_t row_end, uint8_t *kind_out) {
    Options options(*opt);
    if (!valid_options(options) || reference_index >= n_views || target_index >= n_views) return CHIARO_INVALID;
    auto inputs = make_inputs(views, n_views);
    if (!inputs[reference_index].camera || !inputs[target_index].camera) return CHIARO_INVALID;
    size_t cstep = std::max<size_t>(options.grid_step, 4);
    size_t step = std::max<size_t>(cstep / 2, 4);
    size_t columns = div_ceil(inputs[reference_index].width, step) + 1;
    size_t rows = div_ceil(inputs[reference_index].height, step) + 1;
    row_end = std::min(row_end, rows);
    if (row_begin >= row_end) return CHIARO_OK;
    size_t band_rows = row_end - row_begin, n = band_rows * columns, off = row_begin * columns;
    Field field = arrays_to_field(n, has + off, depth + off, confidence + off, nullptr, regularized + off);
    double inverse_step = (1.0 / options.near_depth - 1.0 / options.far_depth) / (double)(options.planes - 1);
    // Shift the band to the origin of its own grid by offsetting node pixels.
    std::vector<NodeWarp> decisions(n);
    const Input &reference = inputs[reference_index];
    const Warp &global = inputs[target_index].warp;
    for (size_t row = 0; row < band_rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            size_t index = row * columns + column;
            Vec2 p = {(double)(column * step), (double)((row + row_begin) * step)};
            NodeWarp &d = decisions[index];
            auto global_q = global.map((float)p[0], (float)p[1]);
            if (!global_q) continue;
            d.kind = CHIARO_NW_GLOBAL;
            d.global = *global_q;
            d.point = *global_q;
            if (!field[index]) continue;
            const NodeDepth node = *field[index];
            auto selected =
                refine_one_view(reference, inputs[target_index], global, p, node.depth, inverse_step, options);
            auto baseline =
                score_one_view(reference, inputs[target_index], global, p, std::nullopt, options.patch_radius);
            bool supported = selected && selected->score >= options.minimum_score &&
                             (!baseline || selected->score + 0.01f >= *baseline);
            bool contradicted = selected && baseline && selected->score + 0.12f < *baseline;
            if (contradicted) {
                d.kind = CHIARO_NW_OCCLUDED;
                d.measured = !node.regularized;
            } else if (supported) {
                d.kind = CHIARO_NW_REFINED;
                d.point = selected->point;
                d.confidence = node.regularized ? node.confidence * 0.6f : 0.5f + 0.5f * node.confidence;
                d.measured = !node.regularized;
            }
        }
    enforce_warp_consensus(decisions, columns, band_rows);
    suppress_warp_boundaries(decisions, guidance + off, columns, band_rows);
    for (size_t i = 0; i < n; ++i) kind_out[i] = (uint8_t)decisions[i].kind;
    return CHIARO_OK;
}

// The whole stage on a sample of coarse rows, timed per stage (the benchmark's CPU
// baseline). coarse_row_mask marks the sampled coarse rows; the direct pass, the
// filters and the decisions take the fine rows those nodes seed (fine rows 2r - 1 and
// 2r round to coarse row r in nearest_coarse_depth, depth.rs:1062-1076). Each stage
// runs as the reference runs it over the full grid:
//   cost volume and direct pass: the reference's worker bands over all rows, each
//     worker working on its own marked rows (depth.rs:1204-1206, 729-731);
//   SGM, winner-take-all, filters and per-target decisions: one thread, over the
//     sampled rows stacked into a grid of their own (the work per node and label is
//     that of the full grid; depth.rs:359-392, 420-547).
// seconds[6] receives the wall time of cost volume, SGM, select, direct, filters and
// decisions; counts[2] the sampled coarse and fine nodes.
int oracle_stage_sample(const chiaro_view *views, size_t n_views, size_t reference_index,
                        const chiaro_depth_options *opt, const uint8_t *coarse_row_mask, int threads,
                        double *seconds, uint64_t *counts) {
    using clock = std::chrono::steady_clock;
    auto since = [](clock::time_point t) { return std::chrono::duration<double>(clock::now() - t).count(); };
    Options options(*opt);
    if (!valid_options(options) || reference_index >= n_views || !views[reference_index].has_camera)
        return CHIARO_INVALID;
    auto inputs = make_inputs(views, n_views);
    const Input &reference = inputs[reference_index];
    size_t cstep = std::max<size_t>(options.grid_step, 4);
    size_t cc = div_ceil(reference.width, cstep) + 1, cr = div_ceil(reference.height, cstep) + 1;
    std::vector<size_t> coarse_rows;
    for (size_t r = 0; r < cr; ++r)
        if (coarse_row_mask[r]) coarse_rows.push_back(r);
    if (coarse_rows.empty()) return CHIARO_INVALID;
    auto t = clock::now();
    CostVolume volume = build_cost_volume(inputs, reference_index, cc, cr, cstep, options, threads, coarse_row_mask);
    seconds[0] = since(t);
    size_t nl = volume.labels.size(), sr = coarse_rows.size(), sn = sr * cc;
    std::vector<float> costs(sn * nl), scores(sn * nl), guidance(sn);
    std::vector<uint8_t> tested(sn);
    for (size_t i = 0; i < sr; ++i) {
        size_t from = coarse_rows[i] * cc, to = i * cc;
        std::memcpy(costs.data() + to * nl, volume.costs.data() + from * nl, cc * nl * 4);
        std::memcpy(scores.data() + to * nl, volume.scores.data() + from * nl, cc * nl * 4);
        std::memcpy(guidance.data() + to, volume.guidance.data() + from, cc * 4);
        std::memcpy(tested.data() + to, volume.tested.data() + from, cc);
    }
    t = clock::now();
    std::vector<float> regularised = semi_global_costs(costs.data(), guidance.data(), cc, sr, nl);
    seconds[1] = since(t);
    Field sampled;
    std::vector<uint8_t> fillable;
    t = clock::now();
    select_depths(volume.labels, scores.data(), tested.data(), sn, regularised.data(), options, sampled, fillable);
    seconds[2] = since(t);
    Field coarse(cc * cr);
    for (size_t i = 0; i < sr; ++i)
        for (size_t c = 0; c < cc; ++c) coarse[coarse_rows[i] * cc + c] = sampled[i * cc + c];
    double inverse_step = (1.0 / options.near_depth - 1.0 / options.far_depth) / (double)(options.planes - 1);
    size_t step = std::max<size_t>(cstep / 2, 4);
    size_t columns = div_ceil(reference.width, step) + 1, rows = div_ceil(reference.height, step) + 1;
    std::vector<uint8_t> fine_mask(rows, 0);
    for (size_t r : coarse_rows) {
        if (2 * r >= 1 && 2 * r - 1 < rows) fine_mask[2 * r - 1] = 1;
        if (2 * r < rows) fine_mask[2 * r] = 1;
    }
    t = clock::now();
    DirectField direct = measure_direct_depths(inputs, reference_index, coarse, cc, cr, cstep, inverse_step, options,
                                               threads, fine_mask.data());
    seconds[3] = since(t);
    std::vector<size_t> fine_rows;
    for (size_t r = 0; r < rows; ++r)
        if (fine_mask[r]) fine_rows.push_back(r);
    size_t fr = fine_rows.size(), fn = fr * columns;
    Field field(fn);
    std::vector<float> fine_guidance(fn);
    for (size_t i = 0; i < fr; ++i)
        for (size_t c = 0; c < columns; ++c) {
            field[i * columns + c] = direct.nodes[fine_rows[i] * columns + c];
            fine_guidance[i * columns + c] = direct.guidance[fine_rows[i] * columns + c];
        }
    t = clock::now();
    reject_isolated_direct_depths(field, fine_guidance.data(), columns, fr, inverse_step * 2.5);
    reject_small_direct_components(field, fine_guidance.data(), columns, fr, inverse_step * 2.5,
                                   MINIMUM_DIRECT_COMPONENT_NODES);
    fit_local_depth_planes(field, fine_guidance.data(), columns, fr, inverse_step * 4.0);
    seconds[4] = since(t);
    t = clock::now();
    for (size_t target_index = 0; target_index < n_views; ++target_index) {
        if (target_index == reference_index || !inputs[target_index].accepted || !inputs[target_index].camera)
            continue;
        auto decisions = target_decisions(inputs, reference_index, target_index, field, fine_guidance.data(),
                                          columns, fr, step, inverse_step, options, fine_rows.data());
        (void)decisions;
    }
    seconds[5] = since(t);
    counts[0] = sn;
    counts[1] = fn;
    return CHIARO_OK;
}

// luminance_half (image.rs:401-428) with flat field 1: samples w*h u16.
void oracle_luminance_half(const uint16_t *samples, size_t width, size_t height, float black_q6, float white_q6,
                           float *out) {
    size_t w = width / 2, h = height / 2;
    float range = fmax_r(white_q6 - black_q6, 1.0f);
    for (size_t j = 0; j < h; ++j) {
        const uint16_t *row0 = samples + 2 * j * width;
        const uint16_t *row1 = samples + (2 * j + 1) * width;
        for (size_t i = 0; i < w; ++i) {
            float sum = (float)row0[2 * i] + (float)row0[2 * i + 1] + (float)row1[2 * i] + (float)row1[2 * i + 1];
            float linear = fmax_r((sum * 0.25f - black_q6) / range, 0.0f) * 1.0f;
            out[j * w + i] = std::log(1.0f + 1000.0f * linear);
        }
    }
}

// VignettingMesh::gain (calibration.rs:362-379) at raster (x, y) of a width x height sensor.
static float vignetting_gain(const float *gains, size_t columns, size_t rows, float x, float y, size_t width,
                             size_t height) {
    if (!gains || columns < 2 || rows < 2) return 1.0f;
    float cmax = (float)(columns - 1), rmax = (float)(rows - 1);
    float fx = fclamp(x / (float)width * cmax, 0.0f, cmax);
    float fy = fclamp(y / (float)height * rmax, 0.0f, rmax);
    size_t c0 = (size_t)std::floor(fx), r0 = (size_t)std::floor(fy);
    size_t c1 = std::min(c0 + 1, columns - 1), r1 = std::min(r0 + 1, rows - 1);
    float tx = fx - (float)c0, ty = fy - (float)r0;
    auto g = [&](size_t c, size_t r) { return gains[r * columns + c]; };
    float top = g(c0, r0) * (1.0f - tx) + g(c1, r0) * tx;
    float bottom = g(c0, r1) * (1.0f - tx) + g(c1, r1) * tx;
    return top * (1.0f - ty) + bottom * ty;
}

// luminance_half (image.rs:401-428) with Mosaic::flat_field (image.rs:145-150): the
// plane, and (when `argument` is given) the log's argument 1 + 1000 * linear per pixel.
void oracle_luminance_half_mesh(const uint16_t *samples, size_t width, size_t height, float black_q6,
                                float white_q6, const float *gains, size_t columns, size_t rows, float *out,
                                float *argument) {
    size_t w = width / 2, h = height / 2;
    float range = fmax_r(white_q6 - black_q6, 1.0f);
    for (size_t j = 0; j < h; ++j) {
        const uint16_t *row0 = samples + 2 * j * width;
        const uint16_t *row1 = samples + (2 * j + 1) * width;
        for (size_t i = 0; i < w; ++i) {
            float sum = (float)row0[2 * i] + (float)row0[2 * i + 1] + (float)row1[2 * i] + (float)row1[2 * i + 1];
            float flat = vignetting_gain(gains, columns, rows, 2.0f * (float)i + 0.5f, 2.0f * (float)j + 0.5f,
                                         width, height);
            float linear = fmax_r((sum * 0.25f - black_q6) / range, 0.0f) * flat;
            float x = 1.0f + 1000.0f * linear;
            if (argument) argument[j * w + i] = x;
            out[j * w + i] = std::log(x);
        }
    }
}

// ---- quantised SGM (no counterpart in the reference) ------------------------------------
// The project's quantised performance mode of semi_global_costs: costs in u16 fixed point
// (Q = 2048 per cost unit; the stage's costs lie in [0, 2.25], so at most 4608), the edge
// penalties of accumulate_path (depth.rs:1358-1361) computed in f32 as the reference does
// and quantised the same way, the path recurrence (depth.rs:1363-1381) in exact integers,
// the 8 path costs summed per cell (a path cost is at most 4608 + 922, the sum at most
// 44240: no overflow), and the winner over labels 1..D-1 (the first minimum, as
// select_depths picks it).
static const float SGM_Q = 2048.0f;
static const uint32_t SGM_COST_MAX_Q = 4608;  // 2.25 * Q

static uint32_t quantise_sgm_cost(float c) {
    if (!(c == c)) return SGM_COST_MAX_Q;  // NaN: the missing cost
    float v = std::nearbyint(c * SGM_Q);
    if (v <= 0.0f) return 0;
    return v >= (float)SGM_COST_MAX_Q ? SGM_COST_MAX_Q : (uint32_t)v;
}

static uint32_t quantise_penalty(float p) { return (uint32_t)std::nearbyint(p * SGM_Q); }

static void accumulate_path_u16(const uint32_t *data, const float *guidance, uint32_t *output, size_t labels,
                                const std::vector<size_t> &path) {
    const uint32_t big = 0xFFFF;
    std::vector<uint32_t> previous(labels), current(labels);
    for (size_t k = 0; k < path.size(); ++k) {
        size_t node = path[k], offset = node * labels;
        if (k == 0) {
            for (size_t l = 0; l < labels; ++l) {
                previous[l] = data[offset + l];
                output[offset + l] += previous[l];
            }
            continue;
        }
        float edge = std::fabs(guidance[node] - guidance[path[k - 1]]);
        float edge_scale = 1.0f / (1.0f + 4.0f * edge);
        uint32_t p1 = quantise_penalty(0.06f * fmax_r(edge_scale, 0.35f));
        uint32_t p2 = quantise_penalty(0.45f * fmax_r(edge_scale, 0.12f));
        uint32_t minimum_previous = big;
        for (size_t l = 0; l < labels; ++l) minimum_previous = std::min(minimum_previous, previous[l]);
        for (size_t l = 0; l < labels; ++l) {
            uint32_t lower = l > 0 ? previous[l - 1] + p1 : big;
            uint32_t higher = l + 1 < labels ? previous[l + 1] + p1 : big;
            uint32_t best = std::min(std::min(previous[l], lower), std::min(higher, minimum_previous + p2));
            current[l] = data[offset + l] + best - minimum_previous;
            output[offset + l] += current[l];
        }
        std::swap(previous, current);
    }
}

void oracle_sgm_u16(const float *costs, const float *guidance, size_t columns, size_t rows, size_t labels,
                    uint16_t *aggregate, uint16_t *best) {
    size_t n = columns * rows;
    std::vector<uint32_t> data(n * labels), output(n * labels, 0);
    for (size_t i = 0; i < n * labels; ++i) data[i] = quantise_sgm_cost(costs[i]);
    std::vector<size_t> forward, reverse;
    auto both = [&](const std::vector<size_t> &path) {
        accumulate_path_u16(data.data(), guidance, output.data(), labels, path);
        reverse.assign(path.rbegin(), path.rend());
        accumulate_path_u16(data.data(), guidance, output.data(), labels, reverse);
    };
    for (size_t row = 0; row < rows; ++row) {
        forward.clear();
        for (size_t column = 0; column < columns; ++column) forward.push_back(row * columns + column);
        both(forward);
    }
    for (size_t column = 0; column < columns; ++column) {
        forward.clear();
        for (size_t row = 0; row < rows; ++row) forward.push_back(row * columns + column);
        both(forward);
    }
    for (int mirrored = 0; mirrored < 2; ++mirrored)
        for (const auto &path : diagonal_paths(columns, rows, mirrored != 0)) both(path);
    for (size_t node = 0; node < n; ++node) {
        const uint32_t *o = output.data() + node * labels;
        if (aggregate)
            for (size_t l = 0; l < labels; ++l) aggregate[node * labels + l] = (uint16_t)o[l];
        if (best) {
            size_t b = labels > 1 ? 1 : 0;
            for (size_t l = 2; l < labels; ++l)
                if (o[l] < o[b]) b = l;
            best[node] = (uint16_t)b;
        }
    }
}

// ---- banded SGM with windowed full-range fallback (no counterpart in the reference) -----
// The project's band-limited form of semi_global_costs (depth.rs:1279-1383): every node
// of a tile (tile x tile coarse nodes) aggregates only the labels [O, O + band) of its
// tile's offset O (1 <= O <= D - band: finite labels). Along a path the band may shift
// between tiles: the previous node's value for label l is its slot l - O_prev when that
// lies in its band, +inf otherwise, and the recurrence of accumulate_path
// (depth.rs:1363-1381) is otherwise unchanged, the minimum taken over the previous band.
// The 8 path costs are added per slot in the reference's order and the winner is the
// first minimum over the band. A tile whose winner sits on a band edge (slot 0 or
// band - 1) at any of its nodes falls back: the full-range SGM over the window of the
// tile grown by `margin` nodes (clipped to the grid) decides its nodes' winners (over
// labels 1..D-1, first minimum).
static void accumulate_path_banded(const float *data, const float *guidance, const int *node_offset, float *output,
                                   size_t labels, size_t band, const std::vector<size_t> &path) {
    const float inf = std::numeric_limits<float>::infinity();
    std::vector<float> previous(band), current(band);
    for (size_t k = 0; k < path.size(); ++k) {
        size_t node = path[k];
        const float *c = data + node * labels + node_offset[node];
        float *o = output + node * band;
        if (k == 0) {
            for (size_t j = 0; j < band; ++j) {
                previous[j] = c[j];
                o[j] += previous[j];
            }
            continue;
        }
        size_t prior = path[k - 1];
        float edge = std::fabs(guidance[node] - guidance[prior]);
        float edge_scale = 1.0f / (1.0f + 4.0f * edge);
        float p1 = 0.06f * fmax_r(edge_scale, 0.35f);
        float p2 = 0.45f * fmax_r(edge_scale, 0.12f);
        float minimum_previous = inf;
        for (size_t j = 0; j < band; ++j) minimum_previous = fmin_r(minimum_previous, previous[j]);
        long delta = (long)node_offset[node] - (long)node_offset[prior];
        for (size_t j = 0; j < band; ++j) {
            long label = node_offset[node] + (long)j, s = (long)j + delta;
            auto at = [&](long slot) { return slot >= 0 && slot < (long)band ? previous[slot] : inf; };
            float same = at(s);
            float lower = label > 0 ? at(s - 1) + p1 : inf;
            float higher = label + 1 < (long)labels ? at(s + 1) + p1 : inf;
            float jump = minimum_previous + p2;
            current[j] = c[j] + fmin_r(fmin_r(fmin_r(same, lower), higher), jump) - minimum_previous;
            o[j] += current[j];
        }
        std::swap(previous, current);
    }
}

static void sgm_paths_generic(size_t columns, size_t rows, const std::function<void(const std::vector<size_t> &)> &walk) {
    std::vector<size_t> forward, reverse;
    auto both = [&](const std::vector<size_t> &path) {
        walk(path);
        reverse.assign(path.rbegin(), path.rend());
        walk(reverse);
    };
    for (size_t row = 0; row < rows; ++row) {
        forward.clear();
        for (size_t column = 0; column < columns; ++column) forward.push_back(row * columns + column);
        both(forward);
    }
    for (size_t column = 0; column < columns; ++column) {
        forward.clear();
        for (size_t row = 0; row < rows; ++row) forward.push_back(row * columns + column);
        both(forward);
    }
    for (int mirrored = 0; mirrored < 2; ++mirrored)
        for (const auto &path : diagonal_paths(columns, rows, mirrored != 0)) both(path);
}

// Winner labels of the banded SGM with fallback; fallback[t] = 1 for tiles that fell back.
int oracle_sgm_banded(const float *costs, const float *guidance, size_t columns, size_t rows, size_t labels,
                      const int *tile_offset, size_t tile, size_t band, size_t margin, int *winner,
                      uint8_t *fallback) {
    if (band < 1 || band > 32 || band + 1 > labels || tile < 1) return CHIARO_ERR_ARGUMENT;
    size_t n = columns * rows, tiles_x = div_ceil(columns, tile), tiles_y = div_ceil(rows, tile);
    std::vector<int> node_offset(n);
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < columns; ++c) {
            int o = tile_offset[(r / tile) * tiles_x + c / tile];
            if (o < 1 || o + band > labels) return CHIARO_ERR_ARGUMENT;
            node_offset[r * columns + c] = o;
        }
    std::vector<float> output(n * band, 0.0f);
    sgm_paths_generic(columns, rows, [&](const std::vector<size_t> &path) {
        accumulate_path_banded(costs, guidance, node_offset.data(), output.data(), labels, band, path);
    });
    std::fill(fallback, fallback + tiles_x * tiles_y, 0);
    for (size_t node = 0; node < n; ++node) {
        const float *o = output.data() + node * band;
        size_t best = 0;
        for (size_t j = 1; j < band; ++j)
            if (total_key_f32(o[j]) < total_key_f32(o[best])) best = j;
        winner[node] = node_offset[node] + (int)best;
        // a band edge wins where labels lie beyond it (not at label 1 or D - 1)
        const int offset = node_offset[node];
        if ((best == 0 && offset > 1) || (best + 1 == band && (size_t)offset + band < labels))
            fallback[((node / columns) / tile) * tiles_x + (node % columns) / tile] = 1;
    }
    // fallback tiles as greedy rectangles in raster order (widest run, then as many
    // rows of it as are all flagged), each rerun at full range in a window of margin
    // nodes around it; where those windows would cover at least the grid, one
    // full-range SGM over the whole grid decides every fallback tile instead
    struct Rect { size_t n0c, n0r, n1c, n1r, c0, r0, c1, r1; };
    std::vector<Rect> rects;
    size_t window_nodes = 0;
    std::vector<uint8_t> taken(tiles_x * tiles_y, 0);
    auto open = [&](size_t x, size_t y) { return fallback[y * tiles_x + x] && !taken[y * tiles_x + x]; };
    for (size_t ty = 0; ty < tiles_y; ++ty)
        for (size_t tx = 0; tx < tiles_x; ++tx) {
            if (!open(tx, ty)) continue;
            size_t w = 1, h = 1;
            while (tx + w < tiles_x && open(tx + w, ty)) ++w;
            for (bool grow = true; grow && ty + h < tiles_y;) {
                for (size_t x = tx; x < tx + w; ++x) grow = grow && open(x, ty + h);
                if (grow) ++h;
            }
            for (size_t y = ty; y < ty + h; ++y)
                for (size_t x = tx; x < tx + w; ++x) taken[y * tiles_x + x] = 1;
            Rect q;
            q.n0c = tx * tile;
            q.n0r = ty * tile;
            q.n1c = std::min(columns, (tx + w) * tile);
            q.n1r = std::min(rows, (ty + h) * tile);
            q.c0 = q.n0c > margin ? q.n0c - margin : 0;
            q.r0 = q.n0r > margin ? q.n0r - margin : 0;
            q.c1 = std::min(columns, q.n1c + margin);
            q.r1 = std::min(rows, q.n1r + margin);
            window_nodes += (q.c1 - q.c0) * (q.r1 - q.r0);
            rects.push_back(q);
        }
    if (!rects.empty() && window_nodes >= n) rects.assign(1, Rect{0, 0, columns, rows, 0, 0, columns, rows});
    for (const Rect &q : rects) {
        const size_t wc = q.c1 - q.c0, wr = q.r1 - q.r0;
        std::vector<float> wcost(wc * wr * labels), wguid(wc * wr);
        for (size_t r = 0; r < wr; ++r)
            for (size_t c = 0; c < wc; ++c) {
                size_t src = (q.r0 + r) * columns + q.c0 + c;
                wguid[r * wc + c] = guidance[src];
                std::copy(costs + src * labels, costs + (src + 1) * labels, wcost.begin() + (r * wc + c) * labels);
            }
        auto agg = semi_global_costs(wcost.data(), wguid.data(), wc, wr, labels);
        for (size_t r = q.n0r; r < q.n1r; ++r)
            for (size_t c = q.n0c; c < q.n1c; ++c) {
                if (!fallback[(r / tile) * tiles_x + c / tile]) continue;
                const float *o = agg.data() + ((r - q.r0) * wc + (c - q.c0)) * labels;
                size_t best = 1;
                for (size_t l = 2; l < labels; ++l)
                    if (total_key_f32(o[l]) < total_key_f32(o[best])) best = l;
                winner[r * columns + c] = (int)best;
            }
    }
    return CHIARO_OK;
}

// ---- band proposal network, fp32 (no counterpart in the reference) -------------------------
// The oracle of the learned band proposal: the same network in plain fp32 loops
// (NHWC, 32 channels, zero padding, six 3x3 convolutions, ReLU after the first
// five, Huber loss with delta 0.02 on channel 0 over the masked nodes, mean over
// them) and its backward pass. Parameters: per layer [tap][co][ci] weights then
// 32 biases.
static const int NET_CH_O = 32, NET_LAYERS_O = 6, NET_W_O = 9 * 32 * 32;

// The band proposal's sampled labels: 16 finite labels spread evenly over 1..labels-1
// (the first and the last included), label(b) = 1 + (b (labels - 2) + 7) / 15.
static int net_sample_label(int b, int labels) { return 1 + (b * (labels - 2) + 7) / 15; }

void oracle_net_sample_labels(size_t labels, int *out) {
    for (int b = 0; b < 16; ++b) out[b] = net_sample_label(b, (int)labels);
}

// Features of the band network per node: the reference luminance at the node
// (guidance / 8); the costs of the 16 sampled labels minus the lowest of them; the
// first of the sampled labels holding that lowest cost, as (label - 1) / (labels - 2);
// and the lowest cost. costs rows hold `stride` values: the full volume (stride =
// labels, a label's cost at its index) or the pre-pass's rows (stride = 17, label 0
// then the sampled labels in order).
void oracle_bandnet_features(const float *costs, const float *guidance, size_t nodes, size_t labels, size_t stride,
                             float *features) {
    const int bins = 16;
    for (size_t node = 0; node < nodes; ++node) {
        const float *c = costs + node * stride;
        float v[16], lowest = std::numeric_limits<float>::infinity();
        int argmin = 1;
        for (int b = 0; b < bins; ++b) {
            const int label = net_sample_label(b, (int)labels);
            v[b] = c[stride == labels ? label : 1 + b];
            if (v[b] < lowest) {
                lowest = v[b];
                argmin = label;
            }
        }
        float *f = features + node * NET_CH_O;
        f[0] = guidance[node] * 0.125f;
        for (int b = 0; b < bins; ++b) f[1 + b] = v[b] - lowest;
        f[1 + bins] = (float)(argmin - 1) / (float)(labels - 2);
        f[2 + bins] = lowest;
        for (int k = 3 + bins; k < NET_CH_O; ++k) f[k] = 0.0f;
    }
}

static void net_conv_o(const float *in, int images, int h, int w, const float *wt, const float *bias, float *out) {
    for (int n = 0; n < images; ++n)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x)
                for (int co = 0; co < NET_CH_O; ++co) {
                    double s = bias ? bias[co] : 0.0;
                    for (int tap = 0; tap < 9; ++tap) {
                        int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
                        if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
                        const float *a = in + (((size_t)n * h + yy) * w + xx) * NET_CH_O;
                        const float *k = wt + ((size_t)tap * NET_CH_O + co) * NET_CH_O;
                        for (int ci = 0; ci < NET_CH_O; ++ci) s += (double)a[ci] * k[ci];
                    }
                    out[(((size_t)n * h + y) * w + x) * NET_CH_O + co] = (float)s;
                }
}

// Round to the nearest bf16 (ties to even), as __float2bfloat16_rn does.
static float bf16_round(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return v;  // inf and NaN stay
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// Loss and gradient of the network on a batch; y (optional) receives channel 0. With
// bf16_storage, every stored activation and pre-activation gradient is rounded to bf16,
// as the GPU stores them (the last layer's channel 0, y, stays fp32 there too).
void oracle_bandnet_loss_grad_mode(const float *params, const float *features, const float *targets,
                                   const uint8_t *mask, size_t images, size_t height, size_t width, float *grads,
                                   float *loss, float *y, int bf16_storage);

void oracle_bandnet_loss_grad(const float *params, const float *features, const float *targets, const uint8_t *mask,
                              size_t images, size_t height, size_t width, float *grads, float *loss, float *y) {
    oracle_bandnet_loss_grad_mode(params, features, targets, mask, images, height, width, grads, loss, y, 0);
}

void oracle_bandnet_loss_grad_mode(const float *params, const float *features, const float *targets,
                                   const uint8_t *mask, size_t images, size_t height, size_t width, float *grads,
                                   float *loss, float *y, int bf16_storage) {
    const int h = (int)height, w = (int)width, nimg = (int)images;
    const size_t pixels = images * height * width, act_n = pixels * NET_CH_O;
    std::vector<std::vector<float>> act(NET_LAYERS_O + 1, std::vector<float>(act_n));
    std::copy(features, features + act_n, act[0].begin());
    for (int l = 0; l < NET_LAYERS_O; ++l) {
        const float *p = params + (size_t)l * (NET_W_O + NET_CH_O);
        net_conv_o(act[l].data(), nimg, h, w, p, p + NET_W_O, act[l + 1].data());
        if (l + 1 < NET_LAYERS_O)
            for (float &v : act[l + 1]) v = std::fmax(v, 0.0f);
        if (bf16_storage && l + 1 < NET_LAYERS_O)
            for (float &v : act[l + 1]) v = bf16_round(v);
    }
    size_t count = 0;
    for (size_t i = 0; i < pixels; ++i) count += mask[i] != 0;
    const double inverse = count ? 1.0 / (double)count : 0.0;
    const float delta = 0.02f;
    std::vector<float> dpre(act_n, 0.0f), dnext(act_n);
    double total = 0.0;
    for (size_t i = 0; i < pixels; ++i) {
        float yi = act[NET_LAYERS_O][i * NET_CH_O];
        if (y) y[i] = yi;
        if (!mask[i]) continue;
        float e = yi - targets[i], a = std::fabs(e);
        total += a <= delta ? 0.5 * e * e : delta * (a - 0.5 * delta);
        dpre[i * NET_CH_O] = (float)((a <= delta ? e : std::copysign(delta, e)) * inverse);
        if (bf16_storage) dpre[i * NET_CH_O] = bf16_round(dpre[i * NET_CH_O]);
    }
    *loss = (float)(total * inverse);
    std::fill(grads, grads + (size_t)NET_LAYERS_O * (NET_W_O + NET_CH_O), 0.0f);
    for (int l = NET_LAYERS_O - 1; l >= 0; --l) {
        const float *p = params + (size_t)l * (NET_W_O + NET_CH_O);
        float *g = grads + (size_t)l * (NET_W_O + NET_CH_O);
        std::vector<double> dw(NET_W_O, 0.0), db(NET_CH_O, 0.0);
        for (int n = 0; n < nimg; ++n)
            for (int y0 = 0; y0 < h; ++y0)
                for (int x0 = 0; x0 < w; ++x0) {
                    const float *d = dpre.data() + (((size_t)n * h + y0) * w + x0) * NET_CH_O;
                    for (int co = 0; co < NET_CH_O; ++co) db[co] += d[co];
                    for (int tap = 0; tap < 9; ++tap) {
                        int yy = y0 + tap / 3 - 1, xx = x0 + tap % 3 - 1;
                        if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
                        const float *a = act[l].data() + (((size_t)n * h + yy) * w + xx) * NET_CH_O;
                        for (int co = 0; co < NET_CH_O; ++co) {
                            if (d[co] == 0.0f) continue;
                            double *row = dw.data() + ((size_t)tap * NET_CH_O + co) * NET_CH_O;
                            for (int ci = 0; ci < NET_CH_O; ++ci) row[ci] += (double)d[co] * a[ci];
                        }
                    }
                }
        for (int i = 0; i < NET_W_O; ++i) g[i] = (float)dw[i];
        for (int co = 0; co < NET_CH_O; ++co) g[NET_W_O + co] = (float)db[co];
        if (l == 0) break;
        // gradient at layer l's input, masked by its ReLU (act[l] is layer l-1's output)
        std::fill(dnext.begin(), dnext.end(), 0.0f);
        for (int n = 0; n < nimg; ++n)
            for (int y0 = 0; y0 < h; ++y0)
                for (int x0 = 0; x0 < w; ++x0) {
                    const float *d = dpre.data() + (((size_t)n * h + y0) * w + x0) * NET_CH_O;
                    for (int tap = 0; tap < 9; ++tap) {
                        int yy = y0 + tap / 3 - 1, xx = x0 + tap % 3 - 1;
                        if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
                        float *o = dnext.data() + (((size_t)n * h + yy) * w + xx) * NET_CH_O;
                        for (int co = 0; co < NET_CH_O; ++co) {
                            if (d[co] == 0.0f) continue;
                            const float *k = p + ((size_t)tap * NET_CH_O + co) * NET_CH_O;
                            for (int ci = 0; ci < NET_CH_O; ++ci) o[ci] += d[co] * k[ci];
                        }
                    }
                }
        for (size_t i = 0; i < act_n; ++i) dpre[i] = act[l][i] > 0.0f ? dnext[i] : 0.0f;
        if (bf16_storage)
            for (float &v : dpre) v = bf16_round(v);
    }
}

}  // extern "C"

// ---- resolution.rs: refine_resolution_warp (232-439) and image.rs: match_patch (531-640) ----

namespace {

float clamp_rust_o(float x, float lo, float hi) {  // f32::clamp: NaN passes through
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

struct PatchMatchO {
    float shift[2];
    float score;
};

// image.rs:531-640
std::optional<PatchMatchO> match_patch_o(const Plane &reference, const Plane &target, size_t rx, size_t ry,
                                         size_t size, size_t radius) {
    if (rx + size > reference.width || ry + size > reference.height || rx < radius || ry < radius ||
        rx + size + radius > target.width || ry + size + radius > target.height || rx + size > target.width ||
        ry + size > target.height)
        return std::nullopt;
    const float n = (float)(size * size);
    std::vector<float> ref_values;
    for (size_t y = ry; y < ry + size; ++y)
        for (size_t x = rx; x < rx + size; ++x) ref_values.push_back(reference.at(x, y));
    float total = -0.0f;  // f32 Sum starts at -0.0
    for (float v : ref_values) total += v;
    const float ref_mean = total / n;
    float squares = -0.0f;
    for (float v : ref_values) squares += (v - ref_mean) * (v - ref_mean);  // powi(2)
    const float ref_std = std::sqrt(squares / n);
    if (ref_std < 1e-4f) return std::nullopt;
    std::vector<float> ref_centered;
    for (float v : ref_values) ref_centered.push_back(v - ref_mean);
    const size_t span = 2 * radius + 1;
    std::vector<float> scores(span * span, -std::numeric_limits<float>::infinity());
    for (size_t dy = 0; dy < span; ++dy)
        for (size_t dx = 0; dx < span; ++dx) {
            const size_t tx = rx + dx - radius, ty = ry + dy - radius;
            float sum = 0.0f, sum_sq = 0.0f, cross = 0.0f;
            for (size_t y = 0; y < size; ++y)
                for (size_t x = 0; x < size; ++x) {
                    const float t = target.at(tx + x, ty + y), r = ref_centered[y * size + x];
                    sum += t;
                    sum_sq += t * t;
                    cross += t * r;
                }
            const float mean = sum / n;
            const float var = fmax_r(sum_sq / n - mean * mean, 0.0f);
            if (var < 1e-8f) continue;
            const float covariance = cross / n;
            scores[dy * span + dx] = covariance / (std::sqrt(var) * ref_std);
        }
    size_t best = 0;  // Iterator::max_by(total_cmp): the last maximum
    for (size_t i = 1; i < scores.size(); ++i)
        if (!(total_key_f32(scores[i]) < total_key_f32(scores[best]))) best = i;
    const float score = scores[best];
    if (!std::isfinite(score)) return std::nullopt;
    const size_t bx = best % span, by = best / span;
    auto refine = [](float minus, float center, float plus) {
        const float denominator = minus - 2.0f * center + plus;
        if (std::fabs(denominator) < 1e-9f) return 0.0f;
        return clamp_rust_o(0.5f * (minus - plus) / denominator, -0.5f, 0.5f);
    };
    const float sub_x =
        bx > 0 && bx + 1 < span ? refine(scores[by * span + bx - 1], score, scores[by * span + bx + 1]) : 0.0f;
    const float sub_y =
        by > 0 && by + 1 < span ? refine(scores[(by - 1) * span + bx], score, scores[(by + 1) * span + bx]) : 0.0f;
    PatchMatchO m;
    m.shift[0] = (float)bx - (float)radius + sub_x;
    m.shift[1] = (float)by - (float)radius + sub_y;
    m.score = score;
    return m;
}

// resolution.rs:441-465
std::optional<float> sample_at_reference_bandwidth_o(const Plane &target, float x, float y, float magnification) {
    if (magnification <= 1.15f) return target.sample(x, y);
    const float sigma = fmax_r(0.42f * magnification, 0.55f);
    const long radius = (long)clamp_rust_o(std::ceil(2.0f * sigma), 1.0f, 4.0f);
    float sum = 0.0f, weight = 0.0f;
    for (long dy = -radius; dy <= radius; ++dy)
        for (long dx = -radius; dx <= radius; ++dx) {
            const float distance_squared = (float)(dx * dx + dy * dy);
            const float kernel = std::exp(-0.5f * distance_squared / (sigma * sigma));  // libm expf
            if (auto value = target.sample(x + (float)dx, y + (float)dy)) {
                sum += kernel * *value;
                weight += kernel;
            }
        }
    if (!(weight > 1.0e-8f)) return std::nullopt;
    return sum / weight;
}

// Warp::confidence (align.rs:113-131)
float warp_confidence_o(const chiaro_warp &w, float x, float y) {
    const float fx = x / (float)w.step, fy = y / (float)w.step;
    if (fx < 0.0f || fy < 0.0f || !w.confidence) return 0.0f;
    const size_t c0 = std::min(sat_usize(std::floor(fx)), (size_t)w.columns - 1);
    const size_t r0 = std::min(sat_usize(std::floor(fy)), (size_t)w.rows - 1);
    const size_t c1 = std::min(c0 + 1, (size_t)w.columns - 1), r1 = std::min(r0 + 1, (size_t)w.rows - 1);
    const float tx = fx - (float)c0, ty = fy - (float)r0;
    auto value = [&](size_t c, size_t r) { return w.confidence[r * w.columns + c]; };
    const float top = value(c0, r0) * (1.0f - tx) + value(c1, r0) * tx;
    const float bottom = value(c0, r1) * (1.0f - tx) + value(c1, r1) * tx;
    return clamp_rust_o(top * (1.0f - ty) + bottom * ty, 0.0f, 1.0f);
}

bool total_less_o(float a, float b) { return total_key_f32(a) < total_key_f32(b); }

}  // namespace

// match_patch (image.rs:531-640); returns 0 for None.
extern "C" int oracle_match_patch(const float *reference, size_t reference_width, size_t reference_height, const float *target,
                       size_t target_width, size_t target_height, size_t rx, size_t ry, size_t size, size_t radius,
                       float *shift, float *score) {
    Plane r, t;
    r.width = reference_width;
    r.height = reference_height;
    r.data = reference;
    t.width = target_width;
    t.height = target_height;
    t.data = target;
    auto m = match_patch_o(r, t, rx, ry, size, radius);
    if (!m) return 0;
    shift[0] = m->shift[0];
    shift[1] = m->shift[1];
    *score = m->score;
    return 1;
}

// refine_resolution_warp (resolution.rs:232-439). out->points / out->confidence hold
// columns * rows nodes; report = (verified, supported, median correction, mean confidence).
extern "C" int oracle_refine_resolution_warp(const float *reference_data, size_t reference_width, size_t reference_height,
                                  const float *target_data, size_t target_width, size_t target_height,
                                  const chiaro_warp *base_c, size_t width, size_t height, chiaro_warp *out,
                                  float *report) {
    constexpr size_t STEP = 32, PATCH = 12, RADIUS = 2, MAGNIFIED_RADIUS = 5;
    constexpr float MINIMUM_SCORE = 0.72f;
    Plane reference, target;
    reference.width = reference_width;
    reference.height = reference_height;
    reference.data = reference_data;
    target.width = target_width;
    target.height = target_height;
    target.data = target_data;
    Warp base;
    base.step = (size_t)base_c->step;
    base.columns = (size_t)base_c->columns;
    base.rows = (size_t)base_c->rows;
    base.points = base_c->points;
    // resolution.rs:239-253
    float magnification = 1.0f;
    if (!oracle_warp_magnification(base_c, (float)width * 0.5f, (float)height * 0.5f, &magnification))
        magnification = 1.0f;
    magnification = clamp_rust_o(magnification, 0.5f, 4.0f);
    const size_t match_radius = magnification > 1.35f ? MAGNIFIED_RADIUS : RADIUS;
    // resolution.rs:255-271
    std::vector<float> rendered_data(reference.width * reference.height);
    for (size_t y = 0; y < reference.height; ++y)
        for (size_t x = 0; x < reference.width; ++x) {
            const float rx = (float)x * 2.0f + 0.5f, ry = (float)y * 2.0f + 0.5f;
            float value = std::numeric_limits<float>::quiet_NaN();
            if (auto q = base.map(rx, ry))
                if (auto v = sample_at_reference_bandwidth_o(target, ((*q)[0] + 0.5f) * 0.5f - 0.5f,
                                                             ((*q)[1] + 0.5f) * 0.5f - 0.5f, magnification))
                    value = *v;
            rendered_data[y * reference.width + x] = value;
        }
    Plane rendered;
    rendered.width = reference.width;
    rendered.height = reference.height;
    rendered.data = rendered_data.data();
    // resolution.rs:273-305
    const size_t columns = div_ceil(width, STEP) + 1, rows = div_ceil(height, STEP) + 1;
    out->step = STEP;
    out->columns = columns;
    out->rows = rows;
    if (out->capacity < columns * rows) return CHIARO_ERR_CAPACITY;
    struct Measured {
        bool some;
        float shift[2];
        float score;
    };
    std::vector<Measured> measured(columns * rows, Measured{false, {0, 0}, 0});
    for (size_t row = 0; row < rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            const float rx = (float)(column * STEP), ry = (float)(row * STEP);
            if (rx >= (float)width || ry >= (float)height) continue;
            const long plane_x = (long)std::round((rx - 0.5f) * 0.5f), plane_y = (long)std::round((ry - 0.5f) * 0.5f);
            const long x = plane_x - (long)PATCH / 2, y = plane_y - (long)PATCH / 2;
            if (x < (long)match_radius || y < (long)match_radius ||
                x + (long)PATCH + (long)match_radius > (long)reference.width ||
                y + (long)PATCH + (long)match_radius > (long)reference.height)
                continue;
            // rendered_window_is_covered (resolution.rs:467-484)
            bool covered = true;
            for (size_t yy = (size_t)y - match_radius; yy < (size_t)y + PATCH + match_radius && covered; ++yy)
                for (size_t xx = (size_t)x - match_radius; xx < (size_t)x + PATCH + match_radius && covered; ++xx)
                    covered = std::isfinite(rendered.at(xx, yy));
            if (!covered) continue;
            auto found = match_patch_o(reference, rendered, (size_t)x, (size_t)y, PATCH, match_radius);
            if (found && found->score >= MINIMUM_SCORE)
                measured[row * columns + column] =
                    Measured{true, {found->shift[0] * 2.0f, found->shift[1] * 2.0f}, found->score};
        }
    // resolution.rs:307-361
    struct Correction {
        bool some;
        float v[2];
    };
    std::vector<float> confidence(columns * rows);
    std::vector<Correction> grid(columns * rows);
    std::vector<float> corrections;
    float confidence_sum = 0.0f;
    for (size_t row = 0; row < rows; ++row)
        for (size_t column = 0; column < columns; ++column) {
            const float rx = (float)(column * STEP), ry = (float)(row * STEP);
            const size_t index = row * columns + column;
            std::optional<std::pair<F2, std::pair<float, F2>>> refined;
            if (measured[index].some) {
                std::vector<float> xs, ys;
                for (size_t nr = row > 0 ? row - 1 : 0; nr <= std::min(row + 1, rows - 1); ++nr)
                    for (size_t nc = column > 0 ? column - 1 : 0; nc <= std::min(column + 1, columns - 1); ++nc)
                        if (measured[nr * columns + nc].some) {
                            xs.push_back(measured[nr * columns + nc].shift[0]);
                            ys.push_back(measured[nr * columns + nc].shift[1]);
                        }
                if (xs.size() >= 3) {
                    std::stable_sort(xs.begin(), xs.end(), total_less_o);
                    std::stable_sort(ys.begin(), ys.end(), total_less_o);
                    const F2 median = {xs[xs.size() / 2], ys[ys.size() / 2]};
                    const Measured &c = measured[index];
                    if (!(std::hypot(c.shift[0] - median[0], c.shift[1] - median[1]) > 1.5f))
                        if (auto q = base.map(rx + median[0], ry + median[1])) {
                            const float v = clamp_rust_o((c.score - MINIMUM_SCORE) / 0.20f, 0.0f, 1.0f);
                            const float score_confidence = v * v * (3.0f - 2.0f * v);  // smoothstep
                            const float base_confidence = warp_confidence_o(*base_c, rx, ry);
                            refined = std::make_pair(*q, std::make_pair(score_confidence * base_confidence, median));
                        }
                }
            }
            if (refined) {
                out->points[2 * index] = refined->first[0];
                out->points[2 * index + 1] = refined->first[1];
                confidence[index] = refined->second.first;
                grid[index] = Correction{true, {refined->second.second[0], refined->second.second[1]}};
                corrections.push_back(std::hypot(refined->second.second[0], refined->second.second[1]));
                confidence_sum += refined->second.first;
            } else {
                auto q = base.map(rx, ry);
                out->points[2 * index] = q ? (*q)[0] : std::numeric_limits<float>::quiet_NaN();
                out->points[2 * index + 1] = q ? (*q)[1] : std::numeric_limits<float>::quiet_NaN();
                confidence[index] = 0.0f;
                grid[index] = Correction{false, {0, 0}};
            }
        }
    // resolution.rs:362-415
    for (int pass = 0; pass < 2; ++pass) {
        const auto grid_snapshot = grid;
        const auto confidence_snapshot = confidence;
        for (size_t row = 0; row < rows; ++row)
            for (size_t column = 0; column < columns; ++column) {
                const size_t index = row * columns + column;
                if (grid_snapshot[index].some) continue;
                std::vector<float> xs, ys;
                float neighbour_sum = 0.0f;
                for (size_t nr = row > 0 ? row - 1 : 0; nr <= std::min(row + 1, rows - 1); ++nr)
                    for (size_t nc = column > 0 ? column - 1 : 0; nc <= std::min(column + 1, columns - 1); ++nc) {
                        const size_t neighbour = nr * columns + nc;
                        if (grid_snapshot[neighbour].some) {
                            xs.push_back(grid_snapshot[neighbour].v[0]);
                            ys.push_back(grid_snapshot[neighbour].v[1]);
                            neighbour_sum += confidence_snapshot[neighbour];
                        }
                    }
                if (xs.size() < 3) continue;
                std::stable_sort(xs.begin(), xs.end(), total_less_o);
                std::stable_sort(ys.begin(), ys.end(), total_less_o);
                const F2 correction = {xs[xs.size() / 2], ys[ys.size() / 2]};
                bool coherent = true;
                for (size_t k = 0; k < xs.size(); ++k)
                    if (!(std::hypot(xs[k] - correction[0], ys[k] - correction[1]) <= 1.5f)) {
                        coherent = false;
                        break;
                    }
                if (!coherent) continue;
                const float rx = (float)(column * STEP), ry = (float)(row * STEP);
                if (auto q = base.map(rx + correction[0], ry + correction[1])) {
                    out->points[2 * index] = (*q)[0];
                    out->points[2 * index + 1] = (*q)[1];
                    confidence[index] = 0.45f * neighbour_sum / (float)xs.size();
                    grid[index] = Correction{true, {correction[0], correction[1]}};
                }
            }
    }
    std::stable_sort(corrections.begin(), corrections.end(), total_less_o);
    const size_t verified = corrections.size();
    size_t supported = 0;
    for (float c : confidence) supported += c > 0.0f;
    if (out->confidence) std::copy(confidence.begin(), confidence.end(), out->confidence);
    const float cells = (float)std::max<size_t>(columns * rows, 1);
    report[0] = (float)verified / cells;
    report[1] = (float)supported / cells;
    report[2] = verified ? corrections[verified / 2] : 0.0f;
    report[3] = confidence_sum / (float)std::max<size_t>(verified, 1);
    return CHIARO_OK;
}

// ---- align.rs: align_module_seeded (281-519) and its helpers (521-830) -------------------

namespace {

struct PlaneBuf {  // an owned Plane
    size_t width = 0, height = 0;
    std::vector<float> data;
    Plane view() const {
        Plane p;
        p.width = width;
        p.height = height;
        p.data = data.data();
        return p;
    }
    float at(size_t x, size_t y) const { return data[y * width + x]; }
};

PlaneBuf plane_copy(const float *data, size_t width, size_t height) {
    PlaneBuf p;
    p.width = width;
    p.height = height;
    p.data.assign(data, data + width * height);
    return p;
}

// Plane::downsample (image.rs:469-483)
PlaneBuf downsample_o(const PlaneBuf &in) {
    PlaneBuf out;
    out.width = std::max<size_t>(in.width / 2, 1);
    out.height = std::max<size_t>(in.height / 2, 1);
    out.data.resize(out.width * out.height);
    for (size_t j = 0; j < out.height; ++j)
        for (size_t i = 0; i < out.width; ++i) {
            const size_t x = 2 * i, y = 2 * j, x1 = std::min(x + 1, in.width - 1), y1 = std::min(y + 1, in.height - 1);
            out.data[j * out.width + i] = 0.25f * (in.at(x, y) + in.at(x1, y) + in.at(x, y1) + in.at(x1, y1));
        }
    return out;
}

// Plane::pyramid (image.rs:487-497)
std::vector<PlaneBuf> pyramid_o(const PlaneBuf &base, size_t min_size) {
    std::vector<PlaneBuf> levels{base};
    while (std::min(levels.back().width, levels.back().height) / 2 >= std::max<size_t>(min_size, 8))
        levels.push_back(downsample_o(levels.back()));
    return levels;
}

struct OwnedWarp {  // Warp with owned arrays
    size_t step = 0, columns = 0, rows = 0;
    std::vector<float> points, confidence;
    Warp view() const {
        Warp w;
        w.step = step;
        w.columns = columns;
        w.rows = rows;
        w.points = points.data();
        return w;
    }
};

// Warp::from_fn (align.rs:50-80)
template <class F>
OwnedWarp from_fn_o(size_t width, size_t height, size_t step, F map) {
    OwnedWarp w;
    w.step = step;
    w.columns = div_ceil(width, step) + 1;
    w.rows = div_ceil(height, step) + 1;
    for (size_t row = 0; row < w.rows; ++row)
        for (size_t column = 0; column < w.columns; ++column) {
            const Vec2 p = {(double)(column * step), (double)(row * step)};
            const std::optional<Vec2> q = map(p);
            if (q) {
                w.points.push_back((float)(*q)[0]);
                w.points.push_back((float)(*q)[1]);
                w.confidence.push_back(1.0f);
            } else {
                w.points.push_back(std::numeric_limits<float>::quiet_NaN());
                w.points.push_back(std::numeric_limits<float>::quiet_NaN());
                w.confidence.push_back(0.0f);
            }
        }
    return w;
}

Mat3 mat_mul_o(const Mat3 &a, const Mat3 &b) {  // math.rs:48-56
    Mat3 out{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
    return out;
}

std::optional<Vec2> apply_homography_o(const Mat3 &h, const Vec2 &p) {  // math.rs:131-138
    const Vec3 v = mul_vec(h, {p[0], p[1], 1.0});
    if (std::fabs(v[2]) < 1e-12) return std::nullopt;
    return Vec2{v[0] / v[2], v[1] / v[2]};
}

// solve_linear (align.rs:765-793)
std::optional<std::array<double, 8>> solve_linear_o(std::array<std::array<double, 8>, 8> a, std::array<double, 8> b) {
    for (size_t column = 0; column < 8; ++column) {
        size_t pivot = column;  // max_by(total_cmp) over |a[i][column]|: the last maximum
        for (size_t i = column + 1; i < 8; ++i)
            if (!(total_key_f64(std::fabs(a[i][column])) < total_key_f64(std::fabs(a[pivot][column])))) pivot = i;
        if (std::fabs(a[pivot][column]) < 1e-12) return std::nullopt;
        std::swap(a[column], a[pivot]);
        std::swap(b[column], b[pivot]);
        const std::array<double, 8> pivot_row = a[column];
        for (size_t row = column + 1; row < 8; ++row) {
            const double factor = a[row][column] / pivot_row[column];
            for (size_t k = column; k < 8; ++k) a[row][k] -= factor * pivot_row[k];
            b[row] -= factor * b[column];
        }
    }
    std::array<double, 8> x{};
    for (int row = 7; row >= 0; --row) {
        double sum = b[row];
        for (size_t k = row + 1; k < 8; ++k) sum -= a[row][k] * x[k];
        x[row] = sum / a[row][row];
    }
    return x;
}

struct PairO {
    Vec2 a, b;
    float score;
};

// fit_homography_least_squares (align.rs:702-760)
std::optional<Mat3> fit_least_squares_o(const std::vector<PairO> &pairs) {
    if (pairs.size() < 4) return std::nullopt;
    const double n = (double)pairs.size();
    auto mean = [&](auto f) {
        double s = -0.0;  // f64 Sum
        for (const PairO &p : pairs) s += f(p);
        return s / n;
    };
    const double ax = mean([](const PairO &p) { return p.a[0]; }), ay = mean([](const PairO &p) { return p.a[1]; });
    const double bx = mean([](const PairO &p) { return p.b[0]; }), by = mean([](const PairO &p) { return p.b[1]; });
    const double sa = dmax_r(mean([&](const PairO &p) {
        return std::sqrt((p.a[0] - ax) * (p.a[0] - ax) + (p.a[1] - ay) * (p.a[1] - ay));
    }), 1e-9);
    const double sb = dmax_r(mean([&](const PairO &p) {
        return std::sqrt((p.b[0] - bx) * (p.b[0] - bx) + (p.b[1] - by) * (p.b[1] - by));
    }), 1e-9);
    std::array<std::array<double, 8>, 8> ata{};
    std::array<double, 8> atb{};
    for (const PairO &p : pairs) {
        const double w = dmax_r((double)p.score, 0.05);
        const double x = (p.a[0] - ax) / sa, y = (p.a[1] - ay) / sa;
        const double u = (p.b[0] - bx) / sb, v = (p.b[1] - by) / sb;
        const double rows[2][8] = {{x, y, 1.0, 0.0, 0.0, 0.0, -u * x, -u * y}, {0.0, 0.0, 0.0, x, y, 1.0, -v * x, -v * y}};
        const double rhs[2] = {u, v};
        for (int r = 0; r < 2; ++r)
            for (int i = 0; i < 8; ++i) {
                atb[i] += w * rows[r][i] * rhs[r];
                for (int j = 0; j < 8; ++j) ata[i][j] += w * rows[r][i] * rows[r][j];
            }
    }
    const auto s = solve_linear_o(ata, atb);
    if (!s) return std::nullopt;
    const Mat3 normalized = {{{(*s)[0], (*s)[1], (*s)[2]}, {(*s)[3], (*s)[4], (*s)[5]}, {(*s)[6], (*s)[7], 1.0}}};
    const Mat3 t_a = {{{1.0 / sa, 0.0, -ax / sa}, {0.0, 1.0 / sa, -ay / sa}, {0.0, 0.0, 1.0}}};
    const Mat3 t_b_inv = {{{sb, 0.0, bx}, {0.0, sb, by}, {0.0, 0.0, 1.0}}};
    Mat3 h = mat_mul_o(mat_mul_o(t_b_inv, normalized), t_a);
    const double scale = h[2][2];
    if (std::fabs(scale) < 1e-12 || !std::isfinite(scale)) return std::nullopt;
    for (auto &row : h)
        for (double &v : row) v = v / scale;
    return h;
}

struct FitO {
    Mat3 h;
    size_t inliers;
    std::vector<float> residuals;
};

// fit_homography_ransac (align.rs:631-700)
std::optional<FitO> fit_ransac_o(const std::vector<PairO> &pairs, float threshold) {
    if (pairs.size() < 6) return std::nullopt;
    std::vector<size_t> best_inliers;
    uint64_t state = 0x9E3779B97F4A7C15ull ^ (uint64_t)pairs.size();
    auto next = [&](size_t n) {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return (size_t)(state >> 33) % n;
    };
    for (int iteration = 0; iteration < 300; ++iteration) {
        size_t sample[4] = {0, 0, 0, 0};
        for (int slot = 0; slot < 4; ++slot)
            for (;;) {
                const size_t candidate = next(pairs.size());
                bool taken = false;
                for (int k = 0; k < slot; ++k) taken = taken || sample[k] == candidate;
                if (!taken) {
                    sample[slot] = candidate;
                    break;
                }
            }
        std::vector<PairO> subset;
        for (size_t i : sample) subset.push_back(pairs[i]);
        const auto h = fit_least_squares_o(subset);
        if (!h) continue;
        std::vector<size_t> inliers;
        for (size_t i = 0; i < pairs.size(); ++i) {
            const auto p = apply_homography_o(*h, pairs[i].a);
            if (p && std::sqrt(((*p)[0] - pairs[i].b[0]) * ((*p)[0] - pairs[i].b[0]) +
                               ((*p)[1] - pairs[i].b[1]) * ((*p)[1] - pairs[i].b[1])) <= (double)threshold)
                inliers.push_back(i);
        }
        if (inliers.size() > best_inliers.size()) best_inliers = inliers;
    }
    if (best_inliers.size() < 6) return std::nullopt;
    std::vector<PairO> inlier_pairs;
    for (size_t i : best_inliers) inlier_pairs.push_back(pairs[i]);
    const auto h = fit_least_squares_o(inlier_pairs);
    if (!h) return std::nullopt;
    FitO fit{*h, 0, {}};
    for (const PairO &pair : pairs)
        if (auto p = apply_homography_o(*h, pair.a)) {
            const float r = (float)std::sqrt(((*p)[0] - pair.b[0]) * ((*p)[0] - pair.b[0]) +
                                             ((*p)[1] - pair.b[1]) * ((*p)[1] - pair.b[1]));
            if (r <= threshold) {
                ++fit.inliers;
                fit.residuals.push_back(r);
            }
        }
    if (fit.inliers < 6) return std::nullopt;
    std::stable_sort(fit.residuals.begin(), fit.residuals.end(), total_less_o);
    return fit;
}

// photometric_gain (align.rs:795-826)
std::optional<float> photometric_gain_o(const Plane &reference, const Plane &target, const Warp &warp) {
    std::vector<float> ratios;
    const size_t step = 16;
    for (size_t y = step; y + step < reference.height; y += step)
        for (size_t x = step; x + step < reference.width; x += step) {
            const float rx = (float)x * 2.0f + 0.5f, ry = (float)y * 2.0f + 0.5f;
            const auto q = warp.map(rx, ry);
            if (!q) continue;
            const auto t = target.sample(((*q)[0] - 0.5f) / 2.0f, ((*q)[1] - 0.5f) / 2.0f);
            if (!t) continue;
            const float r = reference.at(x, y);
            const float lr = (std::exp(r) - 1.0f) / 1000.0f, lt = (std::exp(*t) - 1.0f) / 1000.0f;
            if (lr > 0.01f && lt > 0.01f && lr < 0.95f && lt < 0.95f) ratios.push_back(lr / lt);
        }
    if (ratios.size() < 16) return std::nullopt;
    std::stable_sort(ratios.begin(), ratios.end(), total_less_o);
    return clamp_rust_o(ratios[ratios.size() / 2], 0.25f, 4.0f);
}

// coarse_global_shift (align.rs:561-628); nullopt with a message for Err
std::optional<Vec2> coarse_global_shift_o(const PlaneBuf &reference_luma, const PlaneBuf &target_luma, double scale,
                                          float min_score, std::string &error) {
    const auto reference_pyramid = pyramid_o(reference_luma, 32);
    const PlaneBuf &reference_plane = reference_pyramid.back();
    const double reference_scale = (double)((size_t)1 << (reference_pyramid.size() - 1));
    const auto target_pyramid = pyramid_o(target_luma, 16);
    const double wanted = reference_scale * scale;
    const size_t target_level =
        std::min(sat_usize(dmax_r(std::round(std::log2(wanted)), 0.0)), target_pyramid.size() - 1);
    const PlaneBuf &target_plane = target_pyramid[target_level];
    const double target_scale = (double)((size_t)1 << target_level);
    const float ratio = (float)(target_scale / wanted);
    const size_t rw = sat_usize(fmax_r(std::floor((float)target_plane.width * ratio), 4.0f));
    const size_t rh = sat_usize(fmax_r(std::floor((float)target_plane.height * ratio), 4.0f));
    PlaneBuf resampled;
    resampled.width = rw;
    resampled.height = rh;
    resampled.data.resize(rw * rh);
    const Plane tp = target_plane.view();
    for (size_t y = 0; y < rh; ++y)
        for (size_t x = 0; x < rw; ++x) resampled.data[y * rw + x] = tp.sample((float)x / ratio, (float)y / ratio).value_or(0.0f);
    if (rw + 2 > reference_plane.width || rh + 2 > reference_plane.height) return Vec2{0.0, 0.0};
    const size_t patch = std::min({rw, rh, reference_plane.width / 2, reference_plane.height / 2});
    const size_t radius = std::max<size_t>((std::min(reference_plane.width, reference_plane.height) - patch) / 2, 1);
    const size_t rx = (reference_plane.width - patch) / 2, ry = (reference_plane.height - patch) / 2;
    const size_t tx = (rw - patch) / 2, ty = (rh - patch) / 2;
    PlaneBuf embedded;
    embedded.width = reference_plane.width;
    embedded.height = reference_plane.height;
    embedded.data.assign(embedded.width * embedded.height, std::numeric_limits<float>::quiet_NaN());
    for (size_t y = 0; y < patch; ++y)
        for (size_t x = 0; x < patch; ++x) embedded.data[(ry + y) * embedded.width + rx + x] = resampled.at(tx + x, ty + y);
    const auto found =
        match_patch_o(reference_plane.view(), embedded.view(), rx, ry, patch, std::min({radius, rx, ry}));
    if (!found) {
        error = "no correlation between the module and the reference";
        return std::nullopt;
    }
    if (found->score < min_score * 0.6f) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "module does not correlate with the reference (%.2f)", found->score);
        error = buf;
        return std::nullopt;
    }
    return Vec2{-(double)found->shift[0] * reference_scale * 2.0 * scale,
                -(double)found->shift[1] * reference_scale * 2.0 * scale};
}

}  // namespace

// fit_homography_ransac (align.rs:631-700) over (ax, ay, bx, by) pairs with f32 scores.
// Returns 0 for None; h is row-major.
extern "C" int oracle_fit_homography_ransac(const double *points, const float *scores, size_t n, float threshold,
                                            double *h, size_t *inliers, float *residuals) {
    std::vector<PairO> pairs(n);
    for (size_t i = 0; i < n; ++i)
        pairs[i] = PairO{{points[4 * i], points[4 * i + 1]}, {points[4 * i + 2], points[4 * i + 3]}, scores[i]};
    const auto fit = fit_ransac_o(pairs, threshold);
    if (!fit) return 0;
    for (int i = 0; i < 9; ++i) h[i] = fit->h[i / 3][i % 3];
    *inliers = fit->inliers;
    if (residuals) std::copy(fit->residuals.begin(), fit->residuals.end(), residuals);
    return 1;
}

// align_module_seeded (align.rs:281-519). error (optional, 128 bytes) receives the Err message.
extern "C" int oracle_align_module(const chiaro_align_input *reference, const chiaro_align_input *target,
                                   int target_is_reference, const chiaro_align_options *options,
                                   const chiaro_warp *seed, chiaro_warp *out_warp, float *gain,
                                   chiaro_alignment_report *report, char *error) {
    constexpr double FAR_DEPTH = 1.0e8;
    const size_t width = (size_t)reference->width, height = (size_t)reference->height;
    std::memset(report, 0, sizeof(*report));
    auto emit = [&](const OwnedWarp &w) {
        out_warp->step = w.step;
        out_warp->columns = w.columns;
        out_warp->rows = w.rows;
        if (out_warp->capacity < w.columns * w.rows) return (int)CHIARO_ERR_CAPACITY;
        std::copy(w.points.begin(), w.points.end(), out_warp->points);
        if (out_warp->confidence) std::copy(w.confidence.begin(), w.confidence.end(), out_warp->confidence);
        return (int)CHIARO_OK;
    };
    if (target_is_reference) {
        const OwnedWarp w = from_fn_o(width, height, options->grid_step, [](const Vec2 &p) { return std::optional<Vec2>(p); });
        report->initialised_from = CHIARO_INIT_REFERENCE;
        report->coverage = 1.0f;
        report->inlier_ratio = 1.0f;
        report->accepted = 1;
        report->status = CHIARO_ALIGN_REFERENCE;
        *gain = 1.0f;
        return emit(w);
    }
    const PlaneBuf reference_luma = plane_copy(reference->luminance, reference->luma_width, reference->luma_height);
    const PlaneBuf target_luma = plane_copy(target->luminance, target->luma_width, target->luma_height);
    // Step 1 (align.rs:311-345)
    OwnedWarp initial_grid;
    if (seed) {
        report->initialised_from = CHIARO_INIT_SEED;
        initial_grid.step = seed->step;
        initial_grid.columns = seed->columns;
        initial_grid.rows = seed->rows;
        initial_grid.points.assign(seed->points, seed->points + 2 * seed->columns * seed->rows);
        initial_grid.confidence.assign(seed->columns * seed->rows, 1.0f);
        if (seed->confidence) initial_grid.confidence.assign(seed->confidence, seed->confidence + seed->columns * seed->rows);
    } else if (reference->has_camera && target->has_camera) {
        report->initialised_from = CHIARO_INIT_CALIBRATION;
        const Camera reference_camera(reference->camera), target_camera(target->camera);
        initial_grid = from_fn_o(width, height, 8, [&](const Vec2 &p) -> std::optional<Vec2> {
            auto q = target_camera.map_from(reference_camera, p, FAR_DEPTH);
            if (q && std::isfinite((*q)[0]) && std::isfinite((*q)[1])) return q;
            return std::nullopt;
        });
    } else {
        report->initialised_from = CHIARO_INIT_NOMINAL_FOCAL_GROUP;
        const double scale = target->nominal_focal_px / reference->nominal_focal_px;
        const double cx = ((double)width - 1.0) / 2.0, cy = ((double)height - 1.0) / 2.0;
        const double tx = ((double)target->width - 1.0) / 2.0, ty = ((double)target->height - 1.0) / 2.0;
        std::string message;
        const auto shift = coarse_global_shift_o(reference_luma, target_luma, scale, options->min_score, message);
        if (!shift) {
            if (error) std::snprintf(error, 128, "%s", message.c_str());
            return CHIARO_INVALID;
        }
        initial_grid = from_fn_o(width, height, 8, [&](const Vec2 &p) -> std::optional<Vec2> {
            return Vec2{(p[0] - cx) * scale + tx + (*shift)[0], (p[1] - cy) * scale + ty + (*shift)[1]};
        });
    }
    const Warp initial_view = initial_grid.view();
    auto initial = [&](const Vec2 &p) -> std::optional<Vec2> {
        auto q = initial_view.map((float)p[0], (float)p[1]);
        if (!q) return std::nullopt;
        return Vec2{(double)(*q)[0], (double)(*q)[1]};
    };
    // Step 2 (align.rs:347-455)
    Mat3 correction = {{{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}}};
    std::vector<float> finest_residuals;
    if (options->refine) {
        const auto reference_pyramid = pyramid_o(reference_luma, 96);
        const auto target_pyramid = pyramid_o(target_luma, 48);
        double magnification;
        {
            const Vec2 c = {(double)width / 2.0, (double)height / 2.0};
            const double h = 64.0;
            const auto a = initial(c), b = initial({c[0] + h, c[1]}), d = initial({c[0], c[1] + h});
            if (a && b && d) {
                const double dx = std::sqrt(((*b)[0] - (*a)[0]) * ((*b)[0] - (*a)[0]) + ((*b)[1] - (*a)[1]) * ((*b)[1] - (*a)[1])) / h;
                const double dy = std::sqrt(((*d)[0] - (*a)[0]) * ((*d)[0] - (*a)[0]) + ((*d)[1] - (*a)[1]) * ((*d)[1] - (*a)[1])) / h;
                magnification = std::sqrt(dx * dy);
            } else {
                magnification = target->nominal_focal_px / reference->nominal_focal_px;
            }
        }
        for (size_t level = reference_pyramid.size(); level-- > 0;) {
            const size_t scale = (size_t)1 << level;
            const Plane reference_plane = reference_pyramid[level].view();
            const size_t target_level = std::min(
                sat_usize(dmax_r(std::round(std::log2((double)scale * magnification)), 0.0)), target_pyramid.size() - 1);
            const Plane target_plane = target_pyramid[target_level].view();
            const double target_scale = (double)((size_t)1 << target_level);
            // render_through (align.rs:523-549)
            PlaneBuf rendered;
            rendered.width = reference_plane.width;
            rendered.height = reference_plane.height;
            rendered.data.resize(rendered.width * rendered.height);
            for (size_t y = 0; y < rendered.height; ++y)
                for (size_t x = 0; x < rendered.width; ++x) {
                    auto to_raster = [&](float v) { return ((double)v * (double)scale * 2.0) + (double)scale - 0.5; };
                    auto from_raster = [&](double v) { return (float)((v + 0.5) / (2.0 * target_scale) - 0.5); };
                    float value = std::numeric_limits<float>::quiet_NaN();
                    if (auto c = apply_homography_o(correction, {to_raster((float)x), to_raster((float)y)}))
                        if (auto q = initial(*c))
                            if (auto s = target_plane.sample(from_raster((*q)[0]), from_raster((*q)[1]))) value = *s;
                    rendered.data[y * rendered.width + x] = value;
                }
            const Plane rendered_view = rendered.view();
            const size_t radius = level + 1 == reference_pyramid.size() ? (size_t)options->coarse_radius : 3;
            const size_t patch = std::max<size_t>(std::min<size_t>(options->patch, reference_plane.width / 4), 8);
            std::vector<PairO> pairs;
            const size_t stride = patch / 2;
            for (size_t y = radius; y + patch + radius <= reference_plane.height; y += stride)
                for (size_t x = radius; x + patch + radius <= reference_plane.width; x += stride) {
                    bool covered = true;  // rendered_covered (align.rs:551-559)
                    for (size_t row = y; row < y + patch && covered; ++row)
                        for (size_t col = x; col < x + patch && covered; ++col)
                            covered = !std::isnan(rendered_view.at(col, row));
                    if (!covered) continue;
                    const auto found = match_patch_o(reference_plane, rendered_view, x, y, patch, radius);
                    if (!found || !(found->score >= options->min_score)) continue;
                    auto convert = [&](float v) { return (double)v * (double)scale * 2.0 + (double)scale - 0.5; };
                    const float half = (float)patch / 2.0f;
                    const Vec2 centre = {convert((float)x + half), convert((float)y + half)};
                    const Vec2 shifted = {convert((float)x + half + found->shift[0]), convert((float)y + half + found->shift[1])};
                    pairs.push_back(PairO{centre, shifted, found->score});
                }
            const float threshold = fmax_r(options->inlier_px * (float)scale * 2.0f, options->inlier_px);
            chiaro_align_level &lr = report->levels[report->n_levels < CHIARO_ALIGN_MAX_LEVELS ? report->n_levels : CHIARO_ALIGN_MAX_LEVELS - 1];
            if (auto fit = fit_ransac_o(pairs, threshold)) {
                correction = mat_mul_o(correction, fit->h);
                lr = chiaro_align_level{scale * 2, pairs.size(), fit->inliers, fit->residuals[fit->residuals.size() / 2]};
                if (level == 0) {
                    finest_residuals = fit->residuals;
                    report->patches = pairs.size();
                    report->inliers = fit->inliers;
                }
            } else {
                lr = chiaro_align_level{scale * 2, pairs.size(), 0, std::numeric_limits<float>::quiet_NaN()};
            }
            if (report->n_levels < CHIARO_ALIGN_MAX_LEVELS) ++report->n_levels;
        }
    }
    // Final warp and report (align.rs:457-519)
    const OwnedWarp warp = from_fn_o(width, height, options->grid_step, [&](const Vec2 &p) -> std::optional<Vec2> {
        auto corrected = apply_homography_o(correction, p);
        if (!corrected) return std::nullopt;
        return initial(*corrected);
    });
    size_t covered = 0;
    for (size_t i = 0; i < warp.columns * warp.rows; ++i) {
        const float qx = warp.points[2 * i], qy = warp.points[2 * i + 1];
        covered += std::isfinite(qx) && qx >= 0.0f && qy >= 0.0f && qx <= (float)(target->width - 1) &&
                   qy <= (float)(target->height - 1);
    }
    report->coverage = (float)covered / (float)(warp.columns * warp.rows);
    if (!finest_residuals.empty()) {
        report->residual_median_px = finest_residuals[finest_residuals.size() / 2];
        report->residual_p90_px = finest_residuals[std::min(finest_residuals.size() * 9 / 10, finest_residuals.size() - 1)];
    }
    {
        const Vec2 centre = {(double)(width / 2), (double)(height / 2)};
        const Vec2 moved = apply_homography_o(correction, centre).value_or(centre);
        report->correction_median_px[0] = (float)(moved[0] - centre[0]);
        report->correction_median_px[1] = (float)(moved[1] - centre[1]);
    }
    report->inlier_ratio = report->patches == 0 ? 0.0f : (float)report->inliers / (float)report->patches;
    report->accepted = !options->refine || report->inlier_ratio >= options->min_inlier_ratio;
    report->status = !report->accepted ? CHIARO_ALIGN_REJECTED
                     : !options->refine ? CHIARO_ALIGN_FACTORY_MODEL
                     : report->inliers >= 12 && report->residual_median_px < options->inlier_px ? CHIARO_ALIGN_REFINED
                     : report->inliers > 0 ? CHIARO_ALIGN_WEAK_REFINEMENT
                                           : CHIARO_ALIGN_NO_SUPPORT;
    *gain = photometric_gain_o(reference_luma.view(), target_luma.view(), warp.view()).value_or(1.0f);
    return emit(warp);
}

// Warp::confidence (align.rs:113-131) at one point.
extern "C" float oracle_warp_confidence(const chiaro_warp *w, float x, float y) { return warp_confidence_o(*w, x, y); }

// DenseDepthMap::sample_nearest (depth.rs:152-159): the node index, or -1 for None.
extern "C" long oracle_sample_nearest(const chiaro_depth_map *map, float x, float y) {
    if (x < 0.0f || y < 0.0f || map->step == 0) return -1;
    const size_t column = sat_usize(std::round(x / (float)map->step));
    const size_t row = sat_usize(std::round(y / (float)map->step));
    if (!(column < map->columns && row < map->rows)) return -1;
    return (long)(row * map->columns + column);
}
