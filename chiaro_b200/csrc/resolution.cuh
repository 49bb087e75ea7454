// resolution.cuh — refine_resolution_warp (crates/chiaro-fusion/src/resolution.rs:232-439):
// the resolution-domain local refinement of a module's warp. Two kernels carry its
// per-pixel and per-node work; the 32 px control grid's median filter and hole
// completion (resolution.rs:307-423) run on the host beside them (stage.cu).
//
// * resolution_render_kernel: the target brought to the reference plane's sampling
//   (resolution.rs:255-271), a thread per reference-plane pixel: the base warp at
//   the pixel's raster position, then sample_at_reference_bandwidth
//   (resolution.rs:441-465): a bilinear sample, or for a magnified target the
//   Gaussian footprint over (2R + 1)^2 bilinear samples summed in the reference's
//   order. NaN where the warp or the samples are undefined.
// * resolution_match_kernel: the control-grid nodes' patch searches
//   (resolution.rs:275-305 with match_patch, image.rs:531-640), a warp per node: the
//   12 x 12 reference window's statistics by lane 0 in the reference's summation
//   order, one (2r + 1)^2 shift per lane at a time (each shift's three sums run in
//   the reference's row order), then the last maximum in total order and the
//   parabolic sub-pixel refinement.
#pragma once

#include "common.cuh"

namespace chiaro {

constexpr int RES_WARP_STEP = 32;      // LOCAL_WARP_STEP
constexpr int RES_PATCH = 12;          // LOCAL_MATCH_PATCH
constexpr int RES_RADIUS = 2;          // LOCAL_MATCH_RADIUS
constexpr int RES_MAGNIFIED_RADIUS = 5;  // MAGNIFIED_MATCH_RADIUS
constexpr float RES_MINIMUM_SCORE = 0.72f;  // LOCAL_MINIMUM_SCORE
constexpr int RES_MAX_SPAN = 2 * RES_MAGNIFIED_RADIUS + 1;

struct ResolutionNode {  // one control node's measurement
    float shift_x, shift_y, score;
    int measured;  // 1: a match with score >= RES_MINIMUM_SCORE
};

// sample_at_reference_bandwidth (resolution.rs:441-465); false for None.
__device__ __forceinline__ bool sample_at_reference_bandwidth(const PlaneRef &target, float x, float y,
                                                              float magnification, float &out) {
    if (magnification <= 1.15f) return plane_sample(target, x, y, out);
    const float sigma = fmaxf(0.42f * magnification, 0.55f);
    const float r = fminf(fmaxf(ceilf(2.0f * sigma), 1.0f), 4.0f);
    const int radius = (int)r;
    float sum = 0.0f, weight = 0.0f;
    for (int dy = -radius; dy <= radius; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
            const float distance_squared = (float)(dx * dx + dy * dy);
            const float kernel = exp_f32(-0.5f * distance_squared / (sigma * sigma));
            float value;
            if (plane_sample(target, x + (float)dx, y + (float)dy, value)) {
                sum += kernel * value;
                weight += kernel;
            }
        }
    if (!(weight > 1.0e-8f)) return false;
    out = sum / weight;
    return true;
}

__global__ void resolution_render_kernel(PlaneRef target, WarpRef base, float magnification, int width, int height,
                                         float *__restrict__ rendered) {
    const long total = (long)width * height;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int y = (int)(i / width), x = (int)(i - (long)y * width);
        const float rx = (float)x * 2.0f + 0.5f, ry = (float)y * 2.0f + 0.5f;
        float qx, qy, value = NAN;
        if (warp_map(base, rx, ry, qx, qy)) {
            float v;
            if (sample_at_reference_bandwidth(target, (qx + 0.5f) * 0.5f - 0.5f, (qy + 0.5f) * 0.5f - 0.5f,
                                              magnification, v))
                value = v;
        }
        rendered[i] = value;
    }
}

// Rust's f32::clamp: NaN passes through.
__device__ __forceinline__ float clamp_rust(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// The parabolic refinement of match_patch (image.rs:603-610).
__device__ __forceinline__ float patch_refine(float minus, float center, float plus) {
    const float denominator = minus - 2.0f * center + plus;
    if (fabsf(denominator) < 1.0e-9f) return 0.0f;
    return clamp_rust(0.5f * (minus - plus) / denominator, -0.5f, 0.5f);
}

// A warp per control node (columns x rows, row-major).
__global__ void __launch_bounds__(256) resolution_match_kernel(PlaneRef reference, PlaneRef rendered, int columns,
                                                               int rows, int width, int height, int radius,
                                                               ResolutionNode *__restrict__ nodes) {
    __shared__ float ref_centered[8][RES_PATCH * RES_PATCH];
    __shared__ float scores[8][RES_MAX_SPAN * RES_MAX_SPAN];
    __shared__ float ref_std_s[8];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int node = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (node >= columns * rows) return;  // whole warp
    const int row = node / columns, column = node - row * columns;
    ResolutionNode result{0.0f, 0.0f, 0.0f, 0};
    const float rx = (float)(column * RES_WARP_STEP), ry = (float)(row * RES_WARP_STEP);
    // resolution.rs:280-296: the window and its search reach inside the reference plane
    bool ok = !(rx >= (float)width || ry >= (float)height);
    int x = 0, y = 0;
    if (ok) {
        const long plane_x = (long)roundf((rx - 0.5f) * 0.5f), plane_y = (long)roundf((ry - 0.5f) * 0.5f);
        const long xl = plane_x - RES_PATCH / 2, yl = plane_y - RES_PATCH / 2;
        ok = !(xl < radius || yl < radius || xl + RES_PATCH + radius > reference.width ||
               yl + RES_PATCH + radius > reference.height);
        x = (int)xl;
        y = (int)yl;
    }
    // rendered_window_is_covered (resolution.rs:467-484)
    if (ok) {
        const int side = RES_PATCH + 2 * radius;
        bool covered = true;
        for (int k = lane; k < side * side; k += 32) {
            const int yy = y - radius + k / side, xx = x - radius + k % side;
            covered &= isfinite(plane_at(rendered, xx, yy));
        }
        ok = __all_sync(full, covered);
    }
    // match_patch (image.rs:531-640): its own bounds (image.rs:539-549), then the reference window
    if (ok)
        ok = !(x + RES_PATCH > reference.width || y + RES_PATCH > reference.height || x < radius || y < radius ||
               x + RES_PATCH + radius > rendered.width || y + RES_PATCH + radius > rendered.height ||
               x + RES_PATCH > rendered.width || y + RES_PATCH > rendered.height);
    const float n = (float)(RES_PATCH * RES_PATCH);
    if (ok && lane == 0) {
        float sum = -0.0f;  // f32 Sum
        for (int k = 0; k < RES_PATCH * RES_PATCH; ++k) sum += plane_at(reference, x + k % RES_PATCH, y + k / RES_PATCH);
        const float mean = sum / n;
        float squares = -0.0f;
        for (int k = 0; k < RES_PATCH * RES_PATCH; ++k) {
            const float d = plane_at(reference, x + k % RES_PATCH, y + k / RES_PATCH) - mean;
            squares += d * d;
        }
        const float ref_std = sqrtf(squares / n);
        ref_std_s[w] = ref_std;
        for (int k = 0; k < RES_PATCH * RES_PATCH; ++k)
            ref_centered[w][k] = plane_at(reference, x + k % RES_PATCH, y + k / RES_PATCH) - mean;
    }
    __syncwarp();
    if (ok) ok = !(ref_std_s[w] < 1.0e-4f);
    if (ok) {
        const float ref_std = ref_std_s[w];
        const int span = 2 * radius + 1;
        for (int s = lane; s < span * span; s += 32) {
            const int dy = s / span, dx = s - dy * span;
            const int tx = x + dx - radius, ty = y + dy - radius;
            float sum = 0.0f, sum_sq = 0.0f, cross = 0.0f;
            for (int yy = 0; yy < RES_PATCH; ++yy)
                for (int xx = 0; xx < RES_PATCH; ++xx) {
                    const float t = plane_at(rendered, tx + xx, ty + yy);
                    sum += t;
                    sum_sq += t * t;
                    cross += t * ref_centered[w][yy * RES_PATCH + xx];
                }
            const float mean = sum / n;
            float var = sum_sq / n - mean * mean;
            var = var != var ? 0.0f : fmaxf(var, 0.0f);  // f32::max(0.0) ignores NaN
            scores[w][s] = var < 1.0e-8f ? -INFINITY : (cross / n) / (sqrtf(var) * ref_std);
        }
        __syncwarp();
        if (lane == 0) {
            // the last maximum in total order (Iterator::max_by with total_cmp)
            int best = 0;
            for (int s = 1; s < span * span; ++s)
                if (total_key(scores[w][s]) >= total_key(scores[w][best])) best = s;
            const float score = scores[w][best];
            if (isfinite(score)) {
                const int bx = best % span, by = best / span;
                const float sub_x = bx > 0 && bx + 1 < span
                                        ? patch_refine(scores[w][by * span + bx - 1], score, scores[w][by * span + bx + 1])
                                        : 0.0f;
                const float sub_y = by > 0 && by + 1 < span
                                        ? patch_refine(scores[w][(by - 1) * span + bx], score,
                                                       scores[w][(by + 1) * span + bx])
                                        : 0.0f;
                const float shift_x = (float)bx - (float)radius + sub_x, shift_y = (float)by - (float)radius + sub_y;
                if (score >= RES_MINIMUM_SCORE) result = ResolutionNode{shift_x * 2.0f, shift_y * 2.0f, score, 1};
            }
        }
    }
    if (lane == 0) nodes[node] = result;
}

}  // namespace chiaro
