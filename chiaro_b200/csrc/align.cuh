// align.cuh — align_module_seeded (crates/chiaro-fusion/src/align.rs:281-519): the device
// half of the global alignment. The host (align_run.cuh) builds the pyramids' shapes,
// the RANSAC samples, the refit, the final warp and the report; these kernels carry the
// per-pixel, per-patch and per-candidate work.
//
// * align_downsample_kernel: Plane::downsample (image.rs:469-483), a thread per pixel.
// * align_initial_grid_kernel: Warp::from_fn on the 8 px grid of the calibrated mapping
//   target.map_from(reference, p, FAR_DEPTH) (align.rs:317-324), a thread per node.
// * align_render_kernel: render_through (align.rs:523-549), a thread per level pixel:
//   the f64 homography, the initial grid's f32 map, the target level's sample.
// * align_match_kernel: the level's patch grid (align.rs:393-425), a warp per patch:
//   rendered_covered (align.rs:551-559) and match_patch (image.rs:531-640) with the
//   window's statistics in the reference's order by lane 0 and one search shift per
//   lane, the last maximum in total order and the parabolic refinement.
// * align_fit_kernel: the 300 RANSAC candidates (align.rs:640-659), a thread per
//   candidate: fit_homography_least_squares (align.rs:702-760) and solve_linear
//   (align.rs:765-793) on its four pairs, in f64 code shared with the host's refit.
// * align_inlier_kernel: the RANSAC inlier counts (align.rs:660-671) of every
//   candidate homography at once, a thread per (candidate, pair).
#pragma once

#include "common.cuh"

namespace chiaro {

struct Hom {  // a 3x3 homography, row-major
    double m[9];
};

// apply_homography (math.rs:131-138); false for None.
CH_HD bool apply_homography(const Hom &h, double px, double py, double &qx, double &qy) {
    const double v0 = h.m[0] * px + h.m[1] * py + h.m[2] * 1.0;
    const double v1 = h.m[3] * px + h.m[4] * py + h.m[5] * 1.0;
    const double v2 = h.m[6] * px + h.m[7] * py + h.m[8] * 1.0;
    if (fabs(v2) < 1e-12) return false;
    qx = v0 / v2;
    qy = v1 / v2;
    return true;
}

CH_HD Hom hom_identity() { return Hom{{1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0}}; }

CH_HD Hom hom_mul(const Hom &a, const Hom &b) {  // math.rs:48-56
    Hom out;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return out;
}

CH_HD int64_t total_key_f64(double v) {  // order of f64::total_cmp
    int64_t bits;
    memcpy(&bits, &v, sizeof bits);
    return bits ^ (int64_t)((uint64_t)(bits >> 63) >> 1);
}

// solve_linear (align.rs:765-793)
CH_HD bool solve_linear8(double a[8][8], double b[8], double x[8]) {
    for (int column = 0; column < 8; ++column) {
        int pivot = column;  // the last maximum of |a[i][column]| in total order
        for (int i = column + 1; i < 8; ++i)
            if (!(total_key_f64(fabs(a[i][column])) < total_key_f64(fabs(a[pivot][column])))) pivot = i;
        if (fabs(a[pivot][column]) < 1e-12) return false;
        for (int k = 0; k < 8; ++k) {
            const double tmp = a[column][k];
            a[column][k] = a[pivot][k];
            a[pivot][k] = tmp;
        }
        const double tb = b[column];
        b[column] = b[pivot];
        b[pivot] = tb;
        double pivot_row[8];
        for (int k = 0; k < 8; ++k) pivot_row[k] = a[column][k];
        for (int row = column + 1; row < 8; ++row) {
            const double factor = a[row][column] / pivot_row[column];
            for (int k = column; k < 8; ++k) a[row][k] -= factor * pivot_row[k];
            b[row] -= factor * b[column];
        }
    }
    for (int row = 7; row >= 0; --row) {
        double sum = b[row];
        for (int k = row + 1; k < 8; ++k) sum -= a[row][k] * x[k];
        x[row] = sum / a[row][row];
    }
    return true;
}

// fit_homography_least_squares (align.rs:702-760) over pairs[idx[0..n)] (idx NULL: 0..n),
// pairs as (ax, ay, bx, by) with their scores; false for None.
CH_HD bool fit_homography(const double4 *pairs, const float *scores, const int *idx, int n, Hom &h) {
    if (n < 4) return false;
    const double count = (double)n;
    double sx = -0.0, sy = -0.0, tx = -0.0, ty = -0.0;  // f64 Sum
    for (int k = 0; k < n; ++k) sx += pairs[idx ? idx[k] : k].x;
    for (int k = 0; k < n; ++k) sy += pairs[idx ? idx[k] : k].y;
    for (int k = 0; k < n; ++k) tx += pairs[idx ? idx[k] : k].z;
    for (int k = 0; k < n; ++k) ty += pairs[idx ? idx[k] : k].w;
    const double ax = sx / count, ay = sy / count, bx = tx / count, by = ty / count;
    double da = -0.0, db = -0.0;
    for (int k = 0; k < n; ++k) {
        const double4 p = pairs[idx ? idx[k] : k];
        da += sqrt((p.x - ax) * (p.x - ax) + (p.y - ay) * (p.y - ay));
    }
    for (int k = 0; k < n; ++k) {
        const double4 p = pairs[idx ? idx[k] : k];
        db += sqrt((p.z - bx) * (p.z - bx) + (p.w - by) * (p.w - by));
    }
    const double sa = fmax(da / count, 1e-9), sb = fmax(db / count, 1e-9);
    double ata[8][8], atb[8];
    for (int i = 0; i < 8; ++i) {
        atb[i] = 0.0;
        for (int j = 0; j < 8; ++j) ata[i][j] = 0.0;
    }
    for (int k = 0; k < n; ++k) {
        const int i_ = idx ? idx[k] : k;
        const double4 p = pairs[i_];
        const double w = fmax((double)scores[i_], 0.05);
        const double x = (p.x - ax) / sa, y = (p.y - ay) / sa, u = (p.z - bx) / sb, v = (p.w - by) / sb;
        const double rows[2][8] = {{x, y, 1.0, 0.0, 0.0, 0.0, -u * x, -u * y},
                                   {0.0, 0.0, 0.0, x, y, 1.0, -v * x, -v * y}};
        const double rhs[2] = {u, v};
        for (int r = 0; r < 2; ++r)
            for (int i = 0; i < 8; ++i) {
                atb[i] += w * rows[r][i] * rhs[r];
                for (int j = 0; j < 8; ++j) ata[i][j] += w * rows[r][i] * rows[r][j];
            }
    }
    double s[8];
    if (!solve_linear8(ata, atb, s)) return false;
    const Hom normalized{{s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], 1.0}};
    const Hom t_a{{1.0 / sa, 0.0, -ax / sa, 0.0, 1.0 / sa, -ay / sa, 0.0, 0.0, 1.0}};
    const Hom t_b_inv{{sb, 0.0, bx, 0.0, sb, by, 0.0, 0.0, 1.0}};
    h = hom_mul(hom_mul(t_b_inv, normalized), t_a);
    const double scale = h.m[8];
    if (fabs(scale) < 1e-12 || !isfinite(scale)) return false;
    for (int k = 0; k < 9; ++k) h.m[k] = h.m[k] / scale;
    return true;
}

// The RANSAC candidates (align.rs:640-659): candidate k fits samples[k]'s four pairs.
__global__ void align_fit_kernel(const double4 *__restrict__ pairs, const float *__restrict__ scores,
                                 const int4 *__restrict__ samples, int count, Hom *__restrict__ candidates,
                                 int *__restrict__ valid) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int4 s = samples[k];
    const int idx[4] = {s.x, s.y, s.z, s.w};
    Hom h = hom_identity();
    valid[k] = fit_homography(pairs, scores, idx, 4, h) ? 1 : 0;
    candidates[k] = h;
}

__global__ void align_downsample_kernel(const float *__restrict__ in, int width, int height, float *__restrict__ out,
                                        int out_width, int out_height) {
    const long total = (long)out_width * out_height;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
        const int j = (int)(k / out_width), i = (int)(k - (long)j * out_width);
        const int x = 2 * i, y = 2 * j, x1 = min(x + 1, width - 1), y1 = min(y + 1, height - 1);
        const float a = in[(size_t)y * width + x], b = in[(size_t)y * width + x1];
        const float c = in[(size_t)y1 * width + x], d = in[(size_t)y1 * width + x1];
        out[k] = 0.25f * (a + b + c + d);
    }
}

__global__ void align_initial_grid_kernel(DevCamera reference, DevCamera target, int columns, int rows, int step,
                                          double depth, float2 *__restrict__ points) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= columns * rows) return;
    const int row = k / columns, column = k - row * columns;
    const double px = (double)(column * step), py = (double)(row * step);
    D3 o, d;
    pixel_to_ray(reference, px, py, o, d);
    double qx, qy;
    const bool some = project(target, along(o, d, depth), qx, qy) && isfinite(qx) && isfinite(qy);
    points[k] = some ? make_float2((float)qx, (float)qy) : make_float2(NAN, NAN);
}

__global__ void align_render_kernel(int width, int height, int scale, PlaneRef target, double target_scale,
                                    WarpRef initial, Hom correction, float *__restrict__ out) {
    const long total = (long)width * height;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
        const int y = (int)(k / width), x = (int)(k - (long)y * width);
        const double s = (double)scale;
        const double px = ((double)(float)x * s * 2.0) + s - 0.5, py = ((double)(float)y * s * 2.0) + s - 0.5;
        float value = NAN;
        double cx, cy;
        if (apply_homography(correction, px, py, cx, cy)) {
            float qx, qy;
            if (warp_map(initial, (float)cx, (float)cy, qx, qy)) {
                const float tx = (float)(((double)qx + 0.5) / (2.0 * target_scale) - 0.5);
                const float ty = (float)(((double)qy + 0.5) / (2.0 * target_scale) - 0.5);
                float v;
                if (plane_sample(target, tx, ty, v)) value = v;
            }
        }
        out[k] = value;
    }
}

struct AlignMatch {
    float shift_x, shift_y, score;
    int found;  // 1: match_patch returned Some with score >= min_score
};

__device__ __forceinline__ float align_refine(float minus, float center, float plus) {
    const float denominator = minus - 2.0f * center + plus;
    if (fabsf(denominator) < 1.0e-9f) return 0.0f;
    float r = 0.5f * (minus - plus) / denominator;  // f32::clamp: NaN passes through
    if (r < -0.5f) r = -0.5f;
    if (r > 0.5f) r = 0.5f;
    return r;
}

// A warp per patch position (x0 + i * stride, y0 + j * stride), i < nx, j < ny.
// Dynamic shared memory per warp: patch^2 centred reference values and (2r + 1)^2 scores.
__global__ void align_match_kernel(PlaneRef reference, PlaneRef target, int patch, int radius, int x0, int y0,
                                   int stride, int nx, int ny, int check_covered, float min_score,
                                   AlignMatch *__restrict__ out) {
    extern __shared__ float align_smem[];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int span = 2 * radius + 1, area = patch * patch;
    float *ref_centered = align_smem + (size_t)w * (area + span * span);
    float *scores = ref_centered + area;
    __shared__ float ref_std_s[32];
    const long job = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (job >= (long)nx * ny) return;  // whole warp
    const int x = x0 + (int)(job % nx) * stride, y = y0 + (int)(job / nx) * stride;
    AlignMatch result{0.0f, 0.0f, 0.0f, 0};
    bool ok = true;
    if (check_covered) {  // rendered_covered: no NaN in the patch window
        bool covered = true;
        for (int k = lane; k < area; k += 32) covered &= !isnan(plane_at(target, x + k % patch, y + k / patch));
        ok = __all_sync(full, covered);
    }
    // match_patch's bounds (image.rs:539-549)
    if (ok)
        ok = !(x + patch > reference.width || y + patch > reference.height || x < radius || y < radius ||
               x + patch + radius > target.width || y + patch + radius > target.height || x + patch > target.width ||
               y + patch > target.height);
    const float n = (float)area;
    if (ok && lane == 0) {
        float sum = -0.0f;  // f32 Sum
        for (int k = 0; k < area; ++k) sum += plane_at(reference, x + k % patch, y + k / patch);
        const float mean = sum / n;
        float squares = -0.0f;
        for (int k = 0; k < area; ++k) {
            const float d = plane_at(reference, x + k % patch, y + k / patch) - mean;
            squares += d * d;
        }
        ref_std_s[w] = sqrtf(squares / n);
        for (int k = 0; k < area; ++k) ref_centered[k] = plane_at(reference, x + k % patch, y + k / patch) - mean;
    }
    __syncwarp();
    if (ok) ok = !(ref_std_s[w] < 1.0e-4f);
    if (ok) {
        const float ref_std = ref_std_s[w];
        for (int s = lane; s < span * span; s += 32) {
            const int dy = s / span, dx = s - dy * span;
            const int tx = x + dx - radius, ty = y + dy - radius;
            float sum = 0.0f, sum_sq = 0.0f, cross = 0.0f;
            for (int yy = 0; yy < patch; ++yy)
                for (int xx = 0; xx < patch; ++xx) {
                    const float t = plane_at(target, tx + xx, ty + yy);
                    sum += t;
                    sum_sq += t * t;
                    cross += t * ref_centered[yy * patch + xx];
                }
            const float mean = sum / n;
            float var = sum_sq / n - mean * mean;
            var = var != var ? 0.0f : fmaxf(var, 0.0f);  // f32::max(0.0) ignores NaN
            scores[s] = var < 1.0e-8f ? -INFINITY : (cross / n) / (sqrtf(var) * ref_std);
        }
        __syncwarp();
        if (lane == 0) {
            int best = 0;  // Iterator::max_by(total_cmp): the last maximum
            for (int s = 1; s < span * span; ++s)
                if (total_key(scores[s]) >= total_key(scores[best])) best = s;
            const float score = scores[best];
            if (isfinite(score)) {
                const int bx = best % span, by = best / span;
                const float sub_x =
                    bx > 0 && bx + 1 < span ? align_refine(scores[by * span + bx - 1], score, scores[by * span + bx + 1])
                                            : 0.0f;
                const float sub_y = by > 0 && by + 1 < span
                                        ? align_refine(scores[(by - 1) * span + bx], score, scores[(by + 1) * span + bx])
                                        : 0.0f;
                if (score >= min_score)
                    result = AlignMatch{(float)bx - (float)radius + sub_x, (float)by - (float)radius + sub_y, score, 1};
            }
        }
    }
    if (lane == 0) out[job] = result;
}

// counts[k] = pairs whose distance under candidate k is within threshold (align.rs:660-671).
__global__ void align_inlier_kernel(const double4 *__restrict__ pairs, int n_pairs, const Hom *__restrict__ candidates,
                                    double threshold, unsigned *__restrict__ counts) {
    const int k = blockIdx.y;
    const Hom h = candidates[k];
    unsigned count = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pairs; i += gridDim.x * blockDim.x) {
        const double4 p = pairs[i];
        double qx, qy;
        if (apply_homography(h, p.x, p.y, qx, qy)) {
            const double ex = qx - p.z, ey = qy - p.w;
            count += sqrt(ex * ex + ey * ey) <= threshold;
        }
    }
    count = __reduce_add_sync(0xffffffffu, count);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(counts + k, count);
}

}  // namespace chiaro
