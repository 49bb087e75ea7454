// luminance.cuh — Mosaic::luminance_half (crates/chiaro-fusion/src/image.rs:401-428)
// with Mosaic::flat_field (image.rs:145-150) and VignettingMesh::gain
// (crates/chiaro-fusion/src/calibration.rs:362-379): the u16 Q6 mosaic becomes
// the half-resolution f32 log-luminance plane the depth stage reads.
//
// A thread per output pixel reads its 2x2 cell as four 2-byte loads (a row
// pair's second row starts at an odd sample when the width is odd, so wider
// loads would not be aligned); a warp's loads of one row cover 128 contiguous
// bytes. The sum, the black/white scaling and the
// flat-field gain are the reference's f32 arithmetic in its order (no FMA).
// The log is CUDA's f64 log rounded to f32: the correctly rounded logarithm in
// all but vanishingly rare cases, where the reference's host logf is within
// 0.82 ulp, so the two agree to 1 ulp and differ on about 0.1% of pixels.
#pragma once

#include "common.cuh"

namespace chiaro {

struct VignettingRef {
    const float *gains;  // [rows][columns], nullptr: no mesh (flat field 1)
    int columns, rows;
};

// VignettingMesh::gain at raster (x, y) of a width x height sensor.
__device__ __forceinline__ float vignetting_gain(const VignettingRef &m, float x, float y, int width, int height) {
    if (!m.gains || m.columns < 2 || m.rows < 2) return 1.0f;
    const float cmax = (float)(m.columns - 1), rmax = (float)(m.rows - 1);
    const float fx = clampf_r(x / (float)width * cmax, 0.0f, cmax);
    const float fy = clampf_r(y / (float)height * rmax, 0.0f, rmax);
    const int c0 = (int)floorf(fx), r0 = (int)floorf(fy);
    const int c1 = min(c0 + 1, m.columns - 1), r1 = min(r0 + 1, m.rows - 1);
    const float tx = fx - (float)c0, ty = fy - (float)r0;
    const float *g0 = m.gains + (size_t)r0 * m.columns, *g1 = m.gains + (size_t)r1 * m.columns;
    const float top = g0[c0] * (1.0f - tx) + g0[c1] * tx;
    const float bottom = g1[c0] * (1.0f - tx) + g1[c1] * tx;
    return top * (1.0f - ty) + bottom * ty;
}

// The argument of the log, 1 + 1000 * linear, for output pixel (i, j).
__device__ __forceinline__ float luminance_argument(const uint16_t *__restrict__ samples, int width, int height,
                                                    float black_q6, float range, const VignettingRef &mesh, int i,
                                                    int j) {
    const uint16_t *row0 = samples + (size_t)(2 * j) * width + 2 * i;
    const uint16_t *row1 = row0 + width;
    const float sum = (float)__ldg(row0) + (float)__ldg(row0 + 1) + (float)__ldg(row1) + (float)__ldg(row1 + 1);
    const float flat = vignetting_gain(mesh, 2.0f * (float)i + 0.5f, 2.0f * (float)j + 0.5f, width, height);
    const float linear = fmaxf((sum * 0.25f - black_q6) / range, 0.0f) * flat;
    return 1.0f + 1000.0f * linear;
}

__global__ void __launch_bounds__(256) luminance_half_kernel(const uint16_t *__restrict__ samples, int width,
                                                             int height, float black_q6, float white_q6,
                                                             VignettingRef mesh, float *__restrict__ out) {
    const int w = width / 2, h = height / 2;
    const long n = (long)w * h;
    const float range = fmaxf(white_q6 - black_q6, 1.0f);
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int j = (int)(k / w), i = (int)(k - (long)j * w);
        const float x = luminance_argument(samples, width, height, black_q6, range, mesh, i, j);
        out[k] = (float)log((double)x);
    }
}

}  // namespace chiaro
