// consumers.cuh — the depth stage's outputs as a GPU synthesis reads them: Warp::map and
// Warp::confidence (crates/chiaro-fusion/src/align.rs:84-131) and
// DenseDepthMap::sample_nearest (depth.rs:152-159), the per-pixel lookups of synthesize
// (synth.rs:591-700), over batches of query points in device memory so that warps and
// depth maps can stay resident for a device-side consumer.
#pragma once

#include "common.cuh"

namespace chiaro {

// Warp::confidence (align.rs:113-131); confidence NULL reads as a length mismatch (0).
CH_HD float warp_confidence_at(const WarpRef &w, const float *confidence, float x, float y) {
    const float fx = x / (float)w.step, fy = y / (float)w.step;
    if (fx < 0.0f || fy < 0.0f || !confidence) return 0.0f;
    const int c0 = sat_index(floorf(fx), w.columns - 1), r0 = sat_index(floorf(fy), w.rows - 1);
    const int c1 = c0 + 1 < w.columns - 1 ? c0 + 1 : w.columns - 1, r1 = r0 + 1 < w.rows - 1 ? r0 + 1 : w.rows - 1;
    const float tx = fx - (float)c0, ty = fy - (float)r0;
    const float v00 = confidence[(size_t)r0 * w.columns + c0], v10 = confidence[(size_t)r0 * w.columns + c1];
    const float v01 = confidence[(size_t)r1 * w.columns + c0], v11 = confidence[(size_t)r1 * w.columns + c1];
    const float top = v00 * (1.0f - tx) + v10 * tx;
    const float bottom = v01 * (1.0f - tx) + v11 * tx;
    float v = top * (1.0f - ty) + bottom * ty;  // f32::clamp(0, 1): NaN passes through
    if (v < 0.0f) v = 0.0f;
    if (v > 1.0f) v = 1.0f;
    return v;
}

__global__ void warp_sample_kernel(WarpRef warp, const float *__restrict__ confidence, const float2 *__restrict__ xy,
                                   long n, float2 *__restrict__ mapped, float *__restrict__ confidence_out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float2 p = xy[i];
        float qx, qy;
        mapped[i] = warp_map(warp, p.x, p.y, qx, qy) ? make_float2(qx, qy) : make_float2(NAN, NAN);
        if (confidence_out) confidence_out[i] = warp_confidence_at(warp, confidence, p.x, p.y);
    }
}

// DenseDepthMap::sample_nearest (depth.rs:152-159): the node index, or -1 for None.
CH_HD long sample_nearest_node(int columns, int rows, int step, float x, float y) {
    if (x < 0.0f || y < 0.0f || step == 0) return -1;
    const float fc = roundf(x / (float)step), fr = roundf(y / (float)step);  // round half away from zero
    // `as usize` saturates (NaN -> 0); then node() bounds-checks
    const double c = fc != fc ? 0.0 : (double)fc, r = fr != fr ? 0.0 : (double)fr;
    if (!(c < (double)columns) || !(r < (double)rows)) return -1;
    return (long)r * columns + (long)c;
}

__global__ void depth_sample_nearest_kernel(const double *__restrict__ depth, const float *__restrict__ confidence,
                                            const uint8_t *__restrict__ provenance, int columns, int rows, int step,
                                            const float2 *__restrict__ xy, long n, double *__restrict__ depth_out,
                                            float *__restrict__ confidence_out, uint8_t *__restrict__ provenance_out,
                                            long long *__restrict__ node_out) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long k = sample_nearest_node(columns, rows, step, xy[i].x, xy[i].y);
        if (node_out) node_out[i] = k;
        if (depth_out) depth_out[i] = k >= 0 ? depth[k] : NAN;
        if (confidence_out) confidence_out[i] = k >= 0 ? confidence[k] : 0.0f;
        if (provenance_out) provenance_out[i] = k >= 0 ? provenance[k] : 0;
    }
}

}  // namespace chiaro
