// hostcheck.cpp — host build of the device math in common.cuh.
//
// Compiled by g++ with -ffp-contract=off, this exposes the exact-arithmetic
// building blocks of the kernels (exp restatements, bilinear fetch, warp
// lookup, camera model) to CPU tests, so they can be checked against the
// platform libm and the oracle without a GPU. It also carries range checkers
// that compare the exp restatements with libm over every float in a range.
#include <vector_types.h>
#include <vector_functions.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "common.cuh"

using namespace chiaro;

extern "C" {

float chiaro_hc_exp_f32(float x) { return exp_f32(x); }
double chiaro_hc_exp_f64(double x) { return exp_f64(x); }

// Mismatches of exp_f32 against libm expf over float bit patterns [lo, hi)
// (sign bit given separately). first_bad receives the first mismatching pattern.
uint64_t chiaro_hc_expf_mismatches(uint32_t lo, uint32_t hi, int negative, uint32_t *first_bad) {
    uint64_t bad = 0;
    for (uint32_t u = lo; u < hi; ++u) {
        uint32_t bits = u | (negative ? 0x80000000u : 0u);
        float x;
        memcpy(&x, &bits, 4);
        float a = std::exp(x), b = exp_f32(x);
        if (f2u(a) != f2u(b) && !(a != a && b != b)) {
            if (!bad && first_bad) *first_bad = bits;
            ++bad;
        }
    }
    return bad;
}

// Mismatches of exp_f64(scale * (double)f) against libm exp for every f32 f
// with bit pattern in [lo, hi).
uint64_t chiaro_hc_exp_mismatches(uint32_t lo, uint32_t hi, double scale, uint32_t *first_bad) {
    uint64_t bad = 0;
    for (uint32_t u = lo; u < hi; ++u) {
        float f;
        memcpy(&f, &u, 4);
        double x = scale * (double)f;
        double a = std::exp(x), b = exp_f64(x);
        if (d2u(a) != d2u(b) && !(a != a && b != b)) {
            if (!bad && first_bad) *first_bad = u;
            ++bad;
        }
    }
    return bad;
}

// Mismatches of floor_frac_small against floorf over float bit patterns [lo, hi).
uint64_t chiaro_hc_floor_mismatches(uint32_t lo, uint32_t hi) {
    uint64_t bad = 0;
    for (uint32_t u = lo; u < hi; ++u) {
        float x;
        memcpy(&x, &u, 4);
        int i;
        float frac = floor_frac_small(x, i);
        float f = std::floor(x);
        if ((float)i != f || f2u(frac) != f2u(x - f)) ++bad;
    }
    return bad;
}

float chiaro_hc_plane_sample(const float *data, int width, int height, float x, float y, int *ok) {
    PlaneRef p{data, width, height};
    float v = 0.0f;
    *ok = plane_sample(p, x, y, v) ? 1 : 0;
    return v;
}

int chiaro_hc_warp_map(const float *points, int step, int columns, int rows, float x, float y, float *out) {
    WarpRef w{reinterpret_cast<const float2 *>(points), step, columns, rows};
    return warp_map(w, x, y, out[0], out[1]) ? 1 : 0;
}

int chiaro_hc_map_from(const chiaro_camera *target, const chiaro_camera *reference, const double *pixel,
                       double depth, double *out) {
    DevCamera t, r;
    camera_from_abi(*target, t);
    camera_from_abi(*reference, r);
    D3 o, d;
    pixel_to_ray(r, pixel[0], pixel[1], o, d);
    return project(t, along(o, d, depth), out[0], out[1]) ? 1 : 0;
}

}  // extern "C"
