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

// aggregate as the reference writes it (depth.rs:1761-1770): compaction, stable
// insertion sort descending by f32::total_cmp, the sum of the best from -0.0.
static bool aggregate_reference(const float *in, int n, int minimum_support, int best_view_count, float &out) {
    float s[8];
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (!(in[i] != in[i])) s[m++] = in[i];
    if (m < minimum_support) return false;
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

// Mismatches of aggregate_small<4> (n <= 4) and <8> (n <= 8) against the reference form
// over `trials` random score sets per n, drawn from a small pool (None, +-0, +-1,
// repeated and random values) so that ties and Nones are frequent.
uint64_t chiaro_hc_aggregate_mismatches(uint64_t trials, uint64_t seed) {
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1, bad = 0;
    auto next = [&x]() { x ^= x << 13; x ^= x >> 7; x ^= x << 17; return x; };
    const float pool[8] = {NAN, 0.0f, -0.0f, 1.0f, -1.0f, 0.5f, 0.25f, -0.125f};
    for (uint64_t t = 0; t < trials; ++t)
        for (int n = 1; n <= 8; ++n) {
            float in[8];
            for (int i = 0; i < 8; ++i) {
                const uint64_t r = next();
                in[i] = (r & 3) ? pool[(r >> 2) & 7] : (float)(int)((r >> 8) % 2001 - 1000) / 1000.0f;
            }
            const int support = 1 + (int)(next() % 3), best = support + (int)(next() % 4);
            float a = 0.0f, b = 0.0f;
            const bool ra = aggregate_reference(in, n, support, best, a);
            const bool rb = aggregate_small<8>(in, 1, n, support, best, b);
            bad += ra != rb || (ra && f2u(a) != f2u(b));
            if (n <= 4) {
                float c = 0.0f;
                const bool rc = aggregate_small<4>(in, 1, n, support, best, c);
                bad += ra != rc || (ra && f2u(a) != f2u(c));
            }
        }
    return bad;
}

// Mismatches of SmallDiv against integer division: every n < 2^16 for d <= 1024, and
// for 1024 < d < 2^16 both ends (q d and q d + d - 1) of every quotient step below 2^16,
// where the multiply's error term is largest.
uint64_t chiaro_hc_smalldiv_mismatches(void) {
    uint64_t bad = 0;
    for (int d = 1; d <= 1024; ++d) {
        const SmallDiv sd(d);
        for (int n = 0; n < 65536; ++n) bad += sd.quotient(n) != n / d;
    }
    for (int d = 1025; d < 65536; ++d) {
        const SmallDiv sd(d);
        for (int base = 0; base < 65536; base += d) {
            const int hi = base + d - 1 < 65535 ? base + d - 1 : 65535;
            bad += sd.quotient(base) != base / d;
            bad += sd.quotient(hi) != hi / d;
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
