// align_run.cuh — the host half of align_module_seeded (crates/chiaro-fusion/src/align.rs:281-830),
// included by stage.cu after its buffer and transfer helpers. The per-pixel and
// per-patch work runs in the kernels of align.cuh; this file holds the pyramids'
// shapes, the initial mapping, the RANSAC samples and fits (their inlier counts on
// the device), the final warp, the report and the photometric gain, each step in
// the reference's order so that the result is bit-identical to it.
#pragma once

namespace align_host {

struct HostPlane {
    int width = 0, height = 0;
    std::vector<float> data;
    PlaneRef ref() const { return PlaneRef{data.data(), width, height}; }
    float at(int x, int y) const { return data[(size_t)y * width + x]; }
};

struct Shape {
    int width, height;
};

// Plane::pyramid's level shapes (image.rs:487-497)
std::vector<Shape> pyramid_shapes(int width, int height, int min_size) {
    std::vector<Shape> levels{{width, height}};
    while (std::min(levels.back().width, levels.back().height) / 2 >= std::max(min_size, 8))
        levels.push_back({std::max(levels.back().width / 2, 1), std::max(levels.back().height / 2, 1)});
    return levels;
}

// Plane::downsample (image.rs:469-483) on the host, for the small no-calibration search
HostPlane downsample(const HostPlane &in) {
    HostPlane out;
    out.width = std::max(in.width / 2, 1);
    out.height = std::max(in.height / 2, 1);
    out.data.resize((size_t)out.width * out.height);
    for (int j = 0; j < out.height; ++j)
        for (int i = 0; i < out.width; ++i) {
            const int x = 2 * i, y = 2 * j, x1 = std::min(x + 1, in.width - 1), y1 = std::min(y + 1, in.height - 1);
            out.data[(size_t)j * out.width + i] = 0.25f * (in.at(x, y) + in.at(x1, y) + in.at(x, y1) + in.at(x1, y1));
        }
    return out;
}

std::vector<HostPlane> host_pyramid(const HostPlane &base, int min_size) {
    std::vector<HostPlane> levels{base};
    while (std::min(levels.back().width, levels.back().height) / 2 >= std::max(min_size, 8))
        levels.push_back(downsample(levels.back()));
    return levels;
}

struct Match {
    float shift_x, shift_y, score;
};

// match_patch (image.rs:531-640) on the host, for the small no-calibration search
bool match_patch(const HostPlane &reference, const HostPlane &target, int rx, int ry, int size, int radius, Match &m) {
    if (rx + size > reference.width || ry + size > reference.height || rx < radius || ry < radius ||
        rx + size + radius > target.width || ry + size + radius > target.height || rx + size > target.width ||
        ry + size > target.height)
        return false;
    const float n = (float)(size * size);
    float total = -0.0f;  // f32 Sum
    for (int y = ry; y < ry + size; ++y)
        for (int x = rx; x < rx + size; ++x) total += reference.at(x, y);
    const float mean = total / n;
    float squares = -0.0f;
    std::vector<float> centred;
    for (int y = ry; y < ry + size; ++y)
        for (int x = rx; x < rx + size; ++x) {
            const float d = reference.at(x, y) - mean;
            squares += d * d;
            centred.push_back(d);
        }
    const float ref_std = std::sqrt(squares / n);
    if (ref_std < 1e-4f) return false;
    const int span = 2 * radius + 1;
    std::vector<float> scores((size_t)span * span, -INFINITY);
    for (int dy = 0; dy < span; ++dy)
        for (int dx = 0; dx < span; ++dx) {
            const int tx = rx + dx - radius, ty = ry + dy - radius;
            float sum = 0.0f, sum_sq = 0.0f, cross = 0.0f;
            for (int y = 0; y < size; ++y)
                for (int x = 0; x < size; ++x) {
                    const float v = target.at(tx + x, ty + y);
                    sum += v;
                    sum_sq += v * v;
                    cross += v * centred[(size_t)y * size + x];
                }
            const float mv = sum / n;
            const float var = std::fmax(sum_sq / n - mv * mv, 0.0f);  // f32::max ignores NaN
            if (var < 1e-8f) continue;
            scores[(size_t)dy * span + dx] = (cross / n) / (std::sqrt(var) * ref_std);
        }
    size_t best = 0;  // the last maximum in total order
    for (size_t k = 1; k < scores.size(); ++k)
        if (total_key(scores[k]) >= total_key(scores[best])) best = k;
    const float score = scores[best];
    if (!std::isfinite(score)) return false;
    const int bx = (int)best % span, by = (int)best / span;
    auto refine = [](float minus, float center, float plus) {
        const float denominator = minus - 2.0f * center + plus;
        if (std::fabs(denominator) < 1e-9f) return 0.0f;
        return resolution_host::clamp_rust(0.5f * (minus - plus) / denominator, -0.5f, 0.5f);
    };
    const float sub_x =
        bx > 0 && bx + 1 < span ? refine(scores[by * span + bx - 1], score, scores[by * span + bx + 1]) : 0.0f;
    const float sub_y =
        by > 0 && by + 1 < span ? refine(scores[(by - 1) * span + bx], score, scores[(by + 1) * span + bx]) : 0.0f;
    m = Match{(float)bx - (float)radius + sub_x, (float)by - (float)radius + sub_y, score};
    return true;
}

double residual(const Hom &h, const double4 &p, bool &some) {
    double qx = 0.0, qy = 0.0;
    some = apply_homography(h, p.x, p.y, qx, qy);
    if (!some) return 0.0;
    return std::sqrt((qx - p.z) * (qx - p.z) + (qy - p.w) * (qy - p.w));
}

struct Fit {
    Hom h;
    size_t inliers = 0;
    std::vector<float> residuals;
};

// fit_homography_ransac (align.rs:631-700): the 300 four-pair samples from the LCG on the
// host (the sequence does not depend on the fits), their fits and inlier counts on the
// device, the refit on the best candidate's inliers and the residuals on the host.
bool fit_ransac(chiaro_depth_ctx *ctx, const std::vector<double4> &pairs, const std::vector<float> &scores,
                float threshold, Fit &fit) {
    if (pairs.size() < 6) return false;
    constexpr int ITERATIONS = 300;
    uint64_t state = 0x9E3779B97F4A7C15ull ^ (uint64_t)pairs.size();
    auto next = [&](size_t n) {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return (size_t)(state >> 33) % n;
    };
    std::vector<int4> samples(ITERATIONS);
    for (int it = 0; it < ITERATIONS; ++it) {
        int sample[4] = {0, 0, 0, 0};
        for (int slot = 0; slot < 4; ++slot)
            for (;;) {
                const int candidate = (int)next(pairs.size());
                bool taken = false;
                for (int k = 0; k < slot; ++k) taken = taken || sample[k] == candidate;
                if (!taken) {
                    sample[slot] = candidate;
                    break;
                }
            }
        samples[it] = make_int4(sample[0], sample[1], sample[2], sample[3]);
    }
    cudaStream_t s = ctx->stream;
    double4 *d_pairs = dbuf<double4>(ctx, "al.pairs", pairs.size());
    float *d_scores = dbuf<float>(ctx, "al.scores", pairs.size());
    int4 *d_samples = dbuf<int4>(ctx, "al.samples", ITERATIONS);
    Hom *d_candidates = dbuf<Hom>(ctx, "al.candidates", ITERATIONS);
    int *d_valid = dbuf<int>(ctx, "al.valid", ITERATIONS);
    unsigned *d_counts = dbuf<unsigned>(ctx, "al.counts", ITERATIONS);
    upload(ctx, d_pairs, pairs.data(), pairs.size());
    upload(ctx, d_scores, scores.data(), scores.size());
    upload(ctx, d_samples, samples.data(), ITERATIONS);
    align_fit_kernel<<<(ITERATIONS + 63) / 64, 64, 0, s>>>(d_pairs, d_scores, d_samples, ITERATIONS, d_candidates,
                                                           d_valid);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(d_counts, 0, ITERATIONS * sizeof(unsigned), s));
    const unsigned blocks = (unsigned)std::min<size_t>(div_ceil(pairs.size(), 256), 64);
    align_inlier_kernel<<<dim3(blocks, ITERATIONS), 256, 0, s>>>(d_pairs, (int)pairs.size(), d_candidates,
                                                                  (double)threshold, d_counts);
    CK(cudaGetLastError());
    std::vector<unsigned> counts(ITERATIONS);
    std::vector<int> valid(ITERATIONS);
    std::vector<Hom> candidates(ITERATIONS);
    CK(cudaMemcpyAsync(counts.data(), d_counts, ITERATIONS * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(valid.data(), d_valid, ITERATIONS * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(candidates.data(), d_candidates, ITERATIONS * sizeof(Hom), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    int best = -1;
    unsigned best_count = 0;  // the first candidate with the most inliers
    for (int it = 0; it < ITERATIONS; ++it)
        if (valid[it] && counts[it] > best_count) {
            best = it;
            best_count = counts[it];
        }
    if (best < 0 || best_count < 6) return false;
    std::vector<int> inliers;
    for (size_t i = 0; i < pairs.size(); ++i) {
        bool some;
        const double r = residual(candidates[best], pairs[i], some);
        if (some && r <= (double)threshold) inliers.push_back((int)i);
    }
    if (!fit_homography(pairs.data(), scores.data(), inliers.data(), (int)inliers.size(), fit.h)) return false;
    fit.inliers = 0;
    fit.residuals.clear();
    for (const double4 &p : pairs) {
        bool some;
        const float r = (float)residual(fit.h, p, some);
        if (some && r <= threshold) {
            ++fit.inliers;
            fit.residuals.push_back(r);
        }
    }
    if (fit.inliers < 6) return false;
    std::sort(fit.residuals.begin(), fit.residuals.end(), resolution_host::total_less);
    return true;
}

// photometric_gain (align.rs:795-826)
bool photometric_gain(const PlaneRef &reference, const PlaneRef &target, const WarpRef &warp, float &gain) {
    std::vector<float> ratios;
    const int step = 16;
    for (int y = step; y + step < reference.height; y += step)
        for (int x = step; x + step < reference.width; x += step) {
            float qx, qy, t;
            if (!warp_map(warp, (float)x * 2.0f + 0.5f, (float)y * 2.0f + 0.5f, qx, qy)) continue;
            if (!plane_sample(target, (qx - 0.5f) / 2.0f, (qy - 0.5f) / 2.0f, t)) continue;
            const float r = reference.data[(size_t)y * reference.width + x];
            const float lr = (std::exp(r) - 1.0f) / 1000.0f, lt = (std::exp(t) - 1.0f) / 1000.0f;
            if (lr > 0.01f && lt > 0.01f && lr < 0.95f && lt < 0.95f) ratios.push_back(lr / lt);
        }
    if (ratios.size() < 16) return false;
    std::sort(ratios.begin(), ratios.end(), resolution_host::total_less);
    gain = resolution_host::clamp_rust(ratios[ratios.size() / 2], 0.25f, 4.0f);
    return true;
}

size_t sat_size(double v) {  // `as usize`: saturating, NaN -> 0
    if (!(v > 0.0)) return 0;
    if (v >= 1.8446744073709552e19) return SIZE_MAX;
    return (size_t)v;
}

// coarse_global_shift (align.rs:561-628) on the host (planes of tens of pixels); false with a message for Err
bool coarse_global_shift(const HostPlane &reference_luma, const HostPlane &target_luma, double scale, float min_score,
                         double shift[2], std::string &error) {
    const auto reference_pyramid = host_pyramid(reference_luma, 32);
    const HostPlane &reference_plane = reference_pyramid.back();
    const double reference_scale = (double)((size_t)1 << (reference_pyramid.size() - 1));
    const auto target_pyramid = host_pyramid(target_luma, 16);
    const double wanted = reference_scale * scale;
    const size_t target_level =
        std::min(sat_size(std::fmax(std::round(std::log2(wanted)), 0.0)), target_pyramid.size() - 1);
    const HostPlane &target_plane = target_pyramid[target_level];
    const double target_scale = (double)((size_t)1 << target_level);
    const float ratio = (float)(target_scale / wanted);
    const int rw = (int)sat_size(std::fmax(std::floor((float)target_plane.width * ratio), 4.0f));
    const int rh = (int)sat_size(std::fmax(std::floor((float)target_plane.height * ratio), 4.0f));
    HostPlane resampled;
    resampled.width = rw;
    resampled.height = rh;
    resampled.data.resize((size_t)rw * rh);
    const PlaneRef tp = target_plane.ref();
    for (int y = 0; y < rh; ++y)
        for (int x = 0; x < rw; ++x) {
            float v;
            resampled.data[(size_t)y * rw + x] = plane_sample(tp, (float)x / ratio, (float)y / ratio, v) ? v : 0.0f;
        }
    if (rw + 2 > reference_plane.width || rh + 2 > reference_plane.height) {
        shift[0] = shift[1] = 0.0;  // wider than the reference at this density: centred
        return true;
    }
    const int patch = std::min({rw, rh, reference_plane.width / 2, reference_plane.height / 2});
    const int radius = std::max((std::min(reference_plane.width, reference_plane.height) - patch) / 2, 1);
    const int rx = (reference_plane.width - patch) / 2, ry = (reference_plane.height - patch) / 2;
    const int tx = (rw - patch) / 2, ty = (rh - patch) / 2;
    HostPlane embedded;
    embedded.width = reference_plane.width;
    embedded.height = reference_plane.height;
    embedded.data.assign((size_t)embedded.width * embedded.height, NAN);
    for (int y = 0; y < patch; ++y)
        for (int x = 0; x < patch; ++x)
            embedded.data[(size_t)(ry + y) * embedded.width + rx + x] = resampled.at(tx + x, ty + y);
    Match found;
    if (!match_patch(reference_plane, embedded, rx, ry, patch, std::min({radius, rx, ry}), found)) {
        error = "no correlation between the module and the reference";
        return false;
    }
    if (found.score < min_score * 0.6f) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "module does not correlate with the reference (%.2f)", found.score);
        error = buf;
        return false;
    }
    shift[0] = -(double)found.shift_x * reference_scale * 2.0 * scale;
    shift[1] = -(double)found.shift_y * reference_scale * 2.0 * scale;
    return true;
}

struct Failure {  // the reference's Err
    std::string message;
};

}  // namespace align_host

int run_align(chiaro_depth_ctx *ctx, const chiaro_align_input &reference, const chiaro_align_input &target,
              bool target_is_reference, const chiaro_align_options &o, const chiaro_warp *seed, chiaro_warp &out,
              float &gain, chiaro_alignment_report &report) {
    using namespace align_host;
    constexpr double FAR_DEPTH = 1.0e8;
    cudaStream_t s = ctx->stream;
    set_smem_limits();  // align_match_kernel's windows may exceed 48 KiB per CTA
    const int width = (int)reference.width, height = (int)reference.height;
    std::memset(&report, 0, sizeof(report));
    const int step = (int)o.grid_step;
    const int columns = (width + step - 1) / step + 1, rows = (height + step - 1) / step + 1;
    out.step = (uint64_t)step;
    out.columns = (uint64_t)columns;
    out.rows = (uint64_t)rows;
    if (out.capacity < (uint64_t)columns * rows) return CHIARO_ERR_CAPACITY;
    auto emit = [&](auto map) {  // Warp::from_fn (align.rs:50-80) into out
        for (int row = 0; row < rows; ++row)
            for (int column = 0; column < columns; ++column) {
                const size_t k = (size_t)row * columns + column;
                double qx = 0.0, qy = 0.0;
                const bool some = map((double)(column * step), (double)(row * step), qx, qy);
                out.points[2 * k] = some ? (float)qx : NAN;
                out.points[2 * k + 1] = some ? (float)qy : NAN;
                if (out.confidence) out.confidence[k] = some ? 1.0f : 0.0f;
            }
    };
    if (target_is_reference) {  // align.rs:290-306
        emit([](double px, double py, double &qx, double &qy) {
            qx = px;
            qy = py;
            return true;
        });
        report.initialised_from = CHIARO_INIT_REFERENCE;
        report.coverage = 1.0f;
        report.inlier_ratio = 1.0f;
        report.accepted = 1;
        report.status = CHIARO_ALIGN_REFERENCE;
        gain = 1.0f;
        return CHIARO_OK;
    }
    const PlaneRef reference_plane{reference.luminance, (int)reference.luma_width, (int)reference.luma_height};
    const PlaneRef target_plane{target.luminance, (int)target.luma_width, (int)target.luma_height};
    // Step 1: the initial mapping on an 8 px grid (align.rs:311-345)
    std::vector<float2> initial_points;
    int init_step = 8, init_columns = (width + 7) / 8 + 1, init_rows = (height + 7) / 8 + 1;
    if (seed) {
        report.initialised_from = CHIARO_INIT_SEED;
        init_step = (int)seed->step;
        init_columns = (int)seed->columns;
        init_rows = (int)seed->rows;
        const float2 *sp = reinterpret_cast<const float2 *>(seed->points);
        initial_points.assign(sp, sp + (size_t)init_columns * init_rows);
    } else if (reference.has_camera && target.has_camera) {
        report.initialised_from = CHIARO_INIT_CALIBRATION;
        DevCamera rc, tc;
        camera_from_abi(reference.camera, rc);
        camera_from_abi(target.camera, tc);
        const size_t nodes = (size_t)init_columns * init_rows;
        float2 *d_grid = dbuf<float2>(ctx, "al.initial", nodes);
        align_initial_grid_kernel<<<(unsigned)div_ceil(nodes, 256), 256, 0, s>>>(rc, tc, init_columns, init_rows, 8,
                                                                                 FAR_DEPTH, d_grid);
        CK(cudaGetLastError());
        initial_points.resize(nodes);
        CK(cudaMemcpyAsync(initial_points.data(), d_grid, nodes * sizeof(float2), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    } else {
        report.initialised_from = CHIARO_INIT_NOMINAL_FOCAL_GROUP;
        const double scale = target.nominal_focal_px / reference.nominal_focal_px;
        const double cx = ((double)width - 1.0) / 2.0, cy = ((double)height - 1.0) / 2.0;
        const double tx = ((double)target.width - 1.0) / 2.0, ty = ((double)target.height - 1.0) / 2.0;
        HostPlane rl, tl;
        rl.width = reference_plane.width;
        rl.height = reference_plane.height;
        rl.data.assign(reference.luminance, reference.luminance + (size_t)rl.width * rl.height);
        tl.width = target_plane.width;
        tl.height = target_plane.height;
        tl.data.assign(target.luminance, target.luminance + (size_t)tl.width * tl.height);
        double shift[2];
        std::string error;
        if (!coarse_global_shift(rl, tl, scale, o.min_score, shift, error)) throw Failure{error};
        initial_points.resize((size_t)init_columns * init_rows);
        for (int row = 0; row < init_rows; ++row)
            for (int column = 0; column < init_columns; ++column) {
                const double px = (double)(column * 8), py = (double)(row * 8);
                initial_points[(size_t)row * init_columns + column] = make_float2(
                    (float)((px - cx) * scale + tx + shift[0]), (float)((py - cy) * scale + ty + shift[1]));
            }
    }
    const WarpRef initial_host{initial_points.data(), init_step, init_columns, init_rows};
    auto initial = [&](double px, double py, double &qx, double &qy) {
        float fx, fy;
        if (!warp_map(initial_host, (float)px, (float)py, fx, fy)) return false;
        qx = (double)fx;
        qy = (double)fy;
        return true;
    };
    // Step 2: coarse-to-fine refinement of the reference-space homography (align.rs:347-455)
    Hom correction = hom_identity();
    std::vector<float> finest_residuals;
    if (o.refine) {
        const auto reference_shapes = pyramid_shapes(reference_plane.width, reference_plane.height, 96);
        const auto target_shapes = pyramid_shapes(target_plane.width, target_plane.height, 48);
        if (reference_shapes.size() > CHIARO_ALIGN_MAX_LEVELS) return CHIARO_ERR_ARGUMENT;
        std::vector<float *> reference_levels, target_levels;
        auto build_pyramid = [&](const PlaneRef &base, const std::vector<Shape> &shapes, const std::string &name,
                                 std::vector<float *> &levels) {
            for (size_t l = 0; l < shapes.size(); ++l) {
                const size_t n = (size_t)shapes[l].width * shapes[l].height;
                float *d = dbuf<float>(ctx, name + std::to_string(l), std::max<size_t>(n, 1));
                if (l == 0) {
                    upload(ctx, d, base.data, n);
                } else {
                    align_downsample_kernel<<<(unsigned)std::min<size_t>(div_ceil(n, 256), (size_t)ctx->sm_count * 16),
                                              256, 0, s>>>(levels[l - 1], shapes[l - 1].width, shapes[l - 1].height, d,
                                                           shapes[l].width, shapes[l].height);
                    CK(cudaGetLastError());
                }
                levels.push_back(d);
            }
        };
        build_pyramid(reference_plane, reference_shapes, "al.ref", reference_levels);
        build_pyramid(target_plane, target_shapes, "al.tgt", target_levels);
        float2 *d_initial = dbuf<float2>(ctx, "al.initial", initial_points.size());
        upload(ctx, d_initial, initial_points.data(), initial_points.size());
        const WarpRef initial_device{d_initial, init_step, init_columns, init_rows};
        double magnification;
        {
            const double c0 = (double)width / 2.0, c1 = (double)height / 2.0, h = 64.0;
            double ax, ay, bx, by, dx_, dy_;
            if (initial(c0, c1, ax, ay) && initial(c0 + h, c1, bx, by) && initial(c0, c1 + h, dx_, dy_)) {
                const double dx = std::sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay)) / h;
                const double dy = std::sqrt((dx_ - ax) * (dx_ - ax) + (dy_ - ay) * (dy_ - ay)) / h;
                magnification = std::sqrt(dx * dy);
            } else {
                magnification = target.nominal_focal_px / reference.nominal_focal_px;
            }
        }
        for (int level = (int)reference_shapes.size() - 1; level >= 0; --level) {
            const int scale = 1 << level;
            const Shape rs = reference_shapes[level];
            const size_t target_level = std::min(
                sat_size(std::fmax(std::round(std::log2((double)scale * magnification)), 0.0)), target_shapes.size() - 1);
            const Shape ts = target_shapes[target_level];
            const double target_scale = (double)((size_t)1 << target_level);
            const size_t plane = (size_t)rs.width * rs.height;
            float *rendered = dbuf<float>(ctx, "al.rendered", std::max<size_t>(plane, 1));
            if (plane) {
                align_render_kernel<<<(unsigned)std::min<size_t>(div_ceil(plane, 256), (size_t)ctx->sm_count * 16),
                                      256, 0, s>>>(rs.width, rs.height, scale,
                                                   PlaneRef{target_levels[target_level], ts.width, ts.height},
                                                   target_scale, initial_device, correction, rendered);
                CK(cudaGetLastError());
            }
            const int radius = level + 1 == (int)reference_shapes.size() ? (int)o.coarse_radius : 3;
            const int patch = std::max(std::min((int)o.patch, rs.width / 4), 8);
            const int stride = patch / 2;
            const int nx = rs.width >= patch + 2 * radius ? (rs.width - patch - 2 * radius) / stride + 1 : 0;
            const int ny = rs.height >= patch + 2 * radius ? (rs.height - patch - 2 * radius) / stride + 1 : 0;
            std::vector<double4> pairs;
            std::vector<float> pair_scores;
            if (nx > 0 && ny > 0) {
                const int span = 2 * radius + 1;
                const size_t per_warp = ((size_t)patch * patch + (size_t)span * span) * sizeof(float);
                if (per_warp > 200 * 1024) return CHIARO_ERR_ARGUMENT;  // the kernel's opted-in maximum
                const int warps = (int)std::min<size_t>(8, 200 * 1024 / per_warp);
                const size_t jobs = (size_t)nx * ny;
                AlignMatch *d_matches = dbuf<AlignMatch>(ctx, "al.matches", jobs);
                align_match_kernel<<<(unsigned)div_ceil(jobs, (size_t)warps), 32 * warps, warps * per_warp, s>>>(
                    PlaneRef{reference_levels[level], rs.width, rs.height}, PlaneRef{rendered, rs.width, rs.height},
                    patch, radius, radius, radius, stride, nx, ny, 1, o.min_score, d_matches);
                CK(cudaGetLastError());
                std::vector<AlignMatch> matches(jobs);
                CK(cudaMemcpyAsync(matches.data(), d_matches, jobs * sizeof(AlignMatch), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                const float half = (float)patch / 2.0f;
                auto convert = [&](float v) { return (double)v * (double)scale * 2.0 + (double)scale - 0.5; };
                for (size_t j = 0; j < jobs; ++j) {  // the reference's scan order: rows, then columns
                    if (!matches[j].found) continue;
                    const int x = radius + (int)(j % nx) * stride, y = radius + (int)(j / nx) * stride;
                    pairs.push_back(make_double4(convert((float)x + half), convert((float)y + half),
                                                 convert((float)x + half + matches[j].shift_x),
                                                 convert((float)y + half + matches[j].shift_y)));
                    pair_scores.push_back(matches[j].score);
                }
            }
            const float threshold = std::fmax(o.inlier_px * (float)scale * 2.0f, o.inlier_px);
            chiaro_align_level &lr = report.levels[report.n_levels++];
            Fit fit;
            if (fit_ransac(ctx, pairs, pair_scores, threshold, fit)) {
                correction = hom_mul(correction, fit.h);
                lr = chiaro_align_level{(uint64_t)scale * 2, pairs.size(), fit.inliers,
                                        fit.residuals[fit.residuals.size() / 2]};
                if (level == 0) {
                    finest_residuals = fit.residuals;
                    report.patches = pairs.size();
                    report.inliers = fit.inliers;
                }
            } else {
                lr = chiaro_align_level{(uint64_t)scale * 2, pairs.size(), 0, NAN};
            }
        }
    }
    // Final warp and report (align.rs:457-519)
    emit([&](double px, double py, double &qx, double &qy) {
        double cx, cy;
        return apply_homography(correction, px, py, cx, cy) && initial(cx, cy, qx, qy);
    });
    size_t covered = 0;
    for (size_t k = 0; k < (size_t)columns * rows; ++k) {
        const float qx = out.points[2 * k], qy = out.points[2 * k + 1];
        covered += std::isfinite(qx) && qx >= 0.0f && qy >= 0.0f && qx <= (float)(target.width - 1) &&
                   qy <= (float)(target.height - 1);
    }
    report.coverage = (float)covered / (float)((size_t)columns * rows);
    if (!finest_residuals.empty()) {
        report.residual_median_px = finest_residuals[finest_residuals.size() / 2];
        report.residual_p90_px =
            finest_residuals[std::min(finest_residuals.size() * 9 / 10, finest_residuals.size() - 1)];
    }
    {
        const double c0 = (double)(width / 2), c1 = (double)(height / 2);
        double mx = c0, my = c1;
        if (!apply_homography(correction, c0, c1, mx, my)) {
            mx = c0;
            my = c1;
        }
        report.correction_median_px[0] = (float)(mx - c0);
        report.correction_median_px[1] = (float)(my - c1);
    }
    report.inlier_ratio = report.patches == 0 ? 0.0f : (float)report.inliers / (float)report.patches;
    report.accepted = !o.refine || report.inlier_ratio >= o.min_inlier_ratio;
    report.status = !report.accepted ? CHIARO_ALIGN_REJECTED
                    : !o.refine      ? CHIARO_ALIGN_FACTORY_MODEL
                    : report.inliers >= 12 && report.residual_median_px < o.inlier_px ? CHIARO_ALIGN_REFINED
                    : report.inliers > 0 ? CHIARO_ALIGN_WEAK_REFINEMENT
                                         : CHIARO_ALIGN_NO_SUPPORT;
    const WarpRef final_warp{reinterpret_cast<const float2 *>(out.points), step, columns, rows};
    if (!photometric_gain(reference_plane, target_plane, final_warp, gain)) gain = 1.0f;
    return CHIARO_OK;
}
