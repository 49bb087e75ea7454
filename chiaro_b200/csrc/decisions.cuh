// decisions.cuh — the per-target cross-camera consistency check
// (crates/chiaro-fusion/src/depth.rs:420-547): refine_one_view (1634-1708),
// score_one_view_at_point (1710-1736), the Refined / Occluded / Global
// classification (458-485), enforce_warp_consensus (582-618),
// suppress_warp_boundaries (620-672) and the output warp (490-532).
//
// One CTA (one warp) per fine node and target. Lanes 0-4 score the five
// inverse-depth offsets and lane 5 the global baseline; after the first
// lane picks the best offset, lanes 0-7 score the eight residual shifts.
#pragma once

#include "cost.cuh"
#include "select.cuh"

namespace chiaro {

struct Decisions {  // NodeWarp (depth.rs:256-271) as arrays
    uint8_t *kind;
    float2 *global;
    float2 *point;
    float *confidence;
    uint8_t *measured;
};

struct DecisionParams {
    const DevView *views;
    int reference;
    int target;  // module index of the target
    int columns, rows, step;
    Field field;
    double inverse_step, near_depth, far_depth;
    int radius;
    const float *spatial;
    float minimum_score;
    Decisions out;
};

__global__ void __launch_bounds__(32) target_decision_kernel(DecisionParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patch;
    __shared__ float sc[16];
    __shared__ float2 pts[16];
    __shared__ int fail;
    const int node = blockIdx.x;
    const int column = node % p.columns, row = node / p.columns;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const double cx = (double)(column * p.step), cy = (double)(row * p.step);
    const DevView &tv = p.views[p.target];
    Decisions o = p.out;

    float gqx, gqy;
    if (!warp_map(tv.warp, (float)cx, (float)cy, gqx, gqy)) {
        if (threadIdx.x == 0) {
            o.kind[node] = CHIARO_NW_UNDEFINED;
            o.global[node] = make_float2(0.0f, 0.0f);
            o.point[node] = make_float2(0.0f, 0.0f);
            o.confidence[node] = 0.0f;
            o.measured[node] = 0;
        }
        return;
    }
    const float2 gq = make_float2(gqx, gqy);
    if (!p.field.has[node]) {
        if (threadIdx.x == 0) {
            o.kind[node] = CHIARO_NW_GLOBAL;
            o.global[node] = gq;
            o.point[node] = gq;
            o.confidence[node] = 0.0f;
            o.measured[node] = 0;
        }
        return;
    }
    const int targets[1] = {p.target};
    NodeSmem s = carve_node_smem(smem_raw, 1, taps);
    load_cameras(s.cams, p.views, p.reference, targets, 1);
    if (threadIdx.x == 0) fail = 0;
    __syncthreads();
    stage_node(s, patch, p.views, p.reference, targets, 1, cx, cy, p.radius, p.spatial, true);
    const ViewGeom &g = s.geom[0];
    const PlaneRef target_plane = tv.luma;
    const double shared_depth = p.field.depth[node];
    const double shared_inverse = 1.0 / shared_depth;
    const double min_inverse = 1.0 / p.far_depth, max_inverse = 1.0 / p.near_depth;
    const int lane = threadIdx.x;

    // phase 1: five inverse-depth offsets (lanes 0-4) and the baseline (lane 5)
    if (lane < 5) {
        const double label_offset = -1.0 + 0.5 * lane;
        double inv = clampd_r(shared_inverse + label_offset * p.inverse_step, min_inverse, max_inverse);
        bool ok = g.ray_ok;
        double qx = 0.0, qy = 0.0;
        if (ok) ok = project(s.cams[1], along({g.ox, g.oy, g.oz}, {g.dx, g.dy, g.dz}, 1.0 / inv), qx, qy);
        if (ok) ok = isfinite(qx) && isfinite(qy);
        float2 point = make_float2((float)qx, (float)qy);
        float score = 0.0f;
        if (ok) {
            double ddx = (double)(point.x - gq.x), ddy = (double)(point.y - gq.y);
            ok = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && patch.ok && g.taps_ok &&
                 zncc_score(target_plane, s.gq, s.w, s.wr, patch, taps, ddx, ddy, score);
        }
        if (!ok) atomicOr(&fail, 1);
        sc[lane] = score;
        pts[lane] = point;
    } else if (lane == 5) {
        float score = NAN;
        float sv;
        if (patch.ok && g.taps_ok && zncc_score(target_plane, s.gq, s.w, s.wr, patch, taps, 0.0, 0.0, sv)) score = sv;
        sc[5] = score;
    }
    __syncthreads();
    float2 depth_point = make_float2(0.0f, 0.0f);
    float depth_score = 0.0f;
    if (!fail) {
        float best_objective = 0.0f;
        for (int k = 0; k < 5; ++k) {
            double label_offset = -1.0 + 0.5 * k;
            float objective = sc[k] - (float)fabs(label_offset) * 0.002f;
            if (k == 0 || objective > best_objective) {
                best_objective = objective;
                depth_score = sc[k];
                depth_point = pts[k];
            }
        }
    }
    const float baseline = sc[5];
    __syncthreads();
    // phase 2: eight residual shifts (dy outer, dx inner, centre skipped)
    if (!fail && lane < 8) {
        int k = lane < 4 ? lane : lane + 1;
        float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
        float2 point = make_float2(depth_point.x + dx, depth_point.y + dy);
        double ddx = (double)(point.x - gq.x), ddy = (double)(point.y - gq.y);
        float score = 0.0f;
        bool ok = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && patch.ok && g.taps_ok &&
                  zncc_score(target_plane, s.gq, s.w, s.wr, patch, taps, ddx, ddy, score);
        if (!ok) atomicOr(&fail, 1);
        sc[6 + lane] = score;
        pts[6 + lane] = point;
    }
    __syncthreads();
    if (lane != 0) return;
    bool selected = !fail;
    float sel_score = 0.0f;
    float2 sel_point = make_float2(0.0f, 0.0f);
    if (selected) {
        float b0 = depth_score, b1 = depth_score;
        float2 b2 = depth_point;
        for (int j = 0; j < 8; ++j) {
            int k = j < 4 ? j : j + 1;
            float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
            float residual_sq = dx * dx + dy * dy;
            float objective = sc[6 + j] - residual_sq * 0.002f;
            if (objective > b0) {
                b0 = objective;
                b1 = sc[6 + j];
                b2 = pts[6 + j];
            }
        }
        sel_score = b1;
        sel_point = b2;
    }
    const bool base_ok = baseline == baseline;
    const bool regularized = p.field.regularized[node] != 0;
    const float node_confidence = p.field.confidence[node];
    bool supported = selected && sel_score >= p.minimum_score && (!base_ok || sel_score + 0.01f >= baseline);
    bool contradicted = selected && base_ok && sel_score + 0.12f < baseline;
    o.global[node] = gq;
    o.measured[node] = regularized ? 0 : 1;
    if (contradicted) {
        o.kind[node] = CHIARO_NW_OCCLUDED;
        o.point[node] = gq;
        o.confidence[node] = 0.0f;
    } else if (supported) {
        o.kind[node] = CHIARO_NW_REFINED;
        o.point[node] = sel_point;
        o.confidence[node] = regularized ? node_confidence * 0.6f : 0.5f + 0.5f * node_confidence;
    } else {
        o.kind[node] = CHIARO_NW_GLOBAL;
        o.point[node] = gq;
        o.confidence[node] = 0.0f;
        o.measured[node] = 0;
    }
}

// warp_decisions_agree (depth.rs:682-712)
__device__ inline bool decisions_agree(int kind, uint8_t ck, float2 cg, float2 cp, uint8_t nk, float2 ng, float2 np) {
    if (kind == 0 && ck == CHIARO_NW_REFINED && nk == CHIARO_NW_REFINED) {
        float cdx = cp.x - cg.x, cdy = cp.y - cg.y;
        float ndx = np.x - ng.x, ndy = np.y - ng.y;
        float dx = cdx - ndx, dy = cdy - ndy;
        return dx * dx + dy * dy <= 9.0f;
    }
    return kind == 1 && ck == CHIARO_NW_OCCLUDED && nk == CHIARO_NW_OCCLUDED;
}

// enforce_warp_consensus: reads `src`, writes `dst` (a copy on entry).
__global__ void warp_consensus_kernel(Decisions src, Decisions dst, int columns, int rows) {
    int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= columns * rows) return;
    uint8_t k = src.kind[index];
    int kind, minimum;
    if (k == CHIARO_NW_REFINED) {
        kind = 0;
        minimum = src.measured[index] ? 2 : 4;
    } else if (k == CHIARO_NW_OCCLUDED) {
        kind = 1;
        minimum = src.measured[index] ? 3 : 5;
    } else {
        return;
    }
    int column = index % columns, row = index / columns;
    float2 cg = src.global[index], cp = src.point[index];
    int neighbours = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int x = column + dx, y = row + dy;
            if (x < 0 || y < 0 || x >= columns || y >= rows) continue;
            int ni = y * columns + x;
            neighbours += decisions_agree(kind, k, cg, cp, src.kind[ni], src.global[ni], src.point[ni]) ? 1 : 0;
        }
    if (neighbours < minimum) {
        dst.kind[index] = CHIARO_NW_GLOBAL;
        dst.point[index] = cg;
        dst.confidence[index] = 0.0f;
        dst.measured[index] = 0;
    }
}

// warp_mapping (depth.rs:674-680)
__device__ inline bool decision_mapping(const Decisions &d, int i, float2 &g, float2 &pt) {
    uint8_t k = d.kind[i];
    if (k == CHIARO_NW_GLOBAL) {
        g = d.global[i];
        pt = g;
        return true;
    }
    if (k == CHIARO_NW_REFINED) {
        g = d.global[i];
        pt = d.point[i];
        return true;
    }
    return false;
}

// Does the 4-connected pair (a, b), a west/north of b, form a warp boundary?
__device__ inline bool boundary_pair(const Decisions &d, const float *guidance, int a, int b) {
    float2 ga, pa, gb, pb;
    if (!decision_mapping(d, a, ga, pa) || !decision_mapping(d, b, gb, pb)) return false;
    float dax = pa.x - ga.x, day = pa.y - ga.y;
    float dbx = pb.x - gb.x, dby = pb.y - gb.y;
    float ex = dax - dbx, ey = day - dby;
    bool mapping_edge = ex * ex + ey * ey > WARP_BOUNDARY_DELTA_PX * WARP_BOUNDARY_DELTA_PX;
    bool image_edge = fabsf(guidance[a] - guidance[b]) > WARP_BOUNDARY_CONTRAST;
    return mapping_edge && image_edge;
}

// suppress_warp_boundaries: reads `src`, writes `dst` (a copy on entry).
__global__ void warp_boundary_kernel(Decisions src, Decisions dst, const float *__restrict__ guidance, int columns,
                                     int rows) {
    int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= columns * rows) return;
    float2 g, pt;
    if (!decision_mapping(src, index, g, pt)) return;
    int column = index % columns, row = index / columns;
    bool boundary = (column + 1 < columns && boundary_pair(src, guidance, index, index + 1)) ||
                    (row + 1 < rows && boundary_pair(src, guidance, index, index + columns)) ||
                    (column > 0 && boundary_pair(src, guidance, index - 1, index)) ||
                    (row > 0 && boundary_pair(src, guidance, index - columns, index));
    if (boundary) {
        dst.kind[index] = CHIARO_NW_BOUNDARY;
        dst.point[index] = g;
        dst.confidence[index] = 0.0f;
    }
}

// Output warp and decision counts (depth.rs:490-532). counts: refined,
// occluded, boundary.
__global__ void warp_output_kernel(Decisions d, float2 *points, float *confidence,
                                   unsigned long long *counts, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int refined = 0, occluded = 0, boundary = 0;
    if (i < n) {
        uint8_t k = d.kind[i];
        float2 pt;
        float c;
        switch (k) {
            case CHIARO_NW_UNDEFINED: pt = make_float2(NAN, NAN); c = 0.0f; break;
            case CHIARO_NW_GLOBAL: pt = d.global[i]; c = 1.0f; break;
            case CHIARO_NW_REFINED: pt = d.point[i]; c = d.confidence[i]; refined = 1; break;
            case CHIARO_NW_OCCLUDED: pt = d.global[i]; c = 0.0f; occluded = 1; break;
            default: pt = d.global[i]; c = 0.0f; boundary = 1; break;
        }
        points[i] = pt;
        confidence[i] = c;
    }
    unsigned full = 0xffffffffu;
    int rc = __popc(__ballot_sync(full, refined)), oc = __popc(__ballot_sync(full, occluded)),
        bc = __popc(__ballot_sync(full, boundary));
    if ((threadIdx.x & 31) == 0) {
        if (rc) atomicAdd(counts + 0, (unsigned long long)rc);
        if (oc) atomicAdd(counts + 1, (unsigned long long)oc);
        if (bc) atomicAdd(counts + 2, (unsigned long long)bc);
    }
}

}  // namespace chiaro
