// decisions.cuh — the per-target cross-camera consistency check
// (crates/chiaro-fusion/src/depth.rs:420-547): refine_one_view (1634-1708),
// score_one_view_at_point (1710-1736), the Refined / Occluded / Global
// classification (458-485), enforce_warp_consensus (582-618),
// suppress_warp_boundaries (620-672) and the output warp (490-532).
//
// Decisions for every target run in one launch: eight lanes per (node, target).
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
    int reference, n_targets;
    int targets[MAX_VIEWS];
    int columns, rows, step;
    Field field;
    const GeomRec *geometry;  // [node][target] of the fine grid
    double inverse_step, near_depth, far_depth;
    int radius;
    const float *spatial;
    float minimum_score;
    Decisions out[MAX_VIEWS];  // per target (index into targets)
};

constexpr int DECISION_LANES = 8;     // lanes per (node, target)
constexpr int DECISION_NODES = 32;    // nodes per CTA (256 threads)

__host__ __device__ inline size_t decision_smem_bytes(int taps) {
    // per node slot: r, w, wr, and the target's tap positions (g/2)
    return (size_t)DECISION_NODES * (3 * taps * sizeof(float) + taps * sizeof(double2));
}

// One CTA handles 32 nodes of one target (blockIdx.y); each node belongs to an
// aligned group of 8 lanes inside one warp. Lanes 0-4 score the five
// inverse-depth offsets and lane 5 the baseline; after lane 0 picks the best
// offset, lanes 0-7 score the eight residual shifts; lane 0 classifies.
__global__ void __launch_bounds__(DECISION_LANES * DECISION_NODES) target_decision_kernel(DecisionParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patch[DECISION_NODES];
    __shared__ float sc[DECISION_NODES][16];
    __shared__ float2 pts[DECISION_NODES][16];
    __shared__ int fail[DECISION_NODES], taps_ok[DECISION_NODES];
    __shared__ TapBox boxes[DECISION_NODES];
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const int slot = threadIdx.x / DECISION_LANES, lane = threadIdx.x % DECISION_LANES;
    const int node = blockIdx.x * DECISION_NODES + slot;
    const int vi = blockIdx.y;
    const int target = p.targets[vi];
    const DevView &tv = p.views[target];
    const DevView &rv = p.views[p.reference];
    Decisions o = p.out[vi];
    float *r = reinterpret_cast<float *>(smem_raw) + (size_t)slot * 3 * taps;
    float *w = r + taps, *wr = w + taps;
    double2 *gh = reinterpret_cast<double2 *>(smem_raw + (size_t)DECISION_NODES * 3 * taps * sizeof(float)) +
                  (size_t)slot * taps;

    bool active = node < p.columns * p.rows;
    const double cx = active ? (double)((node % p.columns) * p.step) : 0.0;
    const double cy = active ? (double)((node / p.columns) * p.step) : 0.0;
    float gqx = 0.0f, gqy = 0.0f;
    if (active) {
        bool defined = warp_map(tv.warp, (float)cx, (float)cy, gqx, gqy);
        if (!defined || !p.field.has[node]) {
            if (lane == 0) {
                o.kind[node] = defined ? CHIARO_NW_GLOBAL : CHIARO_NW_UNDEFINED;
                o.global[node] = make_float2(gqx, gqy);
                o.point[node] = make_float2(gqx, gqy);
                o.confidence[node] = 0.0f;
                o.measured[node] = 0;
            }
            active = false;
        }
    }
    const float2 gq_c = make_float2(gqx, gqy);
    // reference patch and tap positions of this node (8 lanes)
    float centre = 0.0f;
    bool centre_ok = false;
    if (active) {
        centre_ok = plane_sample(rv.luma, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
        if (lane == 0) {
            patch[slot].ok = centre_ok;
            patch[slot].centre = centre;
            taps_ok[slot] = 1;
            fail[slot] = 0;
        }
    }
    __syncwarp();
    if (active) {
        for (int t = lane; t < taps; t += DECISION_LANES) {
            int dx, dy;
            tap_offset(t, p.radius, dx, dy);
            double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
            float value = 0.0f;
            if (!plane_sample(rv.luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value)) patch[slot].ok = 0;
            float weight = p.spatial[t] * exp_f32(-1.2f * fabsf(value - centre));
            r[t] = value;
            w[t] = weight;
            wr[t] = weight * value;
            float qx = 0.0f, qy = 0.0f;
            if (!warp_map(tv.warp, (float)px, (float)py, qx, qy)) taps_ok[slot] = 0;
            gh[t] = make_double2((double)qx * 0.5, (double)qy * 0.5);
        }
    }
    __syncwarp();
    if (active && lane == 3) {  // box of this node's taps (one lane of the group)
        TapBox b{gh[0].x, gh[0].x, gh[0].y, gh[0].y};
        for (int t = 1; t < taps; ++t) {
            b.xmin = fmin(b.xmin, gh[t].x);
            b.xmax = fmax(b.xmax, gh[t].x);
            b.ymin = fmin(b.ymin, gh[t].y);
            b.ymax = fmax(b.ymax, gh[t].y);
        }
        boxes[slot] = b;
    }
    if (active && lane < 3) {  // the three sequential reference sums
        float sum = 0.0f;
        if (lane == 0)
            for (int t = 0; t < taps; ++t) sum += w[t];
        else if (lane == 1)
            for (int t = 0; t < taps; ++t) sum += wr[t];
        else
            for (int t = 0; t < taps; ++t) sum += wr[t] * r[t];
        if (lane == 0) patch[slot].count = sum;
        if (lane == 1) patch[slot].sum_r = sum;
        if (lane == 2) patch[slot].sum_rr = sum;
    }
    __syncwarp();
    if (active && lane == 0)
        patch[slot].ref_energy = patch[slot].sum_rr - patch[slot].sum_r * patch[slot].sum_r / patch[slot].count;
    __syncwarp();
    ViewGeom g;
    if (active) geom_from_rec(p.geometry[(size_t)node * p.n_targets + vi], camera_origin(rv.cam), g);
    const bool zncc_ok = active && patch[slot].ok && taps_ok[slot];
    const TargetRef target_ref{tv.luma, tv.pairs};
    double shared_inverse = 0.0, min_inverse = 1.0 / p.far_depth, max_inverse = 1.0 / p.near_depth;
    if (active) shared_inverse = 1.0 / p.field.depth[node];
    // phase 1: five inverse-depth offsets and the baseline
    if (active && lane < 5) {
        const double label_offset = -1.0 + 0.5 * lane;
        double inv = clampd_r(shared_inverse + label_offset * p.inverse_step, min_inverse, max_inverse);
        bool ok = g.ray_ok;
        double qx = 0.0, qy = 0.0;
        if (ok) ok = project(tv.cam, along({g.ox, g.oy, g.oz}, {g.dx, g.dy, g.dz}, 1.0 / inv), qx, qy);
        if (ok) ok = isfinite(qx) && isfinite(qy);
        float2 point = make_float2((float)qx, (float)qy);
        float score = 0.0f;
        if (ok) {
            double ddx = (double)(point.x - gq_c.x), ddy = (double)(point.y - gq_c.y);
            ok = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && zncc_ok &&
                 zncc_any(target_ref, gh, boxes[slot], w, wr, patch[slot], taps, ddx, ddy, score);
        }
        if (!ok) atomicOr(&fail[slot], 1);
        sc[slot][lane] = score;
        pts[slot][lane] = point;
    } else if (active && lane == 5) {
        float score = NAN, sv;
        if (zncc_ok && zncc_any(target_ref, gh, boxes[slot], w, wr, patch[slot], taps, 0.0, 0.0, sv)) score = sv;
        sc[slot][5] = score;
    }
    __syncwarp();
    if (active && lane == 0 && !fail[slot]) {  // best offset, in order, strict improvement
        float best_objective = 0.0f;
        for (int k = 0; k < 5; ++k) {
            float objective = sc[slot][k] - (float)fabs(-1.0 + 0.5 * k) * 0.002f;
            if (k == 0 || objective > best_objective) {
                best_objective = objective;
                sc[slot][14] = sc[slot][k];
                pts[slot][14] = pts[slot][k];
            }
        }
    }
    __syncwarp();
    // phase 2: eight residual shifts (dy outer, dx inner, centre skipped)
    if (active && !fail[slot]) {
        int k = lane < 4 ? lane : lane + 1;
        float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
        float2 depth_point = pts[slot][14];
        float2 point = make_float2(depth_point.x + dx, depth_point.y + dy);
        double ddx = (double)(point.x - gq_c.x), ddy = (double)(point.y - gq_c.y);
        float score = 0.0f;
        bool ok = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && zncc_ok &&
                  zncc_any(target_ref, gh, boxes[slot], w, wr, patch[slot], taps, ddx, ddy, score);
        if (!ok) atomicOr(&fail[slot], 1);
        sc[slot][6 + lane] = score;
        pts[slot][6 + lane] = point;
    }
    __syncwarp();
    if (!active || lane != 0) return;
    const bool selected = !fail[slot];
    float sel_score = 0.0f;
    float2 sel_point = make_float2(0.0f, 0.0f);
    if (selected) {
        float b0 = sc[slot][14], b1 = sc[slot][14];
        float2 b2 = pts[slot][14];
        for (int j = 0; j < 8; ++j) {
            int k = j < 4 ? j : j + 1;
            float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
            float objective = sc[slot][6 + j] - (dx * dx + dy * dy) * 0.002f;
            if (objective > b0) {
                b0 = objective;
                b1 = sc[slot][6 + j];
                b2 = pts[slot][6 + j];
            }
        }
        sel_score = b1;
        sel_point = b2;
    }
    const float baseline = sc[slot][5];
    const bool base_ok = baseline == baseline;
    const bool regularized = p.field.regularized[node] != 0;
    const float node_confidence = p.field.confidence[node];
    const bool supported = selected && sel_score >= p.minimum_score && (!base_ok || sel_score + 0.01f >= baseline);
    const bool contradicted = selected && base_ok && sel_score + 0.12f < baseline;
    o.global[node] = gq_c;
    o.measured[node] = regularized ? 0 : 1;
    if (contradicted) {
        o.kind[node] = CHIARO_NW_OCCLUDED;
        o.point[node] = gq_c;
        o.confidence[node] = 0.0f;
    } else if (supported) {
        o.kind[node] = CHIARO_NW_REFINED;
        o.point[node] = sel_point;
        o.confidence[node] = regularized ? node_confidence * 0.6f : 0.5f + 0.5f * node_confidence;
    } else {
        o.kind[node] = CHIARO_NW_GLOBAL;
        o.point[node] = gq_c;
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
