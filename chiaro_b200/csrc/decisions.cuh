// decisions.cuh — the per-target cross-camera consistency check
// (crates/chiaro-fusion/src/depth.rs:420-547): refine_one_view (1634-1708),
// score_one_view_at_point (1710-1736), the Refined / Occluded / Global
// classification (458-485), enforce_warp_consensus (582-618),
// suppress_warp_boundaries (620-672) and the output warp (490-532).
//
// Decisions for every target run in one launch: a warp per fine node stages
// the reference patch once and spreads the (target, offset) and (target, shift)
// correlations over its lanes.
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
    TapLattice lattice;       // of the fine grid, or planes == nullptr
    const RefPatch *patches;  // [node] reference patch at `radius`, or nullptr
    double inverse_step, near_depth, far_depth;
    int radius;
    const float *spatial;
    float minimum_score;
    Decisions out[MAX_VIEWS];  // per target (index into targets)
};

constexpr int DECISION_WARPS = 8;  // most nodes (warps) per CTA

// Per-warp shared memory of the decisions for V targets and T taps.
struct DecisionSlot {
    float *rr;             // [T] reference patch (w r) r
    float2 *wt;            // [T] reference patch (w, w r)
    double2 *gh;           // [V][T] tap positions g/2
    TapBox *box;           // [V]
    float *sc;             // [V][16]: 0-4 offsets, 5 baseline, 6-13 shifts, 14 best offset
    float2 *pts;           // [V][16]
    double2 *disp;         // [8 V] displacement of each listed correlation
    unsigned short *list;  // [8 V] listed correlations
    int *flags;            // [V]: nonzero once the target's refinement failed
};

__host__ __device__ inline size_t decision_slot_bytes(int V, int taps) {
    return align16(taps * sizeof(float)) + align16(taps * sizeof(float2)) + align16((size_t)V * taps * sizeof(double2)) +
           align16(V * sizeof(TapBox)) + align16((size_t)V * 16 * sizeof(float)) +
           align16((size_t)V * 16 * sizeof(float2)) + align16((size_t)8 * V * sizeof(double2)) +
           align16((size_t)8 * V * sizeof(unsigned short)) + align16(V * sizeof(int));
}

__device__ inline DecisionSlot carve_decision_slot(unsigned char *base, int V, int taps) {
    DecisionSlot d;
    size_t o = 0;
    d.rr = reinterpret_cast<float *>(base);
    o += align16(taps * sizeof(float));
    d.wt = reinterpret_cast<float2 *>(base + o);
    o += align16(taps * sizeof(float2));
    d.gh = reinterpret_cast<double2 *>(base + o);
    o += align16((size_t)V * taps * sizeof(double2));
    d.box = reinterpret_cast<TapBox *>(base + o);
    o += align16(V * sizeof(TapBox));
    d.sc = reinterpret_cast<float *>(base + o);
    o += align16((size_t)V * 16 * sizeof(float));
    d.pts = reinterpret_cast<float2 *>(base + o);
    o += align16((size_t)V * 16 * sizeof(float2));
    d.disp = reinterpret_cast<double2 *>(base + o);
    o += align16((size_t)8 * V * sizeof(double2));
    d.list = reinterpret_cast<unsigned short *>(base + o);
    o += align16((size_t)8 * V * sizeof(unsigned short));
    d.flags = reinterpret_cast<int *>(base + o);
    return d;
}

__device__ __forceinline__ void write_decision(const Decisions &o, int node, uint8_t kind, float2 g, float2 pt,
                                               float confidence, uint8_t measured) {
    o.kind[node] = kind;
    o.global[node] = g;
    o.point[node] = pt;
    o.confidence[node] = confidence;
    o.measured[node] = measured;
}

// Append the items whose `listed` is set to d.list (in item order) with their
// displacement; returns the new length on every lane. Every lane calls it.
__device__ __forceinline__ int list_items(const DecisionSlot &d, int count, bool listed, int item, double ddx,
                                          double ddy) {
    const unsigned mask = __ballot_sync(0xffffffffu, listed);
    if (listed) {
        const int at = count + __popc(mask & ((1u << (threadIdx.x & 31)) - 1u));
        d.list[at] = (unsigned short)item;
        d.disp[at] = make_double2(ddx, ddy);
    }
    return count + __popc(mask);
}

// Scores the pooled lists of the CTA's nodes (node k's count[k] entries of its
// d.list / d.disp, node after node), so the lanes of all warps share the
// correlations of one phase. Phase 1 items are (target, offset k < 5 or baseline
// k = 5), phase 2 items (target, shift j < 8). A failed correlation of an offset
// or shift marks its target's refinement as failed.
__device__ inline void decision_pool_scores(const DecisionParams &p, unsigned char *smem_raw, size_t slot_bytes,
                                            const RefPatch *patches, const int *count, int nodes, int taps,
                                            bool shifts) {
    const int V = p.n_targets;
    int pooled = 0;
    for (int k = 0; k < nodes; ++k) pooled += count[k];
    for (int j = threadIdx.x; j < pooled; j += blockDim.x) {
        int k = 0, at = j;
        while (at >= count[k]) at -= count[k++];
        const DecisionSlot d = carve_decision_slot(smem_raw + (size_t)k * slot_bytes, V, taps);
        const int item = d.list[at];
        const int v = shifts ? item >> 3 : item / 6;
        const DevView &tv = p.views[p.targets[v]];
        const double2 dd = d.disp[at];
        float score;
        const bool ok = zncc_any(TargetRef{tv.luma, tv.quads}, d.gh + v * taps, d.box[v], d.wt, patches[k], taps,
                                 dd.x, dd.y, score);
        const int kk = shifts ? 6 + (item & 7) : item - v * 6;
        if (ok)
            d.sc[v * 16 + kk] = score;
        else if (shifts || kk < 5)
            atomicOr(&d.flags[v], 1);
    }
}

// A warp per fine node, every target (depth.rs:420-485 with refine_one_view,
// depth.rs:1634-1708). Each phase first settles which correlations run, lists
// them, and runs the list from one call site, so the lanes stay converged.
// POOLED (for one or two targets, whose phases list at most 12 and 16 items per
// node): the CTA scores the pooled lists of all its nodes instead, so few warps
// issue each phase's correlations; nodes without work stay for the CTA's
// barriers.
template <bool POOLED>
__global__ void __launch_bounds__(32 * DECISION_WARPS) target_decision_kernel(DecisionParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patches[DECISION_WARPS];
    __shared__ int count[DECISION_WARPS];
    const unsigned full = 0xffffffffu;
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nodes = blockDim.x >> 5;
    const int node = blockIdx.x * nodes + slot;
    const bool in_grid = node < p.columns * p.rows;  // whole warp
    if (!POOLED && !in_grid) return;
    const int V = p.n_targets;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const size_t slot_bytes = decision_slot_bytes(V, taps);
    DecisionSlot d = carve_decision_slot(smem_raw + (size_t)slot * slot_bytes, V, taps);
    RefPatch &patch = patches[slot];
    const DevView &rv = p.views[p.reference];
    const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
    const bool has = in_grid && p.field.has[node];
    // the global warp at the node: Undefined, or Global without a depth (depth.rs:433-440);
    // lane v holds target v's mapping
    unsigned defined = 0u;
    float2 gq = make_float2(0.0f, 0.0f);
    if (in_grid && lane < V) {
        float gx = 0.0f, gy = 0.0f;
        const bool ok = warp_map(p.views[p.targets[lane]].warp, (float)cx, (float)cy, gx, gy);
        gq = make_float2(gx, gy);
        if (ok) defined = 1u << lane;
        if (!ok || !has)
            write_decision(p.out[lane], node, ok ? CHIARO_NW_GLOBAL : CHIARO_NW_UNDEFINED, gq, gq, 0.0f, 0);
        d.flags[lane] = 0;
    }
    defined = __reduce_or_sync(full, defined);
    const bool active = has && defined;  // whole warp
    if (!POOLED && !active) return;
    unsigned undefined_taps = 0u;
    if (active)
        undefined_taps = warp_stage_patch(p.views, p.reference, p.targets, V, cx, cy, p.radius, p.spatial, d.rr,
                                          d.wt, d.gh, d.box, patch, p.lattice, p.patches ? p.patches + node : nullptr);
    const bool patch_ok = active && patch.ok;
    const D3 origin = camera_origin(rv.cam);
    const double shared_inverse = active ? 1.0 / p.field.depth[node] : 0.0;
    const double min_inverse = 1.0 / p.far_depth, max_inverse = 1.0 / p.near_depth;
    // phase 1: per target, five inverse-depth offsets (k < 5) and the baseline (k = 5)
    int listed = 0;
    for (int base = 0; active && base < 6 * V; base += 32) {
        const int item = base + lane;
        const int v = item / 6, k = item - v * 6;
        const int vs = v < V ? v : 0;
        const float2 gq_c = make_float2(__shfl_sync(full, gq.x, vs), __shfl_sync(full, gq.y, vs));
        bool zncc = false;
        double ddx = 0.0, ddy = 0.0;
        if (item < 6 * V && ((defined >> v) & 1u)) {
            const DevView &tv = p.views[p.targets[v]];
            const bool zncc_ok = patch_ok && !((undefined_taps >> v) & 1u);
            if (k < 5) {
                ViewGeom g;
                geom_from_rec(p.geometry[(size_t)node * V + v], origin, g);
                const double label_offset = -1.0 + 0.5 * k;
                double inv = clampd_r(shared_inverse + label_offset * p.inverse_step, min_inverse, max_inverse);
                bool ok = g.ray_ok;
                double qx = 0.0, qy = 0.0;
                if (ok) ok = project(tv.cam, along({g.ox, g.oy, g.oz}, {g.dx, g.dy, g.dz}, 1.0 / inv), qx, qy);
                if (ok) ok = isfinite(qx) && isfinite(qy);
                const float2 point = make_float2((float)qx, (float)qy);
                if (ok) {
                    ddx = (double)(point.x - gq_c.x);
                    ddy = (double)(point.y - gq_c.y);
                    ok = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && zncc_ok;
                }
                if (!ok) atomicOr(&d.flags[v], 1);
                d.sc[v * 16 + k] = 0.0f;
                d.pts[v * 16 + k] = point;
                zncc = ok;
            } else {
                d.sc[v * 16 + 5] = NAN;
                zncc = zncc_ok;
            }
        }
        listed = list_items(d, listed, zncc, item, ddx, ddy);
    }
    if constexpr (POOLED) {
        if (lane == 0) count[slot] = listed;
        __syncthreads();
        decision_pool_scores(p, smem_raw, slot_bytes, patches, count, nodes, taps, false);
        __syncthreads();
    } else {
        __syncwarp();
        for (int j = lane; j < listed; j += 32) {
            const int item = d.list[j];
            const int v = item / 6, k = item - v * 6;
            const DevView &tv = p.views[p.targets[v]];
            const double2 dd = d.disp[j];
            float score;
            if (zncc_any(TargetRef{tv.luma, tv.quads}, d.gh + v * taps, d.box[v], d.wt, patch, taps, dd.x, dd.y,
                         score))
                d.sc[v * 16 + k] = score;
            else if (k < 5)
                atomicOr(&d.flags[v], 1);
        }
        __syncwarp();
    }
    // best offset per target: in order, strict improvement
    const unsigned failed = __ballot_sync(full, active && lane < V && d.flags[lane < V ? lane : 0]);
    if (active && lane < V && ((defined >> lane) & 1u) && !((failed >> lane) & 1u)) {
        float *sc = d.sc + lane * 16;
        float2 *pts = d.pts + lane * 16;
        float best_objective = 0.0f;
        for (int k = 0; k < 5; ++k) {
            float objective = sc[k] - (float)fabs(-1.0 + 0.5 * k) * 0.002f;
            if (k == 0 || objective > best_objective) {
                best_objective = objective;
                sc[14] = sc[k];
                pts[14] = pts[k];
            }
        }
    }
    __syncwarp();
    // phase 2: per target, eight residual shifts (dy outer, dx inner, centre skipped)
    listed = 0;
    for (int base = 0; active && base < 8 * V; base += 32) {
        const int item = base + lane;
        const int v = item >> 3, j = item & 7;
        const int vs = v < V ? v : 0;
        const float2 gq_c = make_float2(__shfl_sync(full, gq.x, vs), __shfl_sync(full, gq.y, vs));
        bool zncc = false;
        double ddx = 0.0, ddy = 0.0;
        if (item < 8 * V && ((defined >> v) & 1u) && !((failed >> v) & 1u)) {
            const int k = j < 4 ? j : j + 1;
            const float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
            const float2 depth_point = d.pts[v * 16 + 14];
            const float2 point = make_float2(depth_point.x + dx, depth_point.y + dy);
            ddx = (double)(point.x - gq_c.x);
            ddy = (double)(point.y - gq_c.y);
            zncc = !(fabs(ddx) > 128.0 || fabs(ddy) > 128.0) && patch_ok && !((undefined_taps >> v) & 1u);
            if (!zncc) atomicOr(&d.flags[v], 1);
            d.sc[v * 16 + 6 + j] = 0.0f;
            d.pts[v * 16 + 6 + j] = point;
        }
        listed = list_items(d, listed, zncc, item, ddx, ddy);
    }
    if constexpr (POOLED) {
        __syncwarp();
        if (lane == 0) count[slot] = listed;
        __syncthreads();
        decision_pool_scores(p, smem_raw, slot_bytes, patches, count, nodes, taps, true);
        __syncthreads();
    } else {
        __syncwarp();
        for (int j = lane; j < listed; j += 32) {
            const int item = d.list[j];
            const int v = item >> 3;
            const DevView &tv = p.views[p.targets[v]];
            const double2 dd = d.disp[j];
            float score;
            if (zncc_any(TargetRef{tv.luma, tv.quads}, d.gh + v * taps, d.box[v], d.wt, patch, taps, dd.x, dd.y,
                         score))
                d.sc[v * 16 + 6 + (item & 7)] = score;
            else
                atomicOr(&d.flags[v], 1);
        }
        __syncwarp();
    }
    // classification (depth.rs:458-485), lane v for target v
    if (!active || lane >= V || !((defined >> lane) & 1u)) return;
    const Decisions o = p.out[lane];
    const float *sc = d.sc + lane * 16;
    const float2 *pts = d.pts + lane * 16;
    const bool selected = !d.flags[lane];
    float sel_score = 0.0f;
    float2 sel_point = make_float2(0.0f, 0.0f);
    if (selected) {
        float b0 = sc[14], b1 = sc[14];
        float2 b2 = pts[14];
        for (int j = 0; j < 8; ++j) {
            int k = j < 4 ? j : j + 1;
            float dx = -1.5f + 1.5f * (float)(k % 3), dy = -1.5f + 1.5f * (float)(k / 3);
            float objective = sc[6 + j] - (dx * dx + dy * dy) * 0.002f;
            if (objective > b0) {
                b0 = objective;
                b1 = sc[6 + j];
                b2 = pts[6 + j];
            }
        }
        sel_score = b1;
        sel_point = b2;
    }
    const float baseline = sc[5];
    const bool base_ok = baseline == baseline;
    const bool regularized = p.field.regularized[node] != 0;
    const float node_confidence = p.field.confidence[node];
    const bool supported = selected && sel_score >= p.minimum_score && (!base_ok || sel_score + 0.01f >= baseline);
    const bool contradicted = selected && base_ok && sel_score + 0.12f < baseline;
    const uint8_t measured = regularized ? 0 : 1;
    if (contradicted)
        write_decision(o, node, CHIARO_NW_OCCLUDED, gq, gq, 0.0f, measured);
    else if (supported)
        write_decision(o, node, CHIARO_NW_REFINED, gq, sel_point,
                       regularized ? node_confidence * 0.6f : 0.5f + 0.5f * node_confidence, measured);
    else
        write_decision(o, node, CHIARO_NW_GLOBAL, gq, gq, 0.0f, 0);
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
