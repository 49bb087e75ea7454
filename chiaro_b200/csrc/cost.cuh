// cost.cuh — build_cost_volume (crates/chiaro-fusion/src/depth.rs:1187-1277).
//
// One CTA of four warps per coarse node. The CTA stages the node's reference
// patch, every target's tap positions and the label-independent geometry in
// shared memory. It then settles, for every (target, label) item, whether the
// hypothesis projects within reach and whether all its taps sample inside the
// target (the fast path), and lists the items that are scored, fast ones first,
// view-major so neighbouring lanes share a target. All four warps run the
// correlations of that list, so no lane waits on an item that is never scored
// and the D = planes + 1 labels leave no nearly empty warp. Last, a thread per
// label aggregates the views (depth.rs:1761-1770) and writes the label-minor
// score and cost rows (node-major [N][D], as the reference lays them out).
//
// The same kernel scores a subset of the labels for the learned band: each node
// scores `slots` labels, slot 0 being label 0 (the global warp) and the others
// either one label list shared by every node (the band proposal's sampled labels)
// or its tile's band [O, O + slots - 1); rows are then [N][slots]. A node list
// restricts the CTAs to some nodes (the fallback windows), each writing the row
// of its list position. A label's score and cost do not depend on which other
// labels a node scores, so every subset holds the full volume's values bit for bit.
#pragma once

#include "zncc.cuh"

namespace chiaro {

struct CostParams {
    const DevView *views;       // all modules
    int reference;              // reference module
    int n_targets;              // scored modules (accepted, calibrated, not the reference)
    int targets[MAX_VIEWS];
    int columns, rows, step;    // coarse grid
    int labels;                 // D = planes + 1
    const double *label_depth;  // [D], label 0 unused (the global warp)
    const float *spatial;       // [(2r+1)^2] spatial weights
    const GeomRec *geometry;    // [node][target]
    int radius;
    TapLattice lattice;         // of this grid, or planes == nullptr
    int minimum_support, best_view_count;
    float *scores, *costs, *guidance;
    uint8_t *tested;
    // label subsets (slots == labels with no list and no bands: the full volume)
    int slots;                  // labels scored per node; rows of the outputs
    const int *label_list;      // [slots]: slot -> label, or nullptr
    const int *band_first;      // [tiles_y][tiles_x]: slot s > 0 -> label band_first[tile] + s - 1, or nullptr
    int band_tile, band_tiles_x;
    const int *node_list;       // CTA b scores node node_list[b] into output row b, or nullptr
};

// The label of a slot of `node` (see CostParams).
__device__ __forceinline__ int cost_slot_label(const CostParams &p, int node, int slot) {
    if (p.label_list) return __ldg(p.label_list + slot);
    if (p.band_first) {
        if (slot == 0) return 0;
        const int row = node / p.columns, column = node - row * p.columns;
        return __ldg(p.band_first + (row / p.band_tile) * p.band_tiles_x + column / p.band_tile) + slot - 1;
    }
    return slot;
}

// Threads of a node CTA: T (a multiple of 32) is the kernel's template parameter; the
// stage's default is COST_THREADS, and the autotuner times the COST_SHAPES once per
// (targets, labels scored, radius) bucket. Every shape lists, scores and aggregates the
// same items, each score computed alone and the views aggregated in their order, so the
// results are the same bits whatever the shape.
constexpr int COST_THREADS = 128;
constexpr int COST_SHAPES[] = {64, 96, 128, 160, 192};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) / 16 * 16; }

// Dynamic shared memory of a node CTA.
struct NodeSmem {
    ViewGeom *geom;        // [V]
    TapBox *box;           // [V]
    float *rr;             // [T] (w r) r
    float2 *wt;            // [T] (w, w r)
    double2 *gh;           // [V][T] g/2 of the tap positions
    float *score;          // [V][D] per-view scores, NaN = None
    unsigned short *list;  // [V][D] scored items: fast path from the front, exact path from the back
    double2 *disp;         // [V][D] displacement (ddx, ddy) of each item; ddx NaN: out of reach
};

__host__ __device__ inline size_t node_smem_bytes(int V, int taps, int labels) {
    const size_t items = (size_t)V * labels;
    return align16(V * sizeof(ViewGeom)) + align16(V * sizeof(TapBox)) +
           align16(taps * sizeof(float)) + align16(taps * sizeof(float2)) +
           align16((size_t)V * taps * sizeof(double2)) +
           align16(items * sizeof(float)) + align16(items * sizeof(unsigned short)) + items * sizeof(double2);
}

__device__ inline NodeSmem carve_node_smem(unsigned char *base, int V, int taps, int labels) {
    const size_t items = (size_t)V * labels;
    NodeSmem s;
    size_t o = 0;
    s.geom = reinterpret_cast<ViewGeom *>(base + o);
    o += align16(V * sizeof(ViewGeom));
    s.box = reinterpret_cast<TapBox *>(base + o);
    o += align16(V * sizeof(TapBox));
    s.rr = reinterpret_cast<float *>(base + o);
    o += align16(taps * sizeof(float));
    s.wt = reinterpret_cast<float2 *>(base + o);
    o += align16(taps * sizeof(float2));
    s.gh = reinterpret_cast<double2 *>(base + o);
    o += align16((size_t)V * taps * sizeof(double2));
    s.score = reinterpret_cast<float *>(base + o);
    o += align16(items * sizeof(float));
    s.list = reinterpret_cast<unsigned short *>(base + o);
    o += align16(items * sizeof(unsigned short));
    s.disp = reinterpret_cast<double2 *>(base + o);
    return s;
}

// Registers bounded to 64 per thread at every shape (1024 / T CTAs per SM).
template <int T>
__global__ void __launch_bounds__(T, 1024 / T) cost_volume_kernel(CostParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ RefPatch patch;
    __shared__ unsigned warp_undefined[T / 32];  // bit v: a tap of target v has no global warp
    __shared__ int list_ends[2];                 // fast items listed, exact items listed
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int warps = T / 32;
    const int out_row = blockIdx.x;
    const int node = p.node_list ? __ldg(p.node_list + out_row) : out_row;
    const int V = p.n_targets, D = p.slots, full_labels = p.labels;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const int total = V * D;
    const int chunks = (total + T - 1) / T;
    const SmallDiv by_slots(D), by_taps(taps), side(2 * p.radius + 1);  // item / D, i / taps, tap rows
    NodeSmem s = carve_node_smem(smem_raw, V, taps, D);
    const double cx = (double)((node % p.columns) * p.step), cy = (double)((node / p.columns) * p.step);
    const DevView &rv = p.views[p.reference];
    const D3 origin = camera_origin(rv.cam);

    // ---- staging: geometry, reference patch, tap positions (from the tap lattice when
    // the grid has one)
    if (tid < V) geom_from_rec(p.geometry[(size_t)node * V + tid], origin, s.geom[tid]);
    if (tid < 2) list_ends[tid] = 0;  // read after the staging's barriers
    const TapLattice &lat = p.lattice;
    const size_t at0 = lat.planes ? lat.index(cx, cy) : 0;
    float centre = 0.0f;
    bool centre_ok;
    if (lat.planes) {
        const float2 c = __ldg(lat.planes + at0);
        centre = c.x;
        centre_ok = c.y != 0.0f;
    } else {
        centre_ok = plane_sample(rv.luma, (float)((cx - 0.5) * 0.5), (float)((cy - 0.5) * 0.5), centre);
    }
    bool sampled = true;
    for (int t = tid; t < taps; t += T) {
        int dx, dy;
        tap_offset(t, p.radius, side, dx, dy);
        float value = 0.0f;
        if (lat.planes) {
            const float2 r = __ldg(lat.planes + at0 + (ptrdiff_t)dy * lat.columns + dx);
            value = r.x;
            sampled &= r.y != 0.0f;
        } else {
            double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
            sampled &= plane_sample(rv.luma, (float)((px - 0.5) * 0.5), (float)((py - 0.5) * 0.5), value);
        }
        float weight = p.spatial[t] * exp_f32(-1.2f * fabsf(value - centre));
        float weighted = weight * value;
        s.wt[t] = make_float2(weight, weighted);
        s.rr[t] = weighted * value;
    }
    unsigned undefined = 0u;
    for (int i = tid; i < V * taps; i += T) {
        const int v = by_taps.quotient(i), t = i - v * taps;
        int dx, dy;
        tap_offset(t, p.radius, side, dx, dy);
        float qx = 0.0f, qy = 0.0f;
        if (lat.planes) {
            const float2 q = __ldg(lat.planes + (size_t)(v + 1) * lat.plane_size() + at0 +
                                   (ptrdiff_t)dy * lat.columns + dx);
            qx = q.x;
            qy = q.y;
            if (qx != qx) undefined |= 1u << v;
        } else {
            double px = cx + (double)dx * 2.0, py = cy + (double)dy * 2.0;
            if (!warp_map(p.views[p.targets[v]].warp, (float)px, (float)py, qx, qy)) undefined |= 1u << v;
        }
        s.gh[i] = make_double2((double)qx * 0.5, (double)qy * 0.5);
    }
    undefined = __reduce_or_sync(full, undefined);
    if (lane == 0) warp_undefined[warp] = undefined;
    const bool all_sampled = __syncthreads_and(sampled);
    // displacement of every (target, slot) item, view-major: item = v * D + slot
    for (int item = tid; item < total; item += T) {
        const int v = by_slots.quotient(item), label = cost_slot_label(p, node, item - v * D);
        const ViewGeom &g = s.geom[v];
        double ddx = 0.0, ddy = 0.0;
        bool ok = g.gc_ok;
        if (ok && label > 0) ok = depth_delta(p.views[p.targets[v]].cam, g, p.label_depth[label], ddx, ddy);
        s.disp[item] = make_double2(ok ? ddx : NAN, ddy);
    }
    // tap boxes (eight lanes per target) and the three sequential reference
    // sums (lanes 0-2 of the warp after the box warps)
    for (int vb = warp * 4; vb < V; vb += 4 * warps) {
        const int v = vb + (lane >> 3);
        TapBox b = group8_tap_box(s.gh + (v < V ? v : V - 1) * taps, taps);
        if ((lane & 7) == 0 && v < V) s.box[v] = b;
    }
    if (warp == ((V + 3) / 4) % warps) {
        float sum = 0.0f;
        if (lane < 3)
            sum = lane == 2 ? sequential_sum_unrolled(s.rr, 1, taps)
                            : sequential_sum_unrolled(reinterpret_cast<const float *>(s.wt) + lane, 2, taps);
        const float count = __shfl_sync(full, sum, 0), sum_r = __shfl_sync(full, sum, 1);
        const float sum_rr = __shfl_sync(full, sum, 2);
        if (lane == 0) {
            patch.count = count;
            patch.sum_r = sum_r;
            patch.sum_rr = sum_rr;
            patch.ref_energy = sum_rr - sum_r * sum_r / count;
            patch.centre = centre;
            patch.ok = centre_ok && all_sampled;
        }
    }
    __syncthreads();

    // ---- which items are scored, and on which path; then list them: fast ones from the
    // front, exact ones from the back. A warp reserves its chunk's places at either end with
    // one shared atomic add each; the order of the list only decides which thread scores
    // which item (each score is computed alone into its own slot), so it does not change
    // a result.
    const bool patch_ok = patch.ok;
    unsigned taps_bad = 0u;
    for (int w = 0; w < warps; ++w) taps_bad |= warp_undefined[w];
    const unsigned below = (1u << lane) - 1u;
    for (int c = 0; c < chunks; ++c) {
        const int item = c * T + tid;
        bool scored = false, fast = false;
        if (item < total) {
            const int v = by_slots.quotient(item);
            const double2 dd = s.disp[item];
            scored = !(dd.x != dd.x) && patch_ok && !((taps_bad >> v) & 1u);
            if (scored) {
                const PlaneRef &plane = p.views[p.targets[v]].luma;
                fast = taps_inside(s.box[v], dd.x * 0.5, dd.y * 0.5, plane.width, plane.height);
            } else {
                s.score[item] = NAN;
            }
        }
        const unsigned fast_mask = __ballot_sync(full, scored && fast);
        const unsigned exact_mask = __ballot_sync(full, scored && !fast);
        int fast_at = 0, exact_at = 0;
        if (lane == 0) {
            if (fast_mask) fast_at = atomicAdd(&list_ends[0], __popc(fast_mask));
            if (exact_mask) exact_at = atomicAdd(&list_ends[1], __popc(exact_mask));
        }
        fast_at = __shfl_sync(full, fast_at, 0);
        exact_at = __shfl_sync(full, exact_at, 0);
        if (scored && fast) s.list[fast_at + __popc(fast_mask & below)] = (unsigned short)item;
        if (scored && !fast) s.list[total - 1 - (exact_at + __popc(exact_mask & below))] = (unsigned short)item;
    }
    __syncthreads();
    const int n_fast = list_ends[0], n_exact = list_ends[1];

    // ---- the correlations of the listed items; an item's path is known from its place
    const int listed = n_fast + n_exact;
    for (int j = tid; j < listed; j += T) {
        const bool fast = j < n_fast;
        const int item = s.list[fast ? j : total - 1 - (j - n_fast)];
        const int v = by_slots.quotient(item);
        const DevView &tv = p.views[p.targets[v]];
        const double2 dd = s.disp[item];
        float score;
        bool ok;
        if (fast)
            score = zncc_inside(tv.quads, quad_pair_stride(tv.luma.width), s.gh + v * taps, s.wt, patch, taps,
                                dd.x * 0.5, dd.y * 0.5, ok);
        else
            ok = zncc_score(tv.luma, s.gh + v * taps, s.wt, patch, taps, dd.x, dd.y, score);
        s.score[item] = ok ? score : NAN;
    }
    __syncthreads();

    // ---- aggregate the views per label and price the label (depth.rs:1233-1246)
    int any_finite = 0;
    for (int slot = tid; slot < D; slot += T) {
        const int label = cost_slot_label(p, node, slot);
        float agg = 0.0f;
        bool some;
        if (V <= 4) {  // the views' scores in registers (V is the same for the whole launch)
            some = aggregate_small<4>(s.score + slot, D, V, p.minimum_support, p.best_view_count, agg);
        } else if (V <= 8) {
            some = aggregate_small<8>(s.score + slot, D, V, p.minimum_support, p.best_view_count, agg);
        } else {
            float sc[MAX_VIEWS];
            for (int v = 0; v < V; ++v) sc[v] = s.score[v * D + slot];
            some = aggregate_scores(sc, V, p.minimum_support, p.best_view_count, agg);
        }
        float score = some ? agg : NAN;
        float cost;
        if (isfinite(score)) {
            any_finite = 1;
            float near_prior =
                label == 0 ? 0.0f : NEAR_DEPTH_PRIOR * (float)(label - 1) / (float)(full_labels - 2);
            cost = clampf_r(1.0f - score, 0.0f, 2.0f) + near_prior;
        } else {
            cost = MISSING_COST;
        }
        size_t o = (size_t)out_row * D + slot;
        p.scores[o] = score;
        p.costs[o] = cost;
    }
    const bool tested = __syncthreads_or(any_finite);
    if (tid == 0) {
        p.tested[out_row] = tested;
        p.guidance[out_row] = patch.centre;  // reference_guidance (depth.rs:1824-1832)
    }
}

}  // namespace chiaro
