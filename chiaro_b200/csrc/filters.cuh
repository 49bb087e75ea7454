// filters.cuh — consistency filters on the direct field:
// reject_isolated_direct_depths (crates/chiaro-fusion/src/depth.rs:881-924),
// reject_small_direct_components (depth.rs:933-989) and
// fit_local_depth_planes (depth.rs:995-1060).
//
// Each filter reads an unmodified copy of the field, as the reference does.
// The component filter's depth-first search only ever discovers the connected
// component of its seed (its neighbour relation is symmetric), so a GPU
// union-find over the same edges yields the same components: nodes whose
// component has fewer than the minimum number of nodes are removed.
#pragma once

#include "select.cuh"

namespace chiaro {

__global__ void reject_isolated_kernel(const uint8_t *__restrict__ src_has, const double *__restrict__ depth,
                                       const float *__restrict__ confidence, const float *__restrict__ guidance,
                                       uint8_t *dst_has, int columns, int rows, double tolerance) {
    int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= columns * rows) return;
    if (!src_has[index]) {
        dst_has[index] = 0;
        return;
    }
    int column = index % columns, row = index / columns;
    double inverse = 1.0 / depth[index];
    int agreeing = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int x = column + dx, y = row + dy;
            if (x < 0 || y < 0 || x >= columns || y >= rows) continue;
            int ni = y * columns + x;
            if (!src_has[ni]) continue;
            float image_edge = fabsf(guidance[index] - guidance[ni]);
            if (image_edge <= 0.6f && fabs(1.0 / depth[ni] - inverse) <= tolerance) ++agreeing;
        }
    int minimum = confidence[index] >= 0.75f ? 1 : 2;
    dst_has[index] = agreeing < minimum ? 0 : 1;
}

// ---- connected components ------------------------------------------------------
// uf_find follows parent links to the root with path halving (benign races: any
// ancestor is a valid parent). With through_l2, parent[] is read through L2 (__ldcg),
// where the atomicCAS of uf_union resolves, so a thread never retries a join on a
// stale L1 copy of a root it has just lost; a first attempt reads normally.
template <bool through_l2>
__device__ inline int uf_find(int *parent, int x) {
    int p = through_l2 ? __ldcg(parent + x) : parent[x];
    while (p != x) {
        int gp = through_l2 ? __ldcg(parent + p) : parent[p];
        if (gp != p) parent[x] = gp;
        x = p;
        p = gp;
    }
    return x;
}

// Bit set in the status word when a union gave up (UNION_GAVE_UP): the host turns it
// into CHIARO_ERR_TIMEOUT instead of returning components with an edge left out.
constexpr int UNION_GAVE_UP = 1;

// Lock-free union. A failed compare-and-swap means another thread attached root b (at
// most n - 1 attachments happen in all) or, on the first attempt only, that its reads
// were stale (retries read through L2). With retries >= n + 1 the loop therefore always
// ends by joining or finding a == b; a smaller bound (a caller's choice) can run out,
// which is reported, never silent.
__device__ inline void uf_union(int *parent, int a, int b, int retries, int *status) {
    for (int attempt = 0; attempt < retries; ++attempt) {
        a = attempt ? uf_find<true>(parent, a) : uf_find<false>(parent, a);
        b = attempt ? uf_find<true>(parent, b) : uf_find<false>(parent, b);
        if (a == b) return;
        if (a > b) {
            int t = a;
            a = b;
            b = t;
        }
        // attach the larger root b under a; retry if b stopped being a root
        int old = atomicCAS(parent + b, b, a);
        if (old == b) return;
    }
    atomicOr(status, UNION_GAVE_UP);
}

__device__ inline bool component_edge(const uint8_t *has, const double *depth, const float *guidance, int i, int j,
                                      double tolerance) {
    if (!has[j]) return false;
    float image_edge = fabsf(guidance[i] - guidance[j]);
    double inverse_difference = fabs(1.0 / depth[j] - 1.0 / depth[i]);
    return image_edge <= 0.6f && inverse_difference <= tolerance;
}

__global__ void components_init_kernel(int *parent, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) parent[i] = i;
}

// Union each node with its east, south-west, south and south-east neighbours
// (together with the mirrored pairs this covers all eight directions).
__global__ void components_union_kernel(const uint8_t *__restrict__ has, const double *__restrict__ depth,
                                        const float *__restrict__ guidance, int *parent, int columns, int rows,
                                        double tolerance, int retries, int *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= columns * rows || !has[i]) return;
    int column = i % columns, row = i / columns;
    const int off[4][2] = {{1, 0}, {-1, 1}, {0, 1}, {1, 1}};
    for (int k = 0; k < 4; ++k) {
        int x = column + off[k][0], y = row + off[k][1];
        if (x < 0 || y < 0 || x >= columns || y >= rows) continue;
        int j = y * columns + x;
        if (component_edge(has, depth, guidance, i, j, tolerance)) uf_union(parent, i, j, retries, status);
    }
}

// Component sizes: the lanes of a warp that share a root add their count with one
// atomic (a large component would otherwise serialise one atomic per node on its root).
__global__ void components_size_kernel(const uint8_t *__restrict__ has, int *parent, int *size, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !has[i]) return;
    const unsigned active = __activemask();
    int root = uf_find<false>(parent, i);
    const unsigned peers = __match_any_sync(active, root);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(size + root, __popc(peers));
}

__global__ void components_mark_kernel(const uint8_t *__restrict__ src_has, int *parent, const int *__restrict__ size,
                                       uint8_t *dst_has, int n, int minimum_nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!src_has[i]) {
        dst_has[i] = 0;
        return;
    }
    dst_has[i] = size[uf_find<false>(parent, i)] < minimum_nodes ? 0 : 1;
}

// ---- local plane fit -------------------------------------------------------------
__global__ void fit_local_planes_kernel(const uint8_t *__restrict__ has, const double *__restrict__ src_depth,
                                        const float *__restrict__ confidence, const float *__restrict__ guidance,
                                        const double *__restrict__ spatial25, double *dst_depth, int columns,
                                        int rows, double tolerance) {
    int index = blockIdx.x * blockDim.x + threadIdx.x;
    if (index >= columns * rows) return;
    if (!has[index]) {
        dst_depth[index] = src_depth[index];
        return;
    }
    int column = index % columns, row = index / columns;
    double centre_inverse = 1.0 / src_depth[index];
    double n00 = 0, n01 = 0, n02 = 0, n10 = 0, n11 = 0, n12 = 0, n20 = 0, n21 = 0, n22 = 0;
    double r0 = 0, r1 = 0, r2 = 0;
    int support = 0;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            int x = column + dx, y = row + dy;
            if (x < 0 || y < 0 || x >= columns || y >= rows) continue;
            int ni = y * columns + x;
            if (!has[ni]) continue;
            double inverse = 1.0 / src_depth[ni];
            float image_edge = fabsf(guidance[index] - guidance[ni]);
            if (image_edge > 0.6f || fabs(inverse - centre_inverse) > tolerance) continue;
            double spatial = spatial25[(dy + 2) * 5 + (dx + 2)];
            double weight = (double)confidence[ni] * spatial * exp_f64(-2.5 * (double)image_edge);
            double b0 = 1.0, b1 = (double)dx, b2 = (double)dy;
            r0 += weight * b0 * inverse;
            n00 += weight * b0 * b0;
            n01 += weight * b0 * b1;
            n02 += weight * b0 * b2;
            r1 += weight * b1 * inverse;
            n10 += weight * b1 * b0;
            n11 += weight * b1 * b1;
            n12 += weight * b1 * b2;
            r2 += weight * b2 * inverse;
            n20 += weight * b2 * b0;
            n21 += weight * b2 * b1;
            n22 += weight * b2 * b2;
            ++support;
        }
    dst_depth[index] = src_depth[index];
    if (support < 6) return;
    // math::inverse (math.rs:70-95), first row only, then mul_vec(...)[0]
    double det = n00 * (n11 * n22 - n12 * n21) - n01 * (n10 * n22 - n12 * n20) + n02 * (n10 * n21 - n11 * n20);
    if (fabs(det) < 1e-300) return;
    double inv_det = 1.0 / det;
    double m0 = (n11 * n22 - n12 * n21) * inv_det;
    double m1 = -(n01 * n22 - n02 * n21) * inv_det;
    double m2 = (n01 * n12 - n02 * n11) * inv_det;
    double inverse = m0 * r0 + m1 * r1 + m2 * r2;
    if (!(isfinite(inverse) && inverse > 0.0)) return;
    double maximum_adjustment = tolerance * 0.25;
    inverse = clampd_r(inverse, centre_inverse - maximum_adjustment, centre_inverse + maximum_adjustment);
    dst_depth[index] = 1.0 / inverse;
}

}  // namespace chiaro
