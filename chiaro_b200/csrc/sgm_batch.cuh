// sgm_batch.cuh — many SGM instances (semi_global_costs, crates/chiaro-fusion/src/depth.rs:1279-1383)
// of different sizes and label counts in one persistent launch. The reference
// runs each reference/source grouping's SGM on its own; this is the batched
// form of the design.
//
// Every path of every direction of every instance is a task (instance, path).
// The host lists the tasks longest path first, so the long walks start early
// and the short ones fill the tail. A resident grid of warps pulls tasks from
// the list with one atomicAdd per task (lane 0, broadcast by shuffle) and walks
// each path with the same warp-per-path code as the single-instance SGM
// (sgm_walk_path, one step of prefetch: fewer registers, so more warps walk at once),
// writing that direction's path costs into the instance's path buffers. No warp waits on another: the ordered sum of the 8 path
// buffers, ((0 + L1) + L2) + ... + L8 per cell as the reference adds them,
// runs as a second kernel over all instances. An instance whose label count
// the launch was not built for sets the error word instead of being walked.
#pragma once

#include "sgm.cuh"

namespace chiaro {

struct SgmInstance {
    const float *costs;     // [N][D]
    const float *guidance;  // [N]
    float *paths;           // 8 path buffers of `pitch` floats
    float *out;             // [N][D]
    size_t pitch, cells;    // cells = N * D
    int columns, rows, labels, sets;  // sets = ceil(D / 32)
};

template <int KMAX>
__global__ void sgm_batch_paths_kernel(const SgmInstance *__restrict__ instances, const int2 *__restrict__ tasks,
                                       unsigned n_tasks, unsigned *next_task, int *error) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(next_task, 1u);
        t = __shfl_sync(full, t, 0);
        if (t >= n_tasks) return;  // whole warp
        const int2 task = tasks[t];
        const SgmInstance in = instances[task.x];
        switch (in.sets) {
#define SGM_BATCH_CASE(k)                                                                                    \
    case k:                                                                                                  \
        if (k <= KMAX)                                                                                       \
            sgm_walk_path<(k <= KMAX ? k : 1), 1>(in.costs, in.guidance, in.paths, in.pitch, in.columns, in.rows, \
                                              in.labels, task.y);                                           \
        else if (lane == 0)                                                                                  \
            atomicExch(error, 1);                                                                            \
        break;
            SGM_BATCH_CASE(1) SGM_BATCH_CASE(2) SGM_BATCH_CASE(3) SGM_BATCH_CASE(4)
            SGM_BATCH_CASE(5) SGM_BATCH_CASE(6) SGM_BATCH_CASE(7) SGM_BATCH_CASE(8)
#undef SGM_BATCH_CASE
            default:
                if (lane == 0) atomicExch(error, 1);
        }
    }
}

// out = ((0 + L1) + L2) + ... + L8 per cell of every instance, the reference's order.
__global__ void sgm_batch_sum_kernel(const SgmInstance *__restrict__ instances, int n_instances) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t start = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = 0; i < n_instances; ++i) {
        const SgmInstance in = instances[i];
        for (size_t c = start; c < in.cells; c += stride) {
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) s = s + __ldcs(in.paths + k * in.pitch + c);
            in.out[c] = s;
        }
    }
}

}  // namespace chiaro
