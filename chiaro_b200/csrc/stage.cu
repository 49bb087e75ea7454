// stage.cu — host side of the B200 depth stage and its C ABI.
//
// Orchestrates refine_multiview_depth (crates/chiaro-fusion/src/depth.rs:312-580)
// on one CUDA stream: cost volume -> eight-path SGM -> winner-take-all ->
// optional completion -> direct measurement -> consistency filters -> report
// statistics -> per-target decisions -> output warps and depth map. Every
// stage is a kernel; the host only validates, uploads, launches and reads
// the results back. There is no CPU fallback: a CUDA failure is reported as
// CHIARO_ERR_CUDA.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "cost.cuh"
#include "decisions.cuh"
#include "direct.cuh"
#include "filters.cuh"
#include "luminance.cuh"
#include "select.cuh"
#include "sgm.cuh"
#include "sgm_u16.cuh"
#include "sgm_batch.cuh"
#include "sgm_band.cuh"
#include "bandnet.cuh"
#include "resolution.cuh"
#include "align.cuh"
#include "consumers.cuh"
#include "coarse.cuh"

using namespace chiaro;

struct chiaro_depth_ctx {
    int device = 0;
    int sm_count = 1;
    cudaStream_t stream = nullptr;
    std::string error;
    struct Buffer {
        void *ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buffer> buffers;
    cudaEvent_t events[8] = {};
    cudaStream_t copy_stream = nullptr;  // host transfers that overlap the stage's kernels
    cudaEvent_t planes_ready = nullptr, map_ready = nullptr, ref_ready = nullptr;
    // batched SGM: the last captured graph and the tuned warps per CTA per size bucket
    uint64_t batch_key = 0;
    cudaGraphExec_t batch_exec = nullptr;
    std::map<uint64_t, int> batch_tuning;
    int batch_warps = 0, batch_waves = 0, batch_replayed = 0;
    int band_windows = 0;  // fallback windows of the last banded SGM
    // whole-stage graph of the device-buffer entry point (opt-in): the key of the last
    // call, the buffer-allocation epoch its pointers belong to, and the captured graph
    uint64_t alloc_epoch = 0;  // bumped by every (re)allocation of a cached buffer
    int stage_graph = 0;       // enabled by chiaro_depth_set_stage_graph
    std::string stage_key;     // key of the last device-buffer call
    uint64_t stage_key_epoch = 0;
    cudaGraphExec_t stage_exec = nullptr;
    int stage_graph_state = 0;  // last call: 0 launched, 1 captured, 2 replayed
    float timings[7] = {};
    int launches = 0;  // this library's kernel launches in the last stage call
    // bounds set by the caller: attempts of one union-find join (negative: the node count
    // plus one, which cannot run out) and the bytes the context's buffers may hold (0: no limit)
    int union_retries = -1;
    uint64_t memory_limit = 0;
    uint64_t memory_held = 0;
    // launch shapes chosen by the autotuner: cost-volume threads per node CTA per bucket;
    // autotune: 1 tune, 0 the default shape, or a forced shape (threads per node CTA)
    int autotune = 1;
    std::map<uint64_t, int> cost_tuning;
};

namespace {

struct CudaError {
    cudaError_t code;
    const char *what;
};

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) throw CudaError{e_, #call};         \
    } while (0)

// Grow-only named device buffer of at least `count` elements.
template <class T>
T *dbuf(chiaro_depth_ctx *ctx, const std::string &name, size_t count) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    auto &b = ctx->buffers[name];
    if (b.bytes < bytes) {
        if (ctx->memory_limit && ctx->memory_held - b.bytes + bytes > ctx->memory_limit)
            throw CudaError{cudaErrorMemoryAllocation, "a context buffer beyond the context's memory limit"};
        if (b.ptr) CK(cudaFree(b.ptr));
        ctx->memory_held -= b.bytes;
        b.ptr = nullptr;
        b.bytes = 0;
        CK(cudaMalloc(&b.ptr, bytes));
        b.bytes = bytes;
        ctx->memory_held += bytes;
        ++ctx->alloc_epoch;  // a captured stage graph holding the old pointer is void
    }
    return static_cast<T *>(b.ptr);
}

// Retry bound of the union-find joins for a grid of n nodes (see uf_union).
int union_retries(const chiaro_depth_ctx *ctx, size_t n) {
    if (ctx->union_retries >= 0) return ctx->union_retries;
    return (int)std::min<size_t>(n + 1, INT32_MAX);
}

int fail(chiaro_depth_ctx *ctx, const CudaError &e) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s", e.what, cudaGetErrorString(e.code));
    ctx->error = buf;
    cudaGetLastError();
    return CHIARO_ERR_CUDA;
}

size_t div_ceil(size_t a, size_t b) { return (a + b - 1) / b; }

bool options_valid(const chiaro_depth_options &o) {  // depth.rs:1879-1891
    return o.enabled && o.grid_step > 0 && std::isfinite(o.near_depth) && std::isfinite(o.far_depth) &&
           o.near_depth > 0.0 && o.far_depth > o.near_depth && o.planes >= 3 && o.patch_radius > 0 &&
           o.minimum_support > 0 && o.best_view_count >= o.minimum_support && o.minimum_neighbour_support > 0;
}

// inverse_depth_samples (depth.rs:1834-1843)
std::vector<double> inverse_depth_samples(double near_d, double far_d, size_t count) {
    double near_inverse = 1.0 / near_d, far_inverse = 1.0 / far_d;
    std::vector<double> out(count);
    for (size_t i = 0; i < count; ++i) {
        double weight = (double)i / (double)(count - 1);
        out[i] = 1.0 / (near_inverse * (1.0 - weight) + far_inverse * weight);
    }
    return out;
}

// Spatial weights exp(-d^2 / (2 sigma^2)), sigma = max(0.75 r, 1), in f32 with
// the platform expf exactly as warped_patch_zncc computes them (depth.rs:1777, 1805-1806).
std::vector<float> spatial_weights(int radius) {
    float sigma = std::fmax((float)radius * 0.75f, 1.0f);
    std::vector<float> w;
    for (int dy = -radius; dy <= radius; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
            float distance_sq = (float)(dx * dx + dy * dy);
            w.push_back(std::exp(-distance_sq / (2.0f * sigma * sigma)));
        }
    return w;
}

unsigned blocks_for(size_t n, unsigned threads) { return (unsigned)div_ceil(n, threads); }

// Warps per CTA (1..most) for a warp-per-node kernel with `slot_bytes` of
// dynamic shared memory per warp: the count that keeps the most warps resident.
template <typename Kernel>
int warps_per_cta(Kernel kernel, size_t slot_bytes, int most) {
    int best = 1, resident = 0;
    for (int k = most; k >= 1; --k) {
        int blocks = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, 32 * k, k * slot_bytes));
        if (blocks * k > resident) {
            resident = blocks * k;
            best = k;
        }
    }
    return best;
}

struct Grids {
    size_t coarse_step, coarse_columns, coarse_rows;
    size_t step, columns, rows;
};

Grids grids_for(size_t width, size_t height, const chiaro_depth_options &o) {
    Grids g;
    g.coarse_step = std::max<size_t>(o.grid_step, 4);
    g.coarse_columns = div_ceil(width, g.coarse_step) + 1;
    g.coarse_rows = div_ceil(height, g.coarse_step) + 1;
    g.step = std::max<size_t>(g.coarse_step / 2, 4);
    g.columns = div_ceil(width, g.step) + 1;
    g.rows = div_ceil(height, g.step) + 1;
    return g;
}

template <class T>
void upload(chiaro_depth_ctx *ctx, T *dst, const T *src, size_t count) {
    CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
}
template <class T>
void download(chiaro_depth_ctx *ctx, T *dst, const T *src, size_t count) {
    if (!dst) return;
    CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
}

// Opt the kernels that need more than 48 KiB of dynamic shared memory in, once per
// device (the attribute belongs to the current device's context).
void set_smem_limits() {
    static std::mutex lock;
    static std::vector<int> done_devices;
    int device = 0;
    CK(cudaGetDevice(&device));
    std::lock_guard<std::mutex> guard(lock);
    if (std::find(done_devices.begin(), done_devices.end(), device) != done_devices.end()) return;
    CK(cudaFuncSetAttribute(cost_volume_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(cost_volume_kernel<96>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(cost_volume_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(cost_volume_kernel<160>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(cost_volume_kernel<192>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(direct_depth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(direct_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(target_decision_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(target_decision_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    CK(cudaFuncSetAttribute(align_match_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    done_devices.push_back(device);
}

// ---- cost-volume launch shapes (the autotuner) -----------------------------------------
typedef void (*CostKernel)(CostParams);

CostKernel cost_kernel_for(int threads) {
    switch (threads) {
        case 64: return cost_volume_kernel<64>;
        case 96: return cost_volume_kernel<96>;
        case 160: return cost_volume_kernel<160>;
        case 192: return cost_volume_kernel<192>;
        default: return cost_volume_kernel<128>;
    }
}

// Launch build_cost_volume over n_rows node CTAs. With autotuning on, the first launch of a
// (targets, labels scored, radius) bucket large enough to time (at least 4096 nodes, outside
// any stream capture) runs every shape twice and keeps the fastest second run for the
// context's later launches; every shape writes the same bits, and the last launch below
// writes the outputs again.
void launch_cost(chiaro_depth_ctx *ctx, const CostParams &p, size_t n_rows, size_t smem) {
    cudaStream_t s = ctx->stream;
    const uint64_t key = ((uint64_t)p.n_targets << 24) | ((uint64_t)p.slots << 8) | (uint64_t)p.radius;
    int threads = ctx->autotune > 1 ? ctx->autotune : COST_THREADS;
    auto it = ctx->cost_tuning.find(key);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &capture));
    if (ctx->autotune > 1) {
        // a forced shape
    } else if (it != ctx->cost_tuning.end()) {
        threads = it->second;
    } else if (ctx->autotune == 1 && n_rows >= 4096 && capture == cudaStreamCaptureStatusNone) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = INFINITY;
        for (int t : COST_SHAPES) {
            float ms = 0.0f;
            for (int rep = 0; rep < 2; ++rep) {
                CK(cudaEventRecord(e0, s));
                cost_kernel_for(t)<<<(unsigned)n_rows, t, smem, s>>>(p);
                CK(cudaGetLastError());
                CK(cudaEventRecord(e1, s));
                CK(cudaEventSynchronize(e1));
                CK(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (ms < best) {
                best = ms;
                threads = t;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ctx->cost_tuning[key] = threads;
    }
    cost_kernel_for(threads)<<<(unsigned)n_rows, threads, smem, s>>>(p);
    CK(cudaGetLastError());
}

// Per (node, target) geometry records of a step-spaced grid.
void launch_geometry(chiaro_depth_ctx *ctx, const DevView *d_views, int reference, const std::vector<int> &targets,
                     size_t columns, size_t rows, size_t step, GeomRec *out) {
    if (targets.empty()) return;
    GeometryParams p{};
    p.views = d_views;
    p.reference = reference;
    p.n_targets = (int)targets.size();
    for (size_t v = 0; v < targets.size(); ++v) p.targets[v] = targets[v];
    p.columns = (int)columns;
    p.rows = (int)rows;
    p.step = (int)step;
    p.out = out;
    view_geometry_kernel<<<blocks_for(columns * rows * targets.size(), 128), 128, 0, ctx->stream>>>(p);
    CK(cudaGetLastError());
}

// ---- SGM ---------------------------------------------------------------------------
template <int K>
void sgm_paths(chiaro_depth_ctx *ctx, const float *data, const float *guidance, float *paths, size_t pitch,
               int columns, int rows, int labels) {
    const size_t total_paths = sgm_total_paths(columns, rows);
    const unsigned blocks = (unsigned)div_ceil(total_paths, SGM_PATHS_PER_CTA);
    // more paths than the prefetching form keeps resident (six 4-warp CTAs per SM): the
    // resident form runs them all at once
    if (total_paths > (size_t)ctx->sm_count * 24)
        sgm_paths_resident_kernel<K><<<blocks, 32 * SGM_PATHS_PER_CTA, 0, ctx->stream>>>(
            data, guidance, paths, pitch, columns, rows, labels);
    else
        sgm_paths_kernel<K><<<blocks, 32 * SGM_PATHS_PER_CTA, 0, ctx->stream>>>(data, guidance, paths, pitch,
                                                                                columns, rows, labels);
    CK(cudaGetLastError());
}

// Every direction's path costs in one launch, then their ordered sum (sgm.cuh).
void launch_sgm(chiaro_depth_ctx *ctx, const float *data, const float *guidance, float *out, int columns, int rows,
                int labels) {
    const int K = (labels + 31) / 32;  // label sets per lane
    const size_t total = (size_t)columns * rows * labels;
    const size_t pitch = (total + 63) / 64 * 64;
    float *paths = dbuf<float>(ctx, "sgm_paths", 8 * pitch);
    switch (K) {
#define SGM_CASE(k)                                                         \
    case k:                                                                 \
        sgm_paths<k>(ctx, data, guidance, paths, pitch, columns, rows, labels); \
        break;
        SGM_CASE(1) SGM_CASE(2) SGM_CASE(3) SGM_CASE(4) SGM_CASE(5) SGM_CASE(6) SGM_CASE(7) SGM_CASE(8)
#undef SGM_CASE
        default: throw CudaError{cudaErrorInvalidValue, "labels exceed 256"};
    }
    const unsigned blocks = (unsigned)std::min<size_t>(div_ceil(total, 256), (size_t)ctx->sm_count * 16);
    sgm_sum_kernel<<<blocks, 256, 0, ctx->stream>>>(paths, pitch, total, out);
    CK(cudaGetLastError());
}

template <int K>
void sgm_u16_paths(chiaro_depth_ctx *ctx, const unsigned *data, const float *guidance, unsigned *aggregate,
                   int columns, int rows, int labels) {
    const unsigned blocks = (unsigned)div_ceil(sgm_total_paths(columns, rows), SGM_PATHS_PER_CTA);
    sgm_u16_paths_kernel<K><<<blocks, 32 * SGM_PATHS_PER_CTA, 0, ctx->stream>>>(data, guidance, aggregate, columns,
                                                                                rows, labels);
    CK(cudaGetLastError());
}

// The quantised SGM (sgm_u16.cuh): quantise (and clear the aggregate), every direction's
// paths adding into the one packed aggregate, then the unpacked aggregate and the winner.
void launch_sgm_u16(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, int columns, int rows,
                    int labels, uint16_t *aggregate, uint16_t *best) {
    const size_t nodes = (size_t)columns * rows, pairs = (size_t)(labels + 1) / 2;
    const size_t words = nodes * pairs;
    unsigned *quantised = dbuf<unsigned>(ctx, "sgm16.costs", words);
    unsigned *packed = dbuf<unsigned>(ctx, "sgm16.aggregate", words);
    const unsigned qblocks = (unsigned)std::min<size_t>(div_ceil(words, 256), (size_t)ctx->sm_count * 16);
    sgm_quantise_kernel<<<qblocks, 256, 0, ctx->stream>>>(costs, (int)nodes, labels, quantised, packed);
    CK(cudaGetLastError());
    switch ((int)((pairs + 31) / 32)) {
        case 1: sgm_u16_paths<1>(ctx, quantised, guidance, packed, columns, rows, labels); break;
        case 2: sgm_u16_paths<2>(ctx, quantised, guidance, packed, columns, rows, labels); break;
        case 3: sgm_u16_paths<3>(ctx, quantised, guidance, packed, columns, rows, labels); break;
        case 4: sgm_u16_paths<4>(ctx, quantised, guidance, packed, columns, rows, labels); break;
        default: throw CudaError{cudaErrorInvalidValue, "labels exceed 256"};
    }
    sgm_u16_select_kernel<<<(unsigned)div_ceil(nodes * 32, 256), 256, 0, ctx->stream>>>(packed, (int)nodes, labels,
                                                                                       aggregate, best);
    CK(cudaGetLastError());
}

// ---- batched SGM (sgm_batch.cuh) -------------------------------------------------------
struct BatchWave {
    size_t first, count;          // instances
    size_t task_offset, n_tasks;  // tasks
};

struct BatchPlan {
    std::vector<SgmInstance> descs;  // device path pointers filled in once the scratch is known
    std::vector<size_t> scratch_offset;
    std::vector<int2> tasks;
    std::vector<BatchWave> waves;
    size_t scratch_floats = 0;
    int kmax = 1;
    uint64_t key = 1469598103934665603ull;  // FNV-1a over the batch's description
};

void fnv(uint64_t &h, const void *data, size_t bytes) {
    const unsigned char *c = static_cast<const unsigned char *>(data);
    for (size_t i = 0; i < bytes; ++i) h = (h ^ c[i]) * 1099511628211ull;
}

// Waves under the scratch budget and each wave's tasks, longest path first
// (a counting sort on the path length).
int plan_batch(const chiaro_sgm_instance *in, size_t n, size_t budget_floats, BatchPlan &plan) {
    size_t wave_floats = 0;
    plan.waves.push_back({0, 0, 0, 0});
    for (size_t i = 0; i < n; ++i) {
        const chiaro_sgm_instance &x = in[i];
        if (!x.costs || !x.guidance || !x.out || x.columns < 1 || x.rows < 1 || x.labels < 1 ||
            x.labels > MAX_LABELS || x.columns * x.rows > (1u << 26))
            return CHIARO_ERR_ARGUMENT;
        SgmInstance d{};
        d.costs = x.costs;
        d.guidance = x.guidance;
        d.out = x.out;
        d.columns = (int)x.columns;
        d.rows = (int)x.rows;
        d.labels = (int)x.labels;
        d.sets = (int)((x.labels + 31) / 32);
        d.cells = (size_t)x.columns * x.rows * x.labels;
        d.pitch = (d.cells + 63) / 64 * 64;
        const size_t need = 8 * d.pitch;
        if (need > budget_floats) return CHIARO_ERR_CAPACITY;
        BatchWave &w = plan.waves.back();
        if (w.count > 0 && wave_floats + need > budget_floats) {
            plan.waves.push_back({i, 0, 0, 0});
            wave_floats = 0;
        }
        plan.scratch_offset.push_back(wave_floats);
        wave_floats += need;
        plan.scratch_floats = std::max(plan.scratch_floats, wave_floats);
        plan.waves.back().count += 1;
        plan.kmax = std::max(plan.kmax, d.sets);
        plan.descs.push_back(d);
        fnv(plan.key, &x, sizeof(x));
    }
    for (BatchWave &w : plan.waves) {
        int longest = 0;
        for (size_t i = w.first; i < w.first + w.count; ++i)
            longest = std::max({longest, plan.descs[i].columns, plan.descs[i].rows});
        std::vector<std::vector<int2>> by_length(longest + 1);
        for (size_t i = w.first; i < w.first + w.count; ++i) {
            const SgmInstance &d = plan.descs[i];
            const int paths = (int)sgm_total_paths(d.columns, d.rows);
            for (int k = 0; k < paths; ++k) {
                int pass, path, r0, c0, dr, dc, len;
                sgm_path_of(k, d.columns, d.rows, pass, path);
                sgm_path(pass >> 1, path, d.columns, d.rows, r0, c0, dr, dc, len);
                by_length[len].push_back(make_int2((int)i, k));
            }
        }
        w.task_offset = plan.tasks.size();
        for (int len = longest; len >= 0; --len)
            plan.tasks.insert(plan.tasks.end(), by_length[len].begin(), by_length[len].end());
        w.n_tasks = plan.tasks.size() - w.task_offset;
    }
    return CHIARO_OK;
}

// Device copies of a plan: descriptors (path pointers into the scratch), tasks,
// one task counter per wave and the error word.
struct BatchDevice {
    SgmInstance *descs;
    int2 *tasks;
    unsigned *counters;
    int *error;
    float *scratch;
};

template <int KMAX>
int batch_blocks_per_sm(int warps) {
    int blocks = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sgm_batch_paths_kernel<KMAX>, 32 * warps, 0));
    return std::max(blocks, 1);
}

template <int KMAX>
void enqueue_batch_kmax(chiaro_depth_ctx *ctx, const BatchPlan &plan, const BatchDevice &dev, int warps,
                        int blocks_per_sm) {
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(dev.error, 0, sizeof(int), s));
    CK(cudaMemsetAsync(dev.counters, 0, plan.waves.size() * sizeof(unsigned), s));
    const unsigned sum_blocks = (unsigned)ctx->sm_count * 16;
    for (size_t w = 0; w < plan.waves.size(); ++w) {
        const BatchWave &wave = plan.waves[w];
        if (wave.count == 0) continue;
        sgm_batch_paths_kernel<KMAX><<<(unsigned)(ctx->sm_count * blocks_per_sm), 32 * warps, 0, s>>>(
            dev.descs, dev.tasks + wave.task_offset, (unsigned)wave.n_tasks, dev.counters + w, dev.error);
        CK(cudaGetLastError());
        sgm_batch_sum_kernel<<<sum_blocks, 256, 0, s>>>(dev.descs + wave.first, (int)wave.count);
        CK(cudaGetLastError());
    }
}

// The launch's KMAX: the smallest of 2, 4 and 8 label sets that holds every instance.
int batch_kmax(int kmax) { return kmax <= 2 ? 2 : (kmax <= 4 ? 4 : 8); }

int batch_blocks(const BatchPlan &plan, int warps) {
    switch (batch_kmax(plan.kmax)) {
        case 2: return batch_blocks_per_sm<2>(warps);
        case 4: return batch_blocks_per_sm<4>(warps);
        default: return batch_blocks_per_sm<8>(warps);
    }
}

void enqueue_batch(chiaro_depth_ctx *ctx, const BatchPlan &plan, const BatchDevice &dev, int warps) {
    const int blocks = batch_blocks(plan, warps);
    switch (batch_kmax(plan.kmax)) {
        case 2: enqueue_batch_kmax<2>(ctx, plan, dev, warps, blocks); break;
        case 4: enqueue_batch_kmax<4>(ctx, plan, dev, warps, blocks); break;
        default: enqueue_batch_kmax<8>(ctx, plan, dev, warps, blocks); break;
    }
}

// Size bucket of the autotuner: the launch's KMAX and log2 of the cells per direction.
uint64_t batch_bucket(const BatchPlan &plan) {
    size_t cells = 0;
    for (const SgmInstance &d : plan.descs) cells += d.cells;
    int log2 = 0;
    while ((cells >> log2) > 1) ++log2;
    return (uint64_t)batch_kmax(plan.kmax) | ((uint64_t)log2 << 8);
}

int run_batch(chiaro_depth_ctx *ctx, const chiaro_sgm_instance *in, size_t n, size_t scratch_bytes, int flags) {
    uint64_t key = 1469598103934665603ull;
    fnv(key, in, n * sizeof(chiaro_sgm_instance));
    fnv(key, &scratch_bytes, sizeof(scratch_bytes));
    fnv(key, &flags, sizeof(flags));
    cudaStream_t s = ctx->stream;
    ctx->batch_replayed = 0;
    if ((flags & CHIARO_BATCH_GRAPH) && ctx->batch_exec && ctx->batch_key == key) {
        CK(cudaGraphLaunch(ctx->batch_exec, s));
        ctx->batch_replayed = 1;
    } else {
        ctx->batch_key = 0;  // any other batch may move the scratch: the cached graph is void
        BatchPlan plan;
        const size_t budget = scratch_bytes ? scratch_bytes : ((size_t)16 << 30);
        if (int st = plan_batch(in, n, budget / sizeof(float), plan)) return st;
        BatchDevice dev{};
        dev.scratch = dbuf<float>(ctx, "batch.paths", std::max<size_t>(plan.scratch_floats, 1));
        for (size_t i = 0; i < plan.descs.size(); ++i) plan.descs[i].paths = dev.scratch + plan.scratch_offset[i];
        dev.descs = dbuf<SgmInstance>(ctx, "batch.descs", plan.descs.size());
        dev.tasks = dbuf<int2>(ctx, "batch.tasks", std::max<size_t>(plan.tasks.size(), 1));
        dev.counters = dbuf<unsigned>(ctx, "batch.counters", plan.waves.size());
        dev.error = dbuf<int>(ctx, "batch.error", 1);
        upload(ctx, dev.descs, plan.descs.data(), plan.descs.size());
        upload(ctx, dev.tasks, plan.tasks.data(), plan.tasks.size());
        const uint64_t bucket = batch_bucket(plan);
        int warps = 4;
        auto tuned = ctx->batch_tuning.find(bucket);
        if (tuned != ctx->batch_tuning.end()) {
            warps = tuned->second;
        } else if (flags & CHIARO_BATCH_AUTOTUNE) {
            float best_ms = 0.0f;
            for (int candidate : {1, 2, 4, 8}) {
                enqueue_batch(ctx, plan, dev, candidate);  // warm
                CK(cudaEventRecord(ctx->events[0], s));
                enqueue_batch(ctx, plan, dev, candidate);
                CK(cudaEventRecord(ctx->events[1], s));
                CK(cudaEventSynchronize(ctx->events[1]));
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, ctx->events[0], ctx->events[1]));
                if (candidate == 1 || ms < best_ms) {
                    best_ms = ms;
                    warps = candidate;
                }
            }
            ctx->batch_tuning[bucket] = warps;
        }
        ctx->batch_warps = warps;
        ctx->batch_waves = (int)plan.waves.size();
        if (flags & CHIARO_BATCH_GRAPH) {
            batch_blocks(plan, warps);  // occupancy queried outside the capture
            if (ctx->batch_exec) {
                CK(cudaGraphExecDestroy(ctx->batch_exec));
                ctx->batch_exec = nullptr;
            }
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_batch(ctx, plan, dev, warps);
            } catch (const CudaError &) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            CK(cudaStreamEndCapture(s, &graph));
            cudaError_t e = cudaGraphInstantiate(&ctx->batch_exec, graph, 0);
            cudaGraphDestroy(graph);
            CK(e);
            CK(cudaGraphLaunch(ctx->batch_exec, s));
            ctx->batch_key = key;
        } else {
            enqueue_batch(ctx, plan, dev, warps);
        }
    }
    int error = 0;
    int *d_error = dbuf<int>(ctx, "batch.error", 1);
    CK(cudaMemcpyAsync(&error, d_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (error) throw CudaError{cudaErrorInvalidValue, "batched SGM: an instance's label count exceeds the launch"};
    return CHIARO_OK;
}

// ---- banded SGM with windowed fallback (sgm_band.cuh) ----------------------------------
// Fallback tiles as greedy rectangles in raster order (the widest run, then as many rows
// of it as are all flagged), each with its window of `margin` nodes around it; the
// windows' cost and node offsets pack them one after another ([cells][labels], [cells]).
// Where the windows would cover at least the grid, one window, the whole grid, decides
// every fallback tile instead. most = the largest rectangle's node count.
std::vector<BandWindow> fallback_windows(const std::vector<uint8_t> &flags, int tiles_x, int tiles_y, int tile,
                                         int columns, int rows, int margin, int labels, size_t &cost_floats,
                                         size_t &node_floats, int &most) {
    std::vector<BandWindow> windows;
    std::vector<uint8_t> taken(flags.size(), 0);
    auto open = [&](int x, int y) { return flags[y * tiles_x + x] && !taken[y * tiles_x + x]; };
    cost_floats = node_floats = 0;
    most = 0;
    for (int ty = 0; ty < tiles_y; ++ty)
        for (int tx = 0; tx < tiles_x; ++tx) {
            if (!open(tx, ty)) continue;
            int w = 1, h = 1;
            while (tx + w < tiles_x && open(tx + w, ty)) ++w;
            for (bool grow = true; grow && ty + h < tiles_y;) {
                for (int x = tx; x < tx + w; ++x) grow = grow && open(x, ty + h);
                if (grow) ++h;
            }
            for (int y = ty; y < ty + h; ++y)
                for (int x = tx; x < tx + w; ++x) taken[y * tiles_x + x] = 1;
            BandWindow win{};
            win.tc0 = tx * tile;
            win.tr0 = ty * tile;
            win.tc = std::min(columns, (tx + w) * tile) - win.tc0;
            win.tr = std::min(rows, (ty + h) * tile) - win.tr0;
            win.c0 = std::max(0, win.tc0 - margin);
            win.r0 = std::max(0, win.tr0 - margin);
            win.wc = std::min(columns, win.tc0 + win.tc + margin) - win.c0;
            win.wr = std::min(rows, win.tr0 + win.tr + margin) - win.r0;
            win.cost_offset = cost_floats;
            win.node_offset = node_floats;
            cost_floats += (size_t)win.wc * win.wr * labels;
            node_floats += (size_t)win.wc * win.wr;
            most = std::max(most, win.tc * win.tr);
            windows.push_back(win);
        }
    if (node_floats >= (size_t)columns * rows) {
        BandWindow whole{};
        whole.wc = whole.tc = columns;
        whole.wr = whole.tr = rows;
        windows.assign(1, whole);
        most = columns * rows;
        cost_floats = (size_t)columns * rows * labels;
        node_floats = (size_t)columns * rows;
    }
    return windows;
}

int run_band(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, int columns, int rows, int labels,
             const int *tile_offset, int tile, int band, int margin, int *winner, uint8_t *fallback) {
    cudaStream_t s = ctx->stream;
    const int tiles_x = (columns + tile - 1) / tile, tiles_y = (rows + tile - 1) / tile, tiles = tiles_x * tiles_y;
    int *bad = dbuf<int>(ctx, "band.bad", 1);
    CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
    band_check_kernel<<<(unsigned)div_ceil(tiles, 256), 256, 0, s>>>(tile_offset, tiles, labels, band, bad);
    CK(cudaGetLastError());
    int h_bad = 0;
    CK(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h_bad) return CHIARO_ERR_ARGUMENT;
    const BandGrid grid{tile_offset, tile, tiles_x, band};
    const size_t nodes = (size_t)columns * rows, pitch = (nodes * band + 63) / 64 * 64;
    float *paths = dbuf<float>(ctx, "band.paths", 8 * pitch);
    CK(cudaMemsetAsync(fallback, 0, tiles, s));
    sgm_band_paths_kernel<<<(unsigned)div_ceil(sgm_total_paths(columns, rows), SGM_PATHS_PER_CTA),
                            32 * SGM_PATHS_PER_CTA, 0, s>>>(costs, guidance, grid, paths, pitch, columns, rows, labels, 0);
    CK(cudaGetLastError());
    sgm_band_select_kernel<<<(unsigned)div_ceil(nodes * 32, 256), 256, 0, s>>>(paths, pitch, grid, columns, rows,
                                                                               labels, winner, fallback);
    CK(cudaGetLastError());
    std::vector<uint8_t> flags(tiles);
    CK(cudaMemcpyAsync(flags.data(), fallback, tiles, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    size_t cost_floats = 0, node_floats = 0;
    int most = 0;
    std::vector<BandWindow> windows =
        fallback_windows(flags, tiles_x, tiles_y, tile, columns, rows, margin, labels, cost_floats, node_floats, most);
    ctx->band_windows = (int)windows.size();
    if (!windows.empty()) {
        BandWindow *d_windows = dbuf<BandWindow>(ctx, "band.windows", windows.size());
        upload(ctx, d_windows, windows.data(), windows.size());
        float *wagg;
        if (windows.size() == 1 && windows[0].wc == columns && windows[0].wr == rows) {
            wagg = dbuf<float>(ctx, "band.wagg", nodes * labels);
            launch_sgm(ctx, costs, guidance, wagg, columns, rows, labels);
        } else {
            float *wcosts = dbuf<float>(ctx, "band.wcosts", cost_floats);
            float *wguid = dbuf<float>(ctx, "band.wguid", node_floats);
            wagg = dbuf<float>(ctx, "band.wagg", cost_floats);
            band_crop_kernel<<<dim3(64, (unsigned)windows.size()), 256, 0, s>>>(costs, guidance, columns, labels,
                                                                                 d_windows, wcosts, wguid);
            CK(cudaGetLastError());
            std::vector<chiaro_sgm_instance> instances(windows.size());
            for (size_t i = 0; i < windows.size(); ++i) {
                const BandWindow &w = windows[i];
                instances[i] = chiaro_sgm_instance{wcosts + w.cost_offset, wguid + w.node_offset,
                                                   wagg + w.cost_offset, (uint64_t)w.wc, (uint64_t)w.wr,
                                                   (uint64_t)labels};
            }
            if (int st = run_batch(ctx, instances.data(), instances.size(), 0, 0)) return st;
        }
        band_window_winner_kernel<<<dim3((unsigned)div_ceil((size_t)most * 32, 256), (unsigned)windows.size()), 256,
                                    0, s>>>(wagg, columns, labels, d_windows, grid, fallback, winner);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(s));
    return CHIARO_OK;
}

// ---- refine_resolution_warp (resolution.cuh; resolution.rs:232-439) -----------------
namespace resolution_host {

WarpRef host_warp(const chiaro_warp &w) {
    return WarpRef{reinterpret_cast<const float2 *>(w.points), (int)w.step, (int)w.columns, (int)w.rows};
}

// Rust's f32::clamp: NaN passes through.
float clamp_rust(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// Warp::confidence (align.rs:113-131).
float warp_confidence(const chiaro_warp &w, float x, float y) {
    const float fx = x / (float)w.step, fy = y / (float)w.step;
    if (fx < 0.0f || fy < 0.0f || !w.confidence) return 0.0f;
    const int c0 = sat_index(floorf(fx), (int)w.columns - 1), r0 = sat_index(floorf(fy), (int)w.rows - 1);
    const int c1 = std::min(c0 + 1, (int)w.columns - 1), r1 = std::min(r0 + 1, (int)w.rows - 1);
    const float tx = fx - (float)c0, ty = fy - (float)r0;
    auto value = [&](int c, int r) { return w.confidence[(size_t)r * w.columns + c]; };
    const float top = value(c0, r0) * (1.0f - tx) + value(c1, r0) * tx;
    const float bottom = value(c0, r1) * (1.0f - tx) + value(c1, r1) * tx;
    return clamp_rust(top * (1.0f - ty) + bottom * ty, 0.0f, 1.0f);
}

// Warp::magnification (align.rs:133-145); false for None.
bool warp_magnification(const chiaro_warp &w, float x, float y, float &out) {
    const WarpRef r = host_warp(w);
    const float h = (float)w.step;
    float ax, ay, bx, by, cx, cy;
    if (!warp_map(r, x, y, ax, ay) || !warp_map(r, x + h, y, bx, by) || !warp_map(r, x, y + h, cx, cy)) return false;
    const float dx = std::sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay)) / h;
    const float dy = std::sqrt((cx - ax) * (cx - ax) + (cy - ay) * (cy - ay)) / h;
    out = std::fmax(std::sqrt(dx * dy), 1.0e-6f);
    return true;
}

bool total_less(float a, float b) { return total_key(a) < total_key(b); }

float smoothstep(float v) {
    v = clamp_rust(v, 0.0f, 1.0f);
    return v * v * (3.0f - 2.0f * v);
}

struct Correction {
    bool some;
    float x, y;
};

// Up to nine values of a 3 x 3 neighbourhood, sorted in total order by insertion
// (equal keys are equal bit patterns, so the order among them does not matter).
struct Neighbours {
    float v[9];
    int n = 0;
    void push(float x) { v[n++] = x; }
    void sort() {
        for (int i = 1; i < n; ++i) {
            const float x = v[i];
            int j = i - 1;
            while (j >= 0 && total_less(x, v[j])) {
                v[j + 1] = v[j];
                --j;
            }
            v[j + 1] = x;
        }
    }
    float median() const { return v[n / 2]; }
};

}  // namespace resolution_host

// The device half (render, patch searches) and the host half (the control grid's
// median filter, hole completion and report) of refine_resolution_warp. The planes
// are device pointers; the warps and the report are host memory.
int run_resolution(chiaro_depth_ctx *ctx, const float *d_reference, int reference_width, int reference_height,
                   const float *d_target, int target_width, int target_height, const chiaro_warp &base, int width,
                   int height, chiaro_warp &out, chiaro_resolution_report &report) {
    using namespace resolution_host;
    cudaStream_t s = ctx->stream;
    const int columns = (width + RES_WARP_STEP - 1) / RES_WARP_STEP + 1;
    const int rows = (height + RES_WARP_STEP - 1) / RES_WARP_STEP + 1;
    const size_t n_nodes = (size_t)columns * rows;
    out.step = RES_WARP_STEP;
    out.columns = (uint64_t)columns;
    out.rows = (uint64_t)rows;
    if (out.capacity < n_nodes) return CHIARO_ERR_CAPACITY;
    // resolution.rs:239-253
    float magnification = 1.0f;
    if (!warp_magnification(base, (float)width * 0.5f, (float)height * 0.5f, magnification)) magnification = 1.0f;
    magnification = clamp_rust(magnification, 0.5f, 4.0f);
    const int radius = magnification > 1.35f ? RES_MAGNIFIED_RADIUS : RES_RADIUS;
    // base warp on the device
    const size_t base_nodes = (size_t)base.columns * base.rows;
    float2 *d_points = dbuf<float2>(ctx, "res.base", std::max<size_t>(base_nodes, 1));
    if (base_nodes) upload(ctx, d_points, reinterpret_cast<const float2 *>(base.points), base_nodes);
    const WarpRef dbase{d_points, (int)base.step, (int)base.columns, (int)base.rows};
    const size_t plane = (size_t)reference_width * reference_height;
    float *rendered = dbuf<float>(ctx, "res.rendered", std::max<size_t>(plane, 1));
    if (plane)
        resolution_render_kernel<<<(unsigned)std::min<size_t>(div_ceil(plane, 256), (size_t)ctx->sm_count * 16), 256,
                                   0, s>>>(PlaneRef{d_target, target_width, target_height}, dbase, magnification,
                                           reference_width, reference_height, rendered);
    CK(cudaGetLastError());
    ResolutionNode *d_nodes = dbuf<ResolutionNode>(ctx, "res.nodes", n_nodes);
    resolution_match_kernel<<<(unsigned)div_ceil(n_nodes * 32, 256), 256, 0, s>>>(
        PlaneRef{d_reference, reference_width, reference_height}, PlaneRef{rendered, reference_width, reference_height},
        columns, rows, width, height, radius, d_nodes);
    CK(cudaGetLastError());
    std::vector<ResolutionNode> measured(n_nodes);
    CK(cudaMemcpyAsync(measured.data(), d_nodes, n_nodes * sizeof(ResolutionNode), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));

    // resolution.rs:307-361: neighbourhood medians of the measured shifts
    const WarpRef hbase = host_warp(base);
    std::vector<float> confidence(n_nodes);
    std::vector<Correction> grid(n_nodes);
    std::vector<float> corrections;
    float confidence_sum = 0.0f;
    float *points = out.points;
    for (int row = 0; row < rows; ++row)
        for (int column = 0; column < columns; ++column) {
            const float rx = (float)(column * RES_WARP_STEP), ry = (float)(row * RES_WARP_STEP);
            const size_t index = (size_t)row * columns + column;
            bool refined = false;
            float qx = 0.0f, qy = 0.0f, local = 0.0f, median_x = 0.0f, median_y = 0.0f;
            if (measured[index].measured) {
                Neighbours xs, ys;
                for (int nr = std::max(row - 1, 0); nr <= std::min(row + 1, rows - 1); ++nr)
                    for (int nc = std::max(column - 1, 0); nc <= std::min(column + 1, columns - 1); ++nc) {
                        const ResolutionNode &m = measured[(size_t)nr * columns + nc];
                        if (m.measured) {
                            xs.push(m.shift_x);
                            ys.push(m.shift_y);
                        }
                    }
                if (xs.n >= 3) {
                    xs.sort();
                    ys.sort();
                    median_x = xs.median();
                    median_y = ys.median();
                    const ResolutionNode &c = measured[index];
                    if (!(std::hypot(c.shift_x - median_x, c.shift_y - median_y) > 1.5f) &&
                        warp_map(hbase, rx + median_x, ry + median_y, qx, qy)) {
                        const float score_confidence = smoothstep((c.score - RES_MINIMUM_SCORE) / 0.20f);
                        local = score_confidence * warp_confidence(base, rx, ry);
                        refined = true;
                    }
                }
            }
            if (refined) {
                points[2 * index] = qx;
                points[2 * index + 1] = qy;
                confidence[index] = local;
                grid[index] = Correction{true, median_x, median_y};
                corrections.push_back(std::hypot(median_x, median_y));
                confidence_sum += local;
            } else {
                float bx = NAN, by = NAN;
                if (!warp_map(hbase, rx, ry, bx, by)) bx = by = NAN;
                points[2 * index] = bx;
                points[2 * index + 1] = by;
                confidence[index] = 0.0f;
                grid[index] = Correction{false, 0.0f, 0.0f};
            }
        }
    // resolution.rs:362-415: two passes completing short holes in a coherent correction field
    for (int pass = 0; pass < 2; ++pass) {
        const std::vector<Correction> grid_snapshot = grid;
        const std::vector<float> confidence_snapshot = confidence;
        for (int row = 0; row < rows; ++row)
            for (int column = 0; column < columns; ++column) {
                const size_t index = (size_t)row * columns + column;
                if (grid_snapshot[index].some) continue;
                Neighbours sx, sy;
                float neighbour_confidence = 0.0f;
                for (int nr = std::max(row - 1, 0); nr <= std::min(row + 1, rows - 1); ++nr)
                    for (int nc = std::max(column - 1, 0); nc <= std::min(column + 1, columns - 1); ++nc) {
                        const size_t neighbour = (size_t)nr * columns + nc;
                        if (grid_snapshot[neighbour].some) {
                            sx.push(grid_snapshot[neighbour].x);
                            sy.push(grid_snapshot[neighbour].y);
                            neighbour_confidence += confidence_snapshot[neighbour];
                        }
                    }
                if (sx.n < 3) continue;
                sx.sort();
                sy.sort();
                const float cx = sx.median(), cy = sy.median();
                // coherence over the sorted lists, pairing the k-th sorted x with the k-th sorted y
                bool coherent = true;
                for (int k = 0; k < sx.n && coherent; ++k)
                    coherent = std::hypot(sx.v[k] - cx, sy.v[k] - cy) <= 1.5f;
                if (!coherent) continue;
                const float rx = (float)(column * RES_WARP_STEP), ry = (float)(row * RES_WARP_STEP);
                float qx, qy;
                if (warp_map(hbase, rx + cx, ry + cy, qx, qy)) {
                    points[2 * index] = qx;
                    points[2 * index + 1] = qy;
                    confidence[index] = 0.45f * neighbour_confidence / (float)sx.n;
                    grid[index] = Correction{true, cx, cy};
                }
            }
    }
    std::sort(corrections.begin(), corrections.end(), total_less);
    const size_t verified = corrections.size();
    size_t supported = 0;
    for (float c : confidence) supported += c > 0.0f;
    if (out.confidence) std::copy(confidence.begin(), confidence.end(), out.confidence);
    const float cells = (float)std::max<size_t>(n_nodes, 1);
    report.verified_fraction = (float)verified / cells;
    report.supported_fraction = (float)supported / cells;
    report.median_correction_px = verified ? corrections[verified / 2] : 0.0f;
    report.mean_confidence = confidence_sum / (float)std::max<size_t>(verified, 1);
    return CHIARO_OK;
}

// ---- align_module (align.cuh, align_run.cuh; align.rs:281-830) -----------------------
#include "align_run.cuh"

// ---- learned band network (bandnet.cuh) ----------------------------------------------
struct NetState {
    __nv_bfloat16 *w, *wt;             // packed weights and their transposed, mirrored copy
    __nv_bfloat16 *act[NET_LAYERS + 1];  // act[0] = features, act[l + 1] = output of layer l
    __nv_bfloat16 *grad_a, *grad_b;    // pre-activation gradients, ping-pong
    float *y;                          // channel 0 of the last layer, fp32
    int *status;                       // NET_TC_GAVE_UP when a convolution's bounded wait ran out
    long pixels;
    int images, height, width;
};

NetState net_state(chiaro_depth_ctx *ctx, int images, int height, int width) {
    NetState s{};
    s.images = images;
    s.height = height;
    s.width = width;
    s.pixels = (long)images * height * width;
    const size_t act = (size_t)s.pixels * NET_CH;
    s.w = dbuf<__nv_bfloat16>(ctx, "net.w", (size_t)NET_LAYERS * NET_W);
    s.wt = dbuf<__nv_bfloat16>(ctx, "net.wt", (size_t)NET_LAYERS * NET_W);
    for (int l = 0; l <= NET_LAYERS; ++l) s.act[l] = dbuf<__nv_bfloat16>(ctx, "net.act" + std::to_string(l), act);
    s.grad_a = dbuf<__nv_bfloat16>(ctx, "net.grad_a", act);
    s.grad_b = dbuf<__nv_bfloat16>(ctx, "net.grad_b", act);
    s.y = dbuf<float>(ctx, "net.y", (size_t)s.pixels);
    s.status = dbuf<int>(ctx, "net.status", 1);
    CK(cudaMemsetAsync(s.status, 0, sizeof(int), ctx->stream));
    return s;
}

// Features from full-volume rows (stride == labels) or the pre-pass's compact rows (stride 17).
void net_features(chiaro_depth_ctx *ctx, const NetState &s, const float *costs, const float *guidance, int labels,
                  int stride) {
    const int nodes = (int)s.pixels;
    net_features_kernel<<<(unsigned)div_ceil((size_t)nodes * 32, 256), 256, 0, ctx->stream>>>(costs, stride, guidance,
                                                                                               nodes, labels, s.act[0]);
    CK(cudaGetLastError());
}

// Persistent grid of the tensor-core convolution: four CTAs per SM (44.5 KB of shared memory
// and 32 tensor-memory columns each), or one per 128-pixel tile when there are fewer tiles.
unsigned net_conv_tc_blocks(chiaro_depth_ctx *ctx, const NetState &s) {
    const long tiles = (long)s.images * s.height * ((s.width + NET_TC_M - 1) / NET_TC_M);
    return (unsigned)std::max<long>(1, std::min<long>(tiles, (long)ctx->sm_count * 4));
}

// A convolution of the band network: tcgen05 tiles (bandnet.cuh).
void net_conv(chiaro_depth_ctx *ctx, const NetState &s, const __nv_bfloat16 *in, const __nv_bfloat16 *w,
              const float *bias, int relu, const __nv_bfloat16 *mask, __nv_bfloat16 *out, float *out_f32) {
    net_conv_tc_kernel<<<net_conv_tc_blocks(ctx, s), NET_TC_M, NET_TC_SMEM, ctx->stream>>>(
        in, s.images, s.height, s.width, w, bias, relu, mask, out, out_f32, s.status);
    CK(cudaGetLastError());
}

// The status word of the network's convolutions after the call's work (synchronises).
int net_status(chiaro_depth_ctx *ctx, const NetState &s) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, s.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h & NET_TC_GAVE_UP) {
        ctx->error = "band network: a tensor-core convolution's wait for its MMAs ran out";
        return CHIARO_ERR_TIMEOUT;
    }
    return CHIARO_OK;
}

void net_forward(chiaro_depth_ctx *ctx, const NetState &s, const float *params) {
    cudaStream_t st = ctx->stream;
    net_pack_kernel<<<(unsigned)div_ceil((size_t)NET_LAYERS * NET_W, 256), 256, 0, st>>>(params, s.w, s.wt);
    CK(cudaGetLastError());
    for (int l = 0; l < NET_LAYERS; ++l) {
        const bool last = l + 1 == NET_LAYERS;
        net_conv(ctx, s, s.act[l], s.w + (size_t)l * NET_W, params + (size_t)l * (NET_W + NET_CH) + NET_W,
                 last ? 0 : 1, nullptr, s.act[l + 1], last ? s.y : nullptr);
    }
}

// One forward and backward over the batch: grads (fp32, the parameters' layout)
// and the loss added into *loss_sum (device).
void net_backward(chiaro_depth_ctx *ctx, const NetState &s, const float *params, const float *targets,
                  const uint8_t *mask, float inverse_count, float *grads, float *loss_sum) {
    cudaStream_t st = ctx->stream;
    net_forward(ctx, s, params);
    CK(cudaMemsetAsync(grads, 0, sizeof(float) * NET_PARAMS, st));
    const unsigned eblocks = (unsigned)std::min<size_t>(div_ceil((size_t)s.pixels, 256), (size_t)ctx->sm_count * 8);
    net_loss_kernel<<<eblocks, 256, 0, st>>>(s.y, targets, mask, s.pixels, inverse_count, 0.02f, s.grad_a, loss_sum);
    CK(cudaGetLastError());
    const long chunks = (s.pixels + 16L * NET_WGRAD_STEPS - 1) / (16L * NET_WGRAD_STEPS);
    const unsigned wblocks = (unsigned)div_ceil((size_t)chunks * NET_TAPS, 4);
    __nv_bfloat16 *dpre = s.grad_a, *dnext = s.grad_b;
    for (int l = NET_LAYERS - 1; l >= 0; --l) {
        float *g = grads + (size_t)l * (NET_W + NET_CH);
        net_wgrad_kernel<<<wblocks, 128, 0, st>>>(s.act[l], dpre, s.images, s.height, s.width, g);
        net_bias_grad_kernel<<<(unsigned)ctx->sm_count * 4, 256, 0, st>>>(dpre, s.pixels, g + NET_W);
        CK(cudaGetLastError());
        if (l > 0) {  // gradient at the previous layer's output, masked by its ReLU
            net_conv(ctx, s, dpre, s.wt + (size_t)l * NET_W, nullptr, 0, s.act[l], dnext, nullptr);
            std::swap(dpre, dnext);
        }
    }
}

// Normalised targets (label - 1) / (labels - 2) and the mask of scored nodes.
__global__ void net_targets_kernel(const int *__restrict__ winners, long pixels, int labels, float *targets) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < pixels) targets[p] = (float)(winners[p] - 1) / (float)(labels - 2);
}

// ---- the stage ------------------------------------------------------------------------
// ---- the coarse depth search (coarse.cuh): plain, or with the learned band -----------
struct BandSpec {
    const float *params;  // the network's parameters (device), or nullptr for the naive band
    int tile, band, margin;
    float fraction;  // cross-view fallback above this fraction of contradicted nodes (>= 1: off)
};

// The coarse grid's cost volume for `slots` labels per node (see CostParams), over all
// nodes or the `n_rows` nodes of node_list; rows [n_rows][slots].
struct CoarseGrid {
    std::vector<int> targets;
    int V, D, columns, rows, step;
    double *labels;
    float *spatial;
    GeomRec *geometry;
    TapLattice lattice;
    DevView *views;
};

void coarse_cost(chiaro_depth_ctx *ctx, const CoarseGrid &g, int reference, const chiaro_depth_options &o, int slots,
                 const int *label_list, const BandGrid *band, const int *node_list, size_t n_rows, float *scores,
                 float *costs, float *guidance, uint8_t *tested) {
    if (n_rows == 0) return;
    CostParams p{};
    p.geometry = g.geometry;
    p.views = g.views;
    p.reference = reference;
    p.n_targets = g.V;
    for (int v = 0; v < g.V; ++v) p.targets[v] = g.targets[v];
    p.columns = g.columns;
    p.rows = g.rows;
    p.step = g.step;
    p.labels = g.D;
    p.slots = slots;
    p.label_list = label_list;
    if (band) {
        p.band_first = band->tile_offset;
        p.band_tile = band->tile;
        p.band_tiles_x = band->tiles_x;
    }
    p.node_list = node_list;
    p.label_depth = g.labels;
    p.spatial = g.spatial;
    p.radius = (int)o.patch_radius;
    p.lattice = g.lattice;
    p.minimum_support = (int)o.minimum_support;
    p.best_view_count = (int)std::min<uint64_t>(o.best_view_count, MAX_VIEWS);
    p.scores = scores;
    p.costs = costs;
    p.guidance = guidance;
    p.tested = tested;
    const int taps = (2 * p.radius + 1) * (2 * p.radius + 1);
    const size_t smem = node_smem_bytes(g.V, taps, slots);
    if ((size_t)g.V * slots > 65535 || smem > 200 * 1024)
        throw CudaError{cudaErrorInvalidValue, "cost volume: targets x labels exceed the node CTA's shared memory"};
    launch_cost(ctx, p, n_rows, smem);
}

// The coarse search of the stage's reference grid (depth.rs:1187-1467 up to the winner):
// spec == nullptr runs the plain form (full cost volume, SGM, first minimum over labels
// 1..D-1, bit-identical to the stage's); otherwise the learned-band form (coarse.cuh).
// prepass_only stops after the pre-pass and writes its rows and guidance out.
int run_coarse(chiaro_depth_ctx *ctx, std::vector<DevView> h_views, int reference, const chiaro_depth_options &o,
               const BandSpec *spec, int *winner, uint8_t *tested_out, int *offsets_out, uint8_t *fallback_out,
               chiaro_band_report *report, float *prepass_out, float *guidance_out) {
    cudaStream_t s = ctx->stream;
    set_smem_limits();
    CoarseGrid g{};
    const int n_views = (int)h_views.size();
    for (int i = 0; i < n_views; ++i)
        if (i != reference && h_views[i].accepted && h_views[i].has_camera) g.targets.push_back(i);
    g.V = (int)g.targets.size();
    g.D = (int)o.planes + 1;
    g.step = (int)std::max<uint64_t>(o.grid_step, 4);
    g.columns = (int)div_ceil(h_views[reference].width, g.step) + 1;
    g.rows = (int)div_ceil(h_views[reference].height, g.step) + 1;
    const int D = g.D, radius = (int)o.patch_radius;
    const size_t N = (size_t)g.columns * g.rows;
    if (spec && (g.V < 1 || D < PREPASS_SLOTS + 2)) return CHIARO_ERR_ARGUMENT;
    auto finite_depths = inverse_depth_samples(o.near_depth, o.far_depth, o.planes);
    std::vector<double> labels(D);
    labels[0] = NAN;
    for (int l = 1; l < D; ++l) labels[l] = finite_depths[o.planes - l];
    auto sp = spatial_weights(radius);
    g.labels = dbuf<double>(ctx, "coarse.labels", D);
    g.spatial = dbuf<float>(ctx, "coarse.spatial", sp.size());
    upload(ctx, g.labels, labels.data(), D);
    upload(ctx, g.spatial, sp.data(), sp.size());
    for (int t : g.targets) {
        const PlaneRef &lp = h_views[t].luma;
        h_views[t].quads = dbuf<float4>(ctx, "quads" + std::to_string(t),
                                        (size_t)quad_pair_stride(lp.width) * ((lp.height + 1) / 2));
    }
    g.views = dbuf<DevView>(ctx, "coarse.views", n_views);
    upload(ctx, g.views, h_views.data(), n_views);
    g.geometry = dbuf<GeomRec>(ctx, "coarse_geometry", N * std::max(g.V, 1));
    if (g.V > 0 && g.step % 2 == 0) {
        g.lattice.margin = radius;
        g.lattice.columns = (int)((size_t)(g.columns - 1) * g.step / 2 + 2 * (size_t)radius + 1);
        g.lattice.rows = (int)((size_t)(g.rows - 1) * g.step / 2 + 2 * (size_t)radius + 1);
        g.lattice.planes = dbuf<float2>(ctx, "coarse.lattice", (size_t)(g.V + 1) * g.lattice.columns * g.lattice.rows);
    }
    CK(cudaEventRecord(ctx->events[0], s));
    launch_geometry(ctx, g.views, reference, g.targets, g.columns, g.rows, g.step, g.geometry);
    if (g.lattice.planes) {
        LatticeParams p{};
        p.views = g.views;
        p.reference = reference;
        p.n_targets = g.V;
        for (int v = 0; v < g.V; ++v) p.targets[v] = g.targets[v];
        p.columns = g.lattice.columns;
        p.rows = g.lattice.rows;
        p.margin = g.lattice.margin;
        p.out = const_cast<float2 *>(g.lattice.planes);
        tap_lattice_kernel<<<blocks_for((size_t)g.lattice.columns * g.lattice.rows, 256), 256, 0, s>>>(p);
        CK(cudaGetLastError());
    }
    for (int t : g.targets) {
        const PlaneRef &lp = h_views[t].luma;
        quad_plane_kernel<<<blocks_for((size_t)lp.width * lp.height, 256), 256, 0, s>>>(
            lp.data, lp.width, lp.height, quad_pair_stride(lp.width), const_cast<float4 *>(h_views[t].quads));
        CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ctx->events[1], s));
    uint8_t *tested = dbuf<uint8_t>(ctx, "coarse.tested", N);
    float *guidance = dbuf<float>(ctx, "coarse.guidance", N);
    chiaro_band_report rep{};
    if (!spec) {
        CK(cudaEventRecord(ctx->events[2], s));
        CK(cudaEventRecord(ctx->events[3], s));
        float *scores = dbuf<float>(ctx, "coarse.scores", N * D), *costs = dbuf<float>(ctx, "coarse.costs", N * D);
        CK(cudaMemsetAsync(tested, 0, N, s));
        coarse_cost(ctx, g, reference, o, D, nullptr, nullptr, nullptr, N, scores, costs, guidance, tested);
        CK(cudaEventRecord(ctx->events[4], s));
        float *aggregate = dbuf<float>(ctx, "coarse.aggregate", N * D);
        launch_sgm(ctx, costs, guidance, aggregate, g.columns, g.rows, D);
        aggregate_winner_kernel<<<(unsigned)div_ceil(N * 32, 256), 256, 0, s>>>(aggregate, (int)N, D, winner);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->events[5], s));
        CK(cudaEventRecord(ctx->events[6], s));
    } else {
        const int tile = spec->tile, band = spec->band;
        const int tiles_x = (g.columns + tile - 1) / tile, tiles_y = (g.rows + tile - 1) / tile;
        const int tiles = tiles_x * tiles_y;
        // pre-pass: label 0 and the 16 sampled labels
        std::vector<int> list(PREPASS_SLOTS, 0);
        for (int b = 0; b < NET_BINS; ++b) list[1 + b] = net_sample_label(b, D);
        int *d_list = dbuf<int>(ctx, "coarse.prepass_labels", PREPASS_SLOTS);
        upload(ctx, d_list, list.data(), PREPASS_SLOTS);
        float *pre_scores = dbuf<float>(ctx, "coarse.prepass_scores", N * PREPASS_SLOTS);
        float *pre_costs = dbuf<float>(ctx, "coarse.prepass_costs", N * PREPASS_SLOTS);
        CK(cudaMemsetAsync(tested, 0, N, s));
        coarse_cost(ctx, g, reference, o, PREPASS_SLOTS, d_list, nullptr, nullptr, N, pre_scores, pre_costs, guidance,
                    tested);
        CK(cudaEventRecord(ctx->events[2], s));
        if (prepass_out) {
            CK(cudaMemcpyAsync(prepass_out, pre_costs, N * PREPASS_SLOTS * sizeof(float), cudaMemcpyDeviceToDevice, s));
            if (guidance_out) CK(cudaMemcpyAsync(guidance_out, guidance, N * sizeof(float), cudaMemcpyDeviceToDevice, s));
            if (tested_out) CK(cudaMemcpyAsync(tested_out, tested, N, cudaMemcpyDeviceToDevice, s));
            CK(cudaStreamSynchronize(s));
            return CHIARO_OK;
        }
        // the band proposal: the network on the pre-pass's costs, or the naive band
        int *offsets = dbuf<int>(ctx, "coarse.band_offsets", tiles);
        int *net_status_word = nullptr;
        if (spec->params) {
            NetState ns = net_state(ctx, 1, g.rows, g.columns);
            net_features(ctx, ns, pre_costs, guidance, D, PREPASS_SLOTS);
            net_forward(ctx, ns, spec->params);
            net_tile_offsets_kernel<<<(unsigned)div_ceil(tiles, 128), 128, 0, s>>>(ns.y, g.columns, g.rows, D, tile,
                                                                                   band, offsets);
            net_status_word = ns.status;
        } else {
            naive_band_offsets_kernel<<<(unsigned)div_ceil(tiles, 128), 128, 0, s>>>(pre_costs, g.columns, g.rows, D,
                                                                                     tile, band, offsets);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->events[3], s));
        // the banded cost volume: label 0 and each tile's band
        const BandGrid grid{offsets, tile, tiles_x, band};
        float *band_scores = dbuf<float>(ctx, "coarse.band_scores", N * (1 + band));
        float *band_costs = dbuf<float>(ctx, "coarse.band_costs", N * (1 + band));
        uint8_t *band_tested = dbuf<uint8_t>(ctx, "coarse.band_tested", N);
        float *band_guidance = dbuf<float>(ctx, "coarse.band_guidance", N);
        CK(cudaMemsetAsync(band_tested, 0, N, s));
        coarse_cost(ctx, g, reference, o, 1 + band, nullptr, &grid, nullptr, N, band_scores, band_costs,
                    band_guidance, band_tested);
        CK(cudaEventRecord(ctx->events[4], s));
        // the banded SGM, its winners, the edge and cross-view fallback flags
        const size_t pitch = (N * band + 63) / 64 * 64;
        float *paths = dbuf<float>(ctx, "coarse.band_paths", 8 * pitch);
        uint8_t *fallback = dbuf<uint8_t>(ctx, "coarse.band_fallback", tiles);
        uint8_t *consistency = dbuf<uint8_t>(ctx, "coarse.band_consistency", tiles);
        uint8_t *edge = dbuf<uint8_t>(ctx, "coarse.band_edge", tiles);
        CK(cudaMemsetAsync(fallback, 0, tiles, s));
        CK(cudaMemsetAsync(consistency, 0, tiles, s));
        sgm_band_paths_kernel<<<(unsigned)div_ceil(sgm_total_paths(g.columns, g.rows), SGM_PATHS_PER_CTA),
                                32 * SGM_PATHS_PER_CTA, 0, s>>>(band_costs, guidance, grid, paths, pitch, g.columns,
                                                                g.rows, D, 1);
        CK(cudaGetLastError());
        sgm_band_select_kernel<<<(unsigned)div_ceil(N * 32, 256), 256, 0, s>>>(paths, pitch, grid, g.columns, g.rows,
                                                                               D, winner, fallback);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(edge, fallback, tiles, cudaMemcpyDeviceToDevice, s));
        if (spec->fraction < 1.0f) {
            band_consistency_kernel<<<(unsigned)div_ceil(tiles, 128), 128, 0, s>>>(
                band_scores, band_tested, winner, grid, g.columns, g.rows, spec->fraction, consistency, fallback);
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(ctx->events[5], s));
        std::vector<uint8_t> flags(tiles), edges(tiles), crossed(tiles);
        int net_word = 0;
        if (net_status_word) CK(cudaMemcpyAsync(&net_word, net_status_word, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(flags.data(), fallback, tiles, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(edges.data(), edge, tiles, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(crossed.data(), consistency, tiles, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (net_word & NET_TC_GAVE_UP) {
            ctx->error = "band network: a tensor-core convolution's wait for its MMAs ran out";
            return CHIARO_ERR_TIMEOUT;
        }
        size_t cost_floats = 0, node_count = 0;
        int most = 0;
        std::vector<BandWindow> windows = fallback_windows(flags, tiles_x, tiles_y, tile, g.columns, g.rows,
                                                           spec->margin, D, cost_floats, node_count, most);
        if (!windows.empty()) {
            // full-range costs of every window's nodes, window after window, in row-major order
            std::vector<int> nodes(node_count);
            for (const BandWindow &w : windows)
                for (int r = 0; r < w.wr; ++r)
                    for (int c = 0; c < w.wc; ++c)
                        nodes[w.node_offset + (size_t)r * w.wc + c] = (w.r0 + r) * g.columns + (w.c0 + c);
            int *d_nodes = dbuf<int>(ctx, "coarse.window_nodes", node_count);
            upload(ctx, d_nodes, nodes.data(), node_count);
            BandWindow *d_windows = dbuf<BandWindow>(ctx, "coarse.windows", windows.size());
            upload(ctx, d_windows, windows.data(), windows.size());
            float *wscores = dbuf<float>(ctx, "coarse.window_scores", cost_floats);
            float *wcosts = dbuf<float>(ctx, "coarse.window_costs", cost_floats);
            float *wguid = dbuf<float>(ctx, "coarse.window_guidance", node_count);
            uint8_t *wtested = dbuf<uint8_t>(ctx, "coarse.window_tested", node_count);
            float *wagg = dbuf<float>(ctx, "coarse.window_aggregate", cost_floats);
            coarse_cost(ctx, g, reference, o, D, nullptr, nullptr, d_nodes, node_count, wscores, wcosts, wguid,
                        wtested);
            if (windows.size() == 1 && windows[0].wc == g.columns && windows[0].wr == g.rows) {
                launch_sgm(ctx, wcosts, wguid, wagg, g.columns, g.rows, D);
            } else {
                std::vector<chiaro_sgm_instance> instances(windows.size());
                for (size_t i = 0; i < windows.size(); ++i) {
                    const BandWindow &w = windows[i];
                    instances[i] = chiaro_sgm_instance{wcosts + w.cost_offset, wguid + w.node_offset,
                                                       wagg + w.cost_offset, (uint64_t)w.wc, (uint64_t)w.wr,
                                                       (uint64_t)D};
                }
                if (int st = run_batch(ctx, instances.data(), instances.size(), 0, 0)) return st;
            }
            band_window_winner_kernel<<<dim3((unsigned)div_ceil((size_t)most * 32, 256), (unsigned)windows.size()),
                                        256, 0, s>>>(wagg, g.columns, D, d_windows, grid, fallback, winner);
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(ctx->events[6], s));
        for (int t = 0; t < tiles; ++t) {
            rep.edge_tiles += edges[t] != 0;
            rep.consistency_tiles += crossed[t] != 0;
            rep.fallback_tiles += flags[t] != 0;
        }
        rep.tiles = (uint64_t)tiles;
        rep.windows = windows.size();
        rep.window_nodes = node_count;
        if (offsets_out) CK(cudaMemcpyAsync(offsets_out, offsets, tiles * sizeof(int), cudaMemcpyDeviceToDevice, s));
        if (fallback_out) CK(cudaMemcpyAsync(fallback_out, fallback, tiles, cudaMemcpyDeviceToDevice, s));
    }
    if (tested_out) CK(cudaMemcpyAsync(tested_out, tested, N, cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < 6; ++i) CK(cudaEventElapsedTime(&rep.ms[i], ctx->events[i], ctx->events[i + 1]));
    CK(cudaEventElapsedTime(&rep.ms[6], ctx->events[0], ctx->events[6]));
    if (report) *report = rep;
    return CHIARO_OK;
}

struct StageOutputs {  // device pointers
    double *depth;
    float *confidence;
    uint8_t *provenance;
    float2 *points[MAX_VIEWS];
    float *warp_confidence[MAX_VIEWS];
};

// Host transfers of the host-buffer entry point, issued inside the stage so that
// they overlap its kernels: the luminance planes arrive on the copy stream while
// the geometry kernels run, and the depth map leaves on the copy stream while
// the per-target decisions run.
struct HostTransfers {
    struct Upload {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<Upload> planes;
    double *depth = nullptr;
    float *confidence = nullptr;
    uint8_t *provenance = nullptr;
    float2 *points[MAX_VIEWS] = {};
    float *warp_confidence[MAX_VIEWS] = {};
};

struct Results {  // read back once at the end
    int status;  // UNION_GAVE_UP when a component join ran out of retries
    unsigned long long tested, measured, regularized;
    unsigned long long target_counts[MAX_VIEWS][3];
    double median_depth;
    float median_improvement;
    int has_median_depth, has_median_improvement;
};

__global__ void field_stats_kernel(const uint8_t *__restrict__ tested, Field f, int n, Results *res, double *depth_keys,
                                   float *improvement_keys) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int t = 0, m = 0, r = 0;
    if (i < n) {
        t = tested[i];
        bool has = f.has[i];
        m = has && !f.regularized[i];
        r = has && f.regularized[i];
        depth_keys[i] = has ? f.depth[i] : INFINITY;
        improvement_keys[i] = m ? f.improvement[i] : INFINITY;
    }
    unsigned full = 0xffffffffu;
    int ct = __popc(__ballot_sync(full, t)), cm = __popc(__ballot_sync(full, m)), cr = __popc(__ballot_sync(full, r));
    if ((threadIdx.x & 31) == 0) {
        if (ct) atomicAdd(&res->tested, (unsigned long long)ct);
        if (cm) atomicAdd(&res->measured, (unsigned long long)cm);
        if (cr) atomicAdd(&res->regularized, (unsigned long long)cr);
    }
}

__global__ void medians_kernel(const double *sorted_depth, const float *sorted_improvement, Results *res) {
    unsigned long long nd = res->measured + res->regularized, ni = res->measured;
    res->has_median_depth = nd > 0;
    res->median_depth = nd > 0 ? sorted_depth[nd / 2] : 0.0;
    res->has_median_improvement = ni > 0;
    res->median_improvement = ni > 0 ? sorted_improvement[ni / 2] : 0.0f;
}

__global__ void depth_map_kernel(Field f, const uint8_t *__restrict__ tested, double *depth, float *confidence,
                                 uint8_t *provenance, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (f.has[i]) {
        depth[i] = f.depth[i];
        confidence[i] = f.confidence[i];
        provenance[i] = f.regularized[i] ? CHIARO_REGULARIZED : CHIARO_MEASURED;
    } else {
        depth[i] = NAN;
        confidence[i] = tested[i] ? 1.0f : 0.0f;
        provenance[i] = tested[i] ? CHIARO_GLOBAL : CHIARO_UNSUPPORTED;
    }
}

Field field_bufs(chiaro_depth_ctx *ctx, const std::string &name, size_t n) {
    Field f;
    f.has = dbuf<uint8_t>(ctx, name + ".has", n);
    f.depth = dbuf<double>(ctx, name + ".depth", n);
    f.confidence = dbuf<float>(ctx, name + ".confidence", n);
    f.improvement = dbuf<float>(ctx, name + ".improvement", n);
    f.regularized = dbuf<uint8_t>(ctx, name + ".regularized", n);
    return f;
}

void copy_field(chiaro_depth_ctx *ctx, const Field &dst, const Field &src, size_t n) {
    CK(cudaMemcpyAsync(dst.has, src.has, n, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.depth, src.depth, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.confidence, src.confidence, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.improvement, src.improvement, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.regularized, src.regularized, n, cudaMemcpyDeviceToDevice, ctx->stream));
}

Decisions decision_bufs(chiaro_depth_ctx *ctx, const std::string &name, size_t n) {
    Decisions d;
    d.kind = dbuf<uint8_t>(ctx, name + ".kind", n);
    d.global = dbuf<float2>(ctx, name + ".global", n);
    d.point = dbuf<float2>(ctx, name + ".point", n);
    d.confidence = dbuf<float>(ctx, name + ".confidence", n);
    d.measured = dbuf<uint8_t>(ctx, name + ".measured", n);
    return d;
}

void copy_decisions(chiaro_depth_ctx *ctx, const Decisions &dst, const Decisions &src, size_t n) {
    CK(cudaMemcpyAsync(dst.kind, src.kind, n, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.global, src.global, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.point, src.point, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.confidence, src.confidence, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dst.measured, src.measured, n, cudaMemcpyDeviceToDevice, ctx->stream));
}

void download_field(chiaro_depth_ctx *ctx, const Field &f, size_t n, uint8_t *has, double *depth, float *confidence,
                    float *improvement, uint8_t *regularized) {
    download(ctx, has, f.has, n);
    download(ctx, depth, f.depth, n);
    download(ctx, confidence, f.confidence, n);
    download(ctx, improvement, f.improvement, n);
    download(ctx, regularized, f.regularized, n);
}

// The whole-stage graph of the device-buffer entry point. A call's key holds what the
// captured launches depend on: every view's pointers, sizes, flags and camera, the
// reference, the options, the grids and the output pointers (the data behind the
// pointers may change: a replay reads it afresh). The first call with a key runs the
// stage (and allocates its buffers), the second captures it, later ones replay it;
// any (re)allocation of a cached buffer voids the graph.
template <class T>
void key_put(std::string &key, const T &v) {
    key.append(reinterpret_cast<const char *>(&v), sizeof(T));
}

std::string stage_key(const std::vector<DevView> &views, int reference, const chiaro_depth_options &o, const Grids &g,
                      const StageOutputs &out, const DevView *d_views, const Results *d_results) {
    std::string key;
    for (const DevView &v : views) {
        key_put(key, v.luma.data);
        key_put(key, v.luma.width);
        key_put(key, v.luma.height);
        key_put(key, v.warp.points);
        key_put(key, v.warp.step);
        key_put(key, v.warp.columns);
        key_put(key, v.warp.rows);
        key_put(key, v.width);
        key_put(key, v.height);
        key_put(key, v.has_camera);
        key_put(key, v.accepted);
        key_put(key, v.cam);  // doubles then four ints: no padding
    }
    key_put(key, reference);
    key_put(key, o.enabled);
    key_put(key, o.grid_step);
    key_put(key, o.near_depth);
    key_put(key, o.far_depth);
    key_put(key, o.planes);
    key_put(key, o.patch_radius);
    key_put(key, o.minimum_support);
    key_put(key, o.best_view_count);
    key_put(key, o.minimum_score);
    key_put(key, o.minimum_margin);
    key_put(key, o.minimum_improvement);
    key_put(key, o.minimum_neighbour_support);
    key_put(key, o.completion_iterations);
    key_put(key, g.coarse_step);
    key_put(key, g.coarse_columns);
    key_put(key, g.coarse_rows);
    key_put(key, g.step);
    key_put(key, g.columns);
    key_put(key, g.rows);
    key_put(key, out.depth);
    key_put(key, out.confidence);
    key_put(key, out.provenance);
    for (int t = 0; t < MAX_VIEWS; ++t) {
        key_put(key, out.points[t]);
        key_put(key, out.warp_confidence[t]);
    }
    key_put(key, d_views);
    key_put(key, d_results);
    return key;
}

// Ends a stream capture that an exception interrupted.
struct CaptureGuard {
    cudaStream_t stream = nullptr;
    bool active = false;
    ~CaptureGuard() {
        if (!active) return;
        cudaGraph_t graph = nullptr;
        cudaStreamEndCapture(stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
    }
};

// An event of the stage's timing; inside a capture an external record node, so that a
// replay records it too.
void record_event(cudaEvent_t event, cudaStream_t s, bool capturing) {
    if (capturing)
        CK(cudaEventRecordWithFlags(event, s, cudaEventRecordExternal));
    else
        CK(cudaEventRecord(event, s));
}

// Run the whole stage on device-resident views. h_views: the DevView array
// (device pointers inside), d_views: its device copy.
void run_stage(chiaro_depth_ctx *ctx, std::vector<DevView> h_views, DevView *d_views, int reference,
               const chiaro_depth_options &o, const Grids &g, const StageOutputs &out, Results *d_results,
               Results &h_results, const chiaro_depth_debug *debug, std::vector<int> &rewritten,
               const HostTransfers *host) {
    cudaStream_t s = ctx->stream;
    set_smem_limits();
    const int n_views = (int)h_views.size();
    std::vector<int> targets;
    for (int i = 0; i < n_views; ++i)
        if (i != reference && h_views[i].accepted && h_views[i].has_camera) targets.push_back(i);
    const int V = (int)targets.size();
    const int D = (int)o.planes + 1;
    const int radius = (int)o.patch_radius;
    const int direct_radius = std::max(radius, 3), wide_radius = std::max(2 * radius, 8);
    const size_t N = g.coarse_columns * g.coarse_rows, M = g.columns * g.rows;
    const double inverse_step = (1.0 / o.near_depth - 1.0 / o.far_depth) / (double)(o.planes - 1);

    // constant tables
    auto finite_depths = inverse_depth_samples(o.near_depth, o.far_depth, o.planes);
    std::vector<double> labels(D);
    labels[0] = NAN;
    for (int l = 1; l < D; ++l) labels[l] = finite_depths[o.planes - l];
    auto unseeded = inverse_depth_samples(o.near_depth, o.far_depth, 32);
    std::reverse(unseeded.begin(), unseeded.end());
    auto sp = spatial_weights(radius), sp_direct = spatial_weights(direct_radius),
         sp_wide = spatial_weights(wide_radius);
    std::vector<double> spatial25(25);
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) spatial25[(dy + 2) * 5 + dx + 2] = std::exp((double)(-(dx * dx + dy * dy)) / 6.0);
    double *d_labels = dbuf<double>(ctx, "labels", D);
    double *d_unseeded = dbuf<double>(ctx, "unseeded", 32);
    float *d_sp = dbuf<float>(ctx, "spatial", sp.size());
    float *d_sp_direct = dbuf<float>(ctx, "spatial_direct", sp_direct.size());
    float *d_sp_wide = dbuf<float>(ctx, "spatial_wide", sp_wide.size());
    double *d_sp25 = dbuf<double>(ctx, "spatial25", 25);
    upload(ctx, d_labels, labels.data(), D);
    upload(ctx, d_unseeded, unseeded.data(), 32);
    upload(ctx, d_sp, sp.data(), sp.size());
    upload(ctx, d_sp_direct, sp_direct.data(), sp_direct.size());
    upload(ctx, d_sp_wide, sp_wide.data(), sp_wide.size());
    upload(ctx, d_sp25, spatial25.data(), 25);
    // the quad planes' buffers and the views that point at them, before any launch
    for (int t : targets) {
        const PlaneRef &lp = h_views[t].luma;
        h_views[t].quads = dbuf<float4>(ctx, "quads" + std::to_string(t),
                                        (size_t)quad_pair_stride(lp.width) * ((lp.height + 1) / 2));
    }
    upload(ctx, d_views, h_views.data(), h_views.size());
    GeomRec *coarse_geometry = dbuf<GeomRec>(ctx, "coarse_geometry", N * std::max(V, 1));
    GeomRec *fine_geometry = dbuf<GeomRec>(ctx, "fine_geometry", M * std::max(V, 1));
    // the tap lattice of the grids with an even step (every tap of theirs is a lattice point)
    const bool coarse_lattice = V > 0 && g.coarse_step % 2 == 0, fine_lattice = V > 0 && g.step % 2 == 0;
    TapLattice lattice{};
    if (coarse_lattice || fine_lattice) {
        size_t extent_x = 0, extent_y = 0;
        if (coarse_lattice) {
            extent_x = (g.coarse_columns - 1) * g.coarse_step;
            extent_y = (g.coarse_rows - 1) * g.coarse_step;
        }
        if (fine_lattice) {
            extent_x = std::max(extent_x, (g.columns - 1) * g.step);
            extent_y = std::max(extent_y, (g.rows - 1) * g.step);
        }
        lattice.margin = std::max({radius, direct_radius, wide_radius});
        lattice.columns = (int)(extent_x / 2 + 2 * (size_t)lattice.margin + 1);
        lattice.rows = (int)(extent_y / 2 + 2 * (size_t)lattice.margin + 1);
        lattice.planes = dbuf<float2>(ctx, "tap_lattice", (size_t)(V + 1) * lattice.columns * lattice.rows);
    }
    // quad planes 1 per target, tap lattice 1, geometry 2, cost 1, SGM 2, select 1, completion, direct 2, filters 6, stats 2,
    // decisions 1 + 3 per target, map 1
    ctx->launches = V + (V > 0 ? 2 : 0) + (lattice.planes ? 1 : 0) + 1 + 2 + 1 + (int)o.completion_iterations + 3 + 6 +
                    2 + (V > 0 ? 1 + 3 * V : 0) + 1;
    // the whole-stage graph (device-buffer calls only)
    ctx->stage_graph_state = 0;
    bool capturing = false;
    CaptureGuard guard;
    if (ctx->stage_graph && !host && !debug) {
        const std::string key = stage_key(h_views, reference, o, g, out, d_views, d_results);
        const bool same = key == ctx->stage_key && ctx->alloc_epoch == ctx->stage_key_epoch;
        if (same && ctx->stage_exec) {
            CK(cudaGraphLaunch(ctx->stage_exec, s));
            ctx->stage_graph_state = 2;
            rewritten = targets;
            if (V == 0) rewritten.clear();
            CK(cudaMemcpyAsync(&h_results, d_results, sizeof(Results), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (int i = 0; i < 6; ++i) CK(cudaEventElapsedTime(&ctx->timings[i], ctx->events[i], ctx->events[i + 1]));
            CK(cudaEventElapsedTime(&ctx->timings[6], ctx->events[0], ctx->events[6]));
            return;
        }
        if (ctx->stage_exec) {
            CK(cudaGraphExecDestroy(ctx->stage_exec));
            ctx->stage_exec = nullptr;
        }
        capturing = same;  // the second call with this key: capture it
        ctx->stage_key = key;
    }
    if (capturing) {
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        guard.stream = s;
        guard.active = true;
    }
    CK(cudaMemsetAsync(d_results, 0, sizeof(Results), s));

    record_event(ctx->events[0], s, capturing);
    // per (node, target) geometry of both grids: cameras and warps only, so it runs
    // while the luminance planes are still arriving
    launch_geometry(ctx, d_views, reference, targets, g.coarse_columns, g.coarse_rows, g.coarse_step,
                    coarse_geometry);
    launch_geometry(ctx, d_views, reference, targets, g.columns, g.rows, g.step, fine_geometry);
    // the reference's plane goes up first: the tap lattice and the fine reference patches
    // need only it (and the warps), so they run while the targets' planes arrive
    const bool host_planes = host && !host->planes.empty();
    if (host_planes) {
        const auto &r = host->planes[(size_t)reference];
        CK(cudaMemcpyAsync(r.dst, r.src, r.bytes, cudaMemcpyHostToDevice, ctx->copy_stream));
        CK(cudaEventRecord(ctx->ref_ready, ctx->copy_stream));
        for (size_t i = 0; i < host->planes.size(); ++i) {
            if ((int)i == reference) continue;
            const auto &u = host->planes[i];
            CK(cudaMemcpyAsync(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice, ctx->copy_stream));
        }
        CK(cudaEventRecord(ctx->planes_ready, ctx->copy_stream));
        CK(cudaStreamWaitEvent(s, ctx->ref_ready, 0));
    }
    if (lattice.planes) {
        LatticeParams p{};
        p.views = d_views;
        p.reference = reference;
        p.n_targets = V;
        for (int v = 0; v < V; ++v) p.targets[v] = targets[v];
        p.columns = lattice.columns;
        p.rows = lattice.rows;
        p.margin = lattice.margin;
        p.out = const_cast<float2 *>(lattice.planes);
        tap_lattice_kernel<<<blocks_for((size_t)lattice.columns * lattice.rows, 256), 256, 0, s>>>(p);
        CK(cudaGetLastError());
    }
    // each fine node's reference patch at the direct radius, read by the direct pass and,
    // at the same radius, by the decisions
    RefPatch *fine_patches = dbuf<RefPatch>(ctx, "fine_patches", M);
    {
        PatchParams pp{};
        pp.views = d_views;
        pp.reference = reference;
        pp.columns = (int)g.columns;
        pp.rows = (int)g.rows;
        pp.step = (int)g.step;
        pp.radius = direct_radius;
        pp.spatial = d_sp_direct;
        if (fine_lattice) pp.lattice = lattice;
        pp.out = fine_patches;
        patch_sums_kernel<<<blocks_for(M, 256), 256, 0, s>>>(pp);
        CK(cudaGetLastError());
    }
    if (host_planes) CK(cudaStreamWaitEvent(s, ctx->planes_ready, 0));
    // quad planes of the target luminance for the fast ZNCC path
    for (int t : targets) {
        const PlaneRef &lp = h_views[t].luma;
        size_t n = (size_t)lp.width * lp.height;
        quad_plane_kernel<<<blocks_for(n, 256), 256, 0, s>>>(lp.data, lp.width, lp.height, quad_pair_stride(lp.width),
                                                             const_cast<float4 *>(h_views[t].quads));
        CK(cudaGetLastError());
    }
    // ---- cost volume
    float *scores = dbuf<float>(ctx, "scores", N * D);
    float *costs = dbuf<float>(ctx, "costs", N * D);
    float *guidance = dbuf<float>(ctx, "guidance", N);
    uint8_t *tested = dbuf<uint8_t>(ctx, "tested", N);
    CK(cudaMemsetAsync(tested, 0, N, s));  // the cost kernel only sets tested nodes
    {
        CostParams p{};
        p.geometry = coarse_geometry;
        p.views = d_views;
        p.reference = reference;
        p.n_targets = V;
        for (int v = 0; v < V; ++v) p.targets[v] = targets[v];
        p.columns = (int)g.coarse_columns;
        p.rows = (int)g.coarse_rows;
        p.step = (int)g.coarse_step;
        p.labels = D;
        p.slots = D;
        p.label_depth = d_labels;
        p.spatial = d_sp;
        p.radius = radius;
        if (coarse_lattice) p.lattice = lattice;
        p.minimum_support = (int)o.minimum_support;
        p.best_view_count = (int)std::min<uint64_t>(o.best_view_count, MAX_VIEWS);
        p.scores = scores;
        p.costs = costs;
        p.guidance = guidance;
        p.tested = tested;
        int taps = (2 * radius + 1) * (2 * radius + 1);
        const size_t smem = node_smem_bytes(V, taps, D);
        if ((size_t)V * D > 65535 || smem > 200 * 1024)
            throw CudaError{cudaErrorInvalidValue, "cost volume: targets x labels exceed the node CTA's shared memory"};
        launch_cost(ctx, p, N, smem);
    }
    record_event(ctx->events[1], s, capturing);
    // ---- SGM
    float *regularised = dbuf<float>(ctx, "regularised", N * D);
    launch_sgm(ctx, costs, guidance, regularised, (int)g.coarse_columns, (int)g.coarse_rows, D);
    record_event(ctx->events[2], s, capturing);
    // ---- select (+ completion)
    Field coarse = field_bufs(ctx, "coarse", N);
    uint8_t *fillable = dbuf<uint8_t>(ctx, "fillable", N);
    {
        SelectParams p{};
        p.scores = scores;
        p.regularised = regularised;
        p.tested = tested;
        p.label_depth = d_labels;
        p.nodes = (int)N;
        p.labels = D;
        p.minimum_score = o.minimum_score;
        p.minimum_margin = o.minimum_margin;
        p.minimum_improvement = o.minimum_improvement;
        p.field = coarse;
        p.fillable = fillable;
        select_depths_kernel<<<blocks_for(N * 32, 256), 256, 0, s>>>(p);
        CK(cudaGetLastError());
    }
    if (o.completion_iterations > 0) {
        Field other = field_bufs(ctx, "coarse2", N);
        Field src = coarse, dst = other;
        for (uint64_t it = 0; it < o.completion_iterations; ++it) {
            copy_field(ctx, dst, src, N);
            CompleteParams p{src, dst, guidance, fillable, (int)g.coarse_columns, (int)g.coarse_rows,
                             (int)o.minimum_neighbour_support};
            complete_depth_kernel<<<blocks_for(N, 256), 256, 0, s>>>(p);
            CK(cudaGetLastError());
            std::swap(src, dst);
        }
        if (src.has != coarse.has) copy_field(ctx, coarse, src, N);
    }
    if (debug) {
        download(ctx, debug->coarse_scores, scores, N * D);
        download(ctx, debug->coarse_costs, costs, N * D);
        download(ctx, debug->coarse_guidance, guidance, N);
        download(ctx, debug->coarse_tested, tested, N);
        download(ctx, debug->regularised, regularised, N * D);
        download_field(ctx, coarse, N, debug->coarse_has, debug->coarse_depth, debug->coarse_confidence,
                       debug->coarse_improvement, debug->coarse_regularized);
        download(ctx, debug->coarse_fillable, fillable, N);
    }
    record_event(ctx->events[3], s, capturing);
    // ---- direct measurement
    Field direct = field_bufs(ctx, "direct", M);
    float *fguidance = dbuf<float>(ctx, "fine_guidance", M);
    uint8_t *ftested = dbuf<uint8_t>(ctx, "fine_tested", M);
    {
        DirectParams p{};
        p.geometry = fine_geometry;
        if (fine_lattice) p.lattice = lattice;
        p.patches = fine_patches;
        p.views = d_views;
        p.reference = reference;
        p.n_targets = V;
        for (int v = 0; v < V; ++v) p.targets[v] = targets[v];
        p.columns = (int)g.columns;
        p.rows = (int)g.rows;
        p.step = (int)g.step;
        p.coarse = coarse;
        p.coarse_columns = (int)g.coarse_columns;
        p.coarse_rows = (int)g.coarse_rows;
        p.coarse_step = (int)g.coarse_step;
        p.inverse_step = inverse_step;
        p.near_depth = o.near_depth;
        p.far_depth = o.far_depth;
        p.unseeded = d_unseeded;
        p.radius = direct_radius;
        p.wide_radius = wide_radius;
        p.spatial = d_sp_direct;
        p.spatial_wide = d_sp_wide;
        p.minimum_score = o.minimum_score;
        p.minimum_margin = o.minimum_margin;
        p.minimum_improvement = o.minimum_improvement;
        p.minimum_support = (int)o.minimum_support;
        p.best_view_count = (int)std::min<uint64_t>(o.best_view_count, MAX_VIEWS);
        p.out = direct;
        p.guidance = fguidance;
        p.tested = ftested;
        p.wide_count = dbuf<int>(ctx, "wide_count", 1);
        p.wide_list = dbuf<int4>(ctx, "wide_list", M);
        CK(cudaMemsetAsync(p.wide_count, 0, sizeof(int), s));
        const int taps = (2 * direct_radius + 1) * (2 * direct_radius + 1);
        const int wide_taps = (2 * wide_radius + 1) * (2 * wide_radius + 1);
        const size_t slot = direct_slot_bytes<float2>(V, taps), wide_slot = direct_slot_bytes<float2>(V, wide_taps);
        if (slot > 200 * 1024 || wide_slot > 200 * 1024)
            throw CudaError{cudaErrorInvalidValue, "direct pass shared memory exceeds 200 KiB"};
        p.nodes_per_cta = warps_per_cta(direct_depth_kernel, slot, 8);
        direct_depth_kernel<<<blocks_for(M, p.nodes_per_cta), 32 * p.nodes_per_cta, p.nodes_per_cta * slot, s>>>(p);
        CK(cudaGetLastError());
        const int wide_warps = warps_per_cta(direct_wide_kernel, wide_slot, 8);
        int wide_blocks = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wide_blocks, direct_wide_kernel, 32 * wide_warps,
                                                         wide_warps * wide_slot));
        direct_wide_kernel<<<ctx->sm_count * std::max(1, wide_blocks), 32 * wide_warps, wide_warps * wide_slot,
                             s>>>(p);
        CK(cudaGetLastError());
    }
    if (debug) {
        download_field(ctx, direct, M, debug->direct_has, debug->direct_depth, debug->direct_confidence,
                       debug->direct_improvement, debug->direct_regularized);
        download(ctx, debug->direct_guidance, fguidance, M);
        download(ctx, debug->direct_tested, ftested, M);
    }
    record_event(ctx->events[4], s, capturing);
    // ---- consistency filters (depth.rs:383-392)
    uint8_t *has_a = dbuf<uint8_t>(ctx, "has_isolated", M);
    reject_isolated_kernel<<<blocks_for(M, 256), 256, 0, s>>>(direct.has, direct.depth, direct.confidence, fguidance,
                                                             has_a, (int)g.columns, (int)g.rows, inverse_step * 2.5);
    CK(cudaGetLastError());
    if (debug) download(ctx, debug->isolated_has, has_a, M);
    int *parent = dbuf<int>(ctx, "uf_parent", M);
    int *csize = dbuf<int>(ctx, "uf_size", M);
    components_init_kernel<<<blocks_for(M, 256), 256, 0, s>>>(parent, (int)M);
    CK(cudaMemsetAsync(csize, 0, M * sizeof(int), s));
    components_union_kernel<<<blocks_for(M, 256), 256, 0, s>>>(has_a, direct.depth, fguidance, parent, (int)g.columns,
                                                               (int)g.rows, inverse_step * 2.5,
                                                               union_retries(ctx, M), &d_results->status);
    components_size_kernel<<<blocks_for(M, 256), 256, 0, s>>>(has_a, parent, csize, (int)M);
    Field fin = field_bufs(ctx, "final", M);
    components_mark_kernel<<<blocks_for(M, 256), 256, 0, s>>>(has_a, parent, csize, fin.has, (int)M,
                                                              MINIMUM_DIRECT_COMPONENT_NODES);
    CK(cudaGetLastError());
    if (debug) download(ctx, debug->component_has, fin.has, M);
    fit_local_planes_kernel<<<blocks_for(M, 256), 256, 0, s>>>(fin.has, direct.depth, direct.confidence, fguidance,
                                                               d_sp25, fin.depth, (int)g.columns, (int)g.rows,
                                                               inverse_step * 4.0);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(fin.confidence, direct.confidence, M * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(fin.improvement, direct.improvement, M * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(fin.regularized, direct.regularized, M, cudaMemcpyDeviceToDevice, s));
    // depth of removed nodes: NaN (None)
    if (debug && debug->fitted_depth) {
        std::vector<uint8_t> h(M);
        download(ctx, h.data(), fin.has, M);
        download(ctx, debug->fitted_depth, fin.depth, M);
        CK(cudaStreamSynchronize(s));
        for (size_t i = 0; i < M; ++i)
            if (!h[i]) debug->fitted_depth[i] = NAN;
    }
    // report statistics and medians
    double *depth_keys = dbuf<double>(ctx, "depth_keys", M);
    double *depth_sorted = dbuf<double>(ctx, "depth_sorted", M);
    float *imp_keys = dbuf<float>(ctx, "imp_keys", M);
    float *imp_sorted = dbuf<float>(ctx, "imp_sorted", M);
    field_stats_kernel<<<blocks_for(M, 256), 256, 0, s>>>(ftested, fin, (int)M, d_results, depth_keys, imp_keys);
    CK(cudaGetLastError());
    {
        size_t t1 = 0, t2 = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, t1, depth_keys, depth_sorted, (int)M, 0, 64, s));
        CK(cub::DeviceRadixSort::SortKeys(nullptr, t2, imp_keys, imp_sorted, (int)M, 0, 32, s));
        void *tmp = dbuf<unsigned char>(ctx, "cub_tmp", std::max(t1, t2));
        CK(cub::DeviceRadixSort::SortKeys(tmp, t1, depth_keys, depth_sorted, (int)M, 0, 64, s));
        CK(cub::DeviceRadixSort::SortKeys(tmp, t2, imp_keys, imp_sorted, (int)M, 0, 32, s));
    }
    medians_kernel<<<1, 1, 0, s>>>(depth_sorted, imp_sorted, d_results);
    CK(cudaGetLastError());
    // the depth map needs only the final field, so it is ready before the decisions
    depth_map_kernel<<<blocks_for(M, 256), 256, 0, s>>>(fin, ftested, out.depth, out.confidence, out.provenance, (int)M);
    CK(cudaGetLastError());
    if (host) CK(cudaEventRecord(ctx->map_ready, s));
    record_event(ctx->events[5], s, capturing);
    // ---- per-target decisions (depth.rs:420-547): all targets in one launch
    rewritten.clear();
    if (V > 0) {
        DecisionParams p{};
        p.views = d_views;
        p.reference = reference;
        p.n_targets = V;
        for (int v = 0; v < V; ++v) {
            p.targets[v] = targets[v];
            p.out[v] = decision_bufs(ctx, "dec" + std::to_string(v), M);
        }
        p.columns = (int)g.columns;
        p.rows = (int)g.rows;
        p.step = (int)g.step;
        p.field = fin;
        p.geometry = fine_geometry;
        if (fine_lattice) p.lattice = lattice;
        p.inverse_step = inverse_step;
        p.near_depth = o.near_depth;
        p.far_depth = o.far_depth;
        p.radius = radius;
        p.spatial = d_sp;
        p.patches = radius == direct_radius ? fine_patches : nullptr;  // the same patch and weights
        p.minimum_score = o.minimum_score;
        int taps = (2 * radius + 1) * (2 * radius + 1);
        const size_t slot = decision_slot_bytes(V, taps);
        if (slot > 200 * 1024) throw CudaError{cudaErrorInvalidValue, "decision shared memory exceeds 200 KiB"};
        // one or two targets leave most lanes of a node's warp idle in both phases (6 V and
        // 8 V items): the CTA then pools its nodes' correlations
        const auto decision_kernel = V <= 2 ? target_decision_kernel<true> : target_decision_kernel<false>;
        const int warps = warps_per_cta(decision_kernel, slot, DECISION_WARPS);
        decision_kernel<<<blocks_for(M, warps), 32 * warps, warps * slot, s>>>(p);
        CK(cudaGetLastError());
        Decisions dec2 = decision_bufs(ctx, "dec_consensus", M), dec3 = decision_bufs(ctx, "dec_boundary", M);
        for (int v = 0; v < V; ++v) {
            const int t = targets[v];
            const Decisions &dec = p.out[v];
            copy_decisions(ctx, dec2, dec, M);
            warp_consensus_kernel<<<blocks_for(M, 256), 256, 0, s>>>(dec, dec2, (int)g.columns, (int)g.rows);
            copy_decisions(ctx, dec3, dec2, M);
            warp_boundary_kernel<<<blocks_for(M, 256), 256, 0, s>>>(dec2, dec3, fguidance, (int)g.columns,
                                                                    (int)g.rows);
            warp_output_kernel<<<blocks_for(M, 256), 256, 0, s>>>(dec3, out.points[t], out.warp_confidence[t],
                                                                  d_results->target_counts[t], (int)M);
            CK(cudaGetLastError());
            if (debug && debug->decision_kind) download(ctx, debug->decision_kind + (size_t)t * M, dec3.kind, M);
            rewritten.push_back(t);
        }
    }
    record_event(ctx->events[6], s, capturing);
    if (capturing) {
        cudaGraph_t graph = nullptr;
        guard.active = false;
        CK(cudaStreamEndCapture(s, &graph));
        const cudaError_t e = cudaGraphInstantiate(&ctx->stage_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ctx->stage_exec = nullptr;
            throw CudaError{e, "cudaGraphInstantiate(stage)"};
        }
        CK(cudaGraphLaunch(ctx->stage_exec, s));
        ctx->stage_graph_state = 1;
    }
    if (ctx->stage_graph && !host && !debug) ctx->stage_key_epoch = ctx->alloc_epoch;
    if (host) {
        // every kernel is queued: the depth map leaves on the copy stream while the
        // decisions run (a pageable destination blocks this thread, not the GPU)
        CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->map_ready, 0));
        CK(cudaMemcpyAsync(host->depth, out.depth, M * sizeof(double), cudaMemcpyDeviceToHost, ctx->copy_stream));
        CK(cudaMemcpyAsync(host->confidence, out.confidence, M * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->copy_stream));
        CK(cudaMemcpyAsync(host->provenance, out.provenance, M, cudaMemcpyDeviceToHost, ctx->copy_stream));
        for (int t : rewritten) {
            download(ctx, host->points[t], out.points[t], M);
            download(ctx, host->warp_confidence[t], out.warp_confidence[t], M);
        }
    }
    CK(cudaMemcpyAsync(&h_results, d_results, sizeof(Results), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaStreamSynchronize(ctx->copy_stream));
    for (int i = 0; i < 6; ++i) CK(cudaEventElapsedTime(&ctx->timings[i], ctx->events[i], ctx->events[i + 1]));
    CK(cudaEventElapsedTime(&ctx->timings[6], ctx->events[0], ctx->events[6]));
}

float fraction(unsigned long long count, unsigned long long total) {
    return total == 0 ? 0.0f : (float)count / (float)total;
}

void fill_reports(const Results &r, const std::vector<int> &rewritten, size_t n_views, chiaro_depth_report *reports) {
    if (!reports) return;
    for (size_t i = 0; i < n_views; ++i) reports[i].present = 0;
    unsigned long long fallback =
        r.tested >= r.measured + r.regularized ? r.tested - (r.measured + r.regularized) : 0;
    for (int t : rewritten) {
        chiaro_depth_report &rep = reports[t];
        rep.present = 1;
        rep.tested_nodes = r.tested;
        rep.measured_nodes = r.measured;
        rep.regularized_nodes = r.regularized;
        rep.fallback_nodes = fallback;
        rep.refined_nodes = r.target_counts[t][0];
        rep.occluded_nodes = r.target_counts[t][1];
        rep.boundary_nodes = r.target_counts[t][2];
        rep.reconstructed_fraction = fraction(r.measured + r.regularized, r.tested);
        rep.refined_fraction = fraction(r.target_counts[t][0], r.tested);
        rep.occluded_fraction = fraction(r.target_counts[t][1], r.tested);
        rep.has_median_depth = r.has_median_depth;
        rep.median_depth = r.has_median_depth ? r.median_depth : 0.0;
        rep.has_median_score_improvement = r.has_median_improvement;
        rep.median_score_improvement = r.has_median_improvement ? r.median_improvement : 0.0f;
    }
}

int validate(const chiaro_view *views, size_t n_views, size_t reference_index, const chiaro_depth_options *options) {
    if (!views || !options) return CHIARO_ERR_ARGUMENT;
    if (!options_valid(*options) || reference_index >= n_views || !views[reference_index].has_camera)
        return CHIARO_INVALID;
    if (n_views > (size_t)MAX_VIEWS || options->planes + 1 > (uint64_t)MAX_LABELS ||
        options->patch_radius > (uint64_t)MAX_RADIUS)
        return CHIARO_ERR_ARGUMENT;
    for (size_t i = 0; i < n_views; ++i) {
        const chiaro_view &v = views[i];
        if (!v.luminance || v.luma_width < 1 || v.luma_height < 1 || !v.warp.points || v.warp.step < 1 ||
            v.warp.columns < 1 || v.warp.rows < 1)
            return CHIARO_ERR_ARGUMENT;
        // planes and grids addressed with 32-bit indices; planes below 2^22 pixels per side
        if (v.luma_width >= (1u << 22) || v.luma_height >= (1u << 22) ||
            v.luma_width * v.luma_height >= (1ull << 31) || v.warp.columns * v.warp.rows >= (1ull << 31))
            return CHIARO_ERR_ARGUMENT;
    }
    return CHIARO_OK;
}

DevView dev_view(const chiaro_view &v, const float *luma, const float2 *points) {
    DevView d{};
    d.luma.data = luma;
    d.luma.width = (int)v.luma_width;
    d.luma.height = (int)v.luma_height;
    d.warp.points = points;
    d.warp.step = (int)v.warp.step;
    d.warp.columns = (int)v.warp.columns;
    d.warp.rows = (int)v.warp.rows;
    d.width = (int)v.width;
    d.height = (int)v.height;
    d.has_camera = v.has_camera != 0;
    d.accepted = v.accepted != 0;
    if (v.has_camera) camera_from_abi(v.camera, d.cam);
    return d;
}

int refine(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views, size_t reference_index,
           const chiaro_depth_options *options, chiaro_warp *refined, chiaro_depth_report *reports,
           chiaro_depth_map *out_map, const chiaro_depth_debug *debug, bool device_pointers) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    int st = validate(views, n_views, reference_index, options);
    if (st != CHIARO_OK) {
        if (reports && st == CHIARO_INVALID)
            for (size_t i = 0; i < n_views; ++i) reports[i].present = 0;
        return st;
    }
    const chiaro_depth_options &o = *options;
    Grids g = grids_for(views[reference_index].width, views[reference_index].height, o);
    const size_t M = g.columns * g.rows;
    if (!out_map || out_map->capacity < M || !out_map->depth || !out_map->confidence || !out_map->provenance)
        return CHIARO_ERR_CAPACITY;
    for (size_t t = 0; t < n_views; ++t) {
        bool target = t != reference_index && views[t].accepted && views[t].has_camera;
        if (target && (!refined || refined[t].capacity < M || !refined[t].points || !refined[t].confidence))
            return CHIARO_ERR_CAPACITY;
    }
    try {
        CK(cudaSetDevice(ctx->device));
        std::vector<DevView> h_views(n_views);
        HostTransfers host;
        for (size_t i = 0; i < n_views; ++i) {
            const chiaro_view &v = views[i];
            size_t luma_n = v.luma_width * v.luma_height, warp_n = v.warp.columns * v.warp.rows;
            const float *luma = v.luminance;
            const float2 *pts = reinterpret_cast<const float2 *>(v.warp.points);
            if (!device_pointers) {
                float *dl = dbuf<float>(ctx, "luma" + std::to_string(i), luma_n);
                float2 *dp = dbuf<float2>(ctx, "warp" + std::to_string(i), warp_n);
                host.planes.push_back({dl, v.luminance, luma_n * sizeof(float)});  // sent inside the stage
                upload(ctx, dp, reinterpret_cast<const float2 *>(v.warp.points), warp_n);
                luma = dl;
                pts = dp;
            }
            h_views[i] = dev_view(v, luma, pts);
        }
        DevView *d_views = dbuf<DevView>(ctx, "views", n_views);
        upload(ctx, d_views, h_views.data(), n_views);
        StageOutputs out{};
        if (device_pointers) {
            out.depth = out_map->depth;
            out.confidence = out_map->confidence;
            out.provenance = out_map->provenance;
            for (size_t t = 0; t < n_views; ++t)
                if (refined && refined[t].points) {
                    out.points[t] = reinterpret_cast<float2 *>(refined[t].points);
                    out.warp_confidence[t] = refined[t].confidence;
                }
        } else {
            out.depth = dbuf<double>(ctx, "out.depth", M);
            out.confidence = dbuf<float>(ctx, "out.confidence", M);
            out.provenance = dbuf<uint8_t>(ctx, "out.provenance", M);
            host.depth = out_map->depth;
            host.confidence = out_map->confidence;
            host.provenance = out_map->provenance;
            for (size_t t = 0; t < n_views; ++t) {
                out.points[t] = dbuf<float2>(ctx, "out.points" + std::to_string(t), M);
                out.warp_confidence[t] = dbuf<float>(ctx, "out.wconf" + std::to_string(t), M);
                if (refined) {
                    host.points[t] = reinterpret_cast<float2 *>(refined[t].points);
                    host.warp_confidence[t] = refined[t].confidence;
                }
            }
        }
        Results *d_results = dbuf<Results>(ctx, "results", 1);
        Results h_results{};
        std::vector<int> rewritten;
        run_stage(ctx, h_views, d_views, (int)reference_index, o, g, out, d_results, h_results, debug, rewritten,
                  device_pointers ? nullptr : &host);
        out_map->columns = g.columns;
        out_map->rows = g.rows;
        out_map->step = g.step;
        out_map->near_depth = o.near_depth;
        out_map->far_depth = o.far_depth;
        for (int t : rewritten) {
            refined[t].step = g.step;
            refined[t].columns = g.columns;
            refined[t].rows = g.rows;
        }
        if (h_results.status & UNION_GAVE_UP) {
            ctx->error = "reject_small_direct_components: a union-find join ran out of retries";
            return CHIARO_ERR_TIMEOUT;
        }
        fill_reports(h_results, rewritten, n_views, reports);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------
extern "C" {

int chiaro_depth_abi_version(void) { return CHIARO_DEPTH_ABI_VERSION; }

int chiaro_host_alloc(uint64_t bytes, void **out) {
    if (!out) return CHIARO_ERR_ARGUMENT;
    *out = nullptr;
    if (bytes == 0) return CHIARO_OK;
    return cudaHostAlloc(out, bytes, cudaHostAllocPortable) == cudaSuccess ? CHIARO_OK : CHIARO_ERR_CUDA;
}

void chiaro_host_free(void *ptr) {
    if (ptr) cudaFreeHost(ptr);
}

int chiaro_depth_ctx_create(int device, chiaro_depth_ctx **out) {
    if (!out) return CHIARO_ERR_ARGUMENT;
    *out = nullptr;
    auto *ctx = new chiaro_depth_ctx();
    ctx->device = device;
    try {
        CK(cudaSetDevice(device));
        CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        for (auto &e : ctx->events) CK(cudaEventCreate(&e));
        CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->planes_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ref_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->map_ready, cudaEventDisableTiming));
    } catch (const CudaError &e) {
        delete ctx;
        return CHIARO_ERR_CUDA;
    }
    *out = ctx;
    return CHIARO_OK;
}

void chiaro_depth_ctx_destroy(chiaro_depth_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &kv : ctx->buffers)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (auto &e : ctx->events)
        if (e) cudaEventDestroy(e);
    if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
    if (ctx->stage_exec) cudaGraphExecDestroy(ctx->stage_exec);
    if (ctx->planes_ready) cudaEventDestroy(ctx->planes_ready);
    if (ctx->ref_ready) cudaEventDestroy(ctx->ref_ready);
    if (ctx->map_ready) cudaEventDestroy(ctx->map_ready);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *chiaro_depth_last_error(const chiaro_depth_ctx *ctx) { return ctx ? ctx->error.c_str() : "no context"; }

void chiaro_depth_options_default(chiaro_depth_options *o) {  // depth.rs:69-91
    if (!o) return;
    *o = chiaro_depth_options{};
    o->enabled = 1;
    o->grid_step = 8;
    o->near_depth = 500.0;
    o->far_depth = 10000000.0;
    o->planes = 96;
    o->patch_radius = 4;
    o->minimum_support = 2;
    o->best_view_count = 3;
    o->minimum_score = 0.45f;
    o->minimum_margin = 0.01f;
    o->minimum_improvement = 0.01f;
    o->minimum_neighbour_support = 2;
    o->completion_iterations = 0;
}

int chiaro_depth_options_valid(const chiaro_depth_options *o) { return o && options_valid(*o) ? 1 : 0; }

int chiaro_depth_output_shape(uint64_t width, uint64_t height, const chiaro_depth_options *o, uint64_t *columns,
                              uint64_t *rows, uint64_t *step, uint64_t *coarse_columns, uint64_t *coarse_rows,
                              uint64_t *coarse_step) {
    if (!o) return CHIARO_ERR_ARGUMENT;
    Grids g = grids_for(width, height, *o);
    if (columns) *columns = g.columns;
    if (rows) *rows = g.rows;
    if (step) *step = g.step;
    if (coarse_columns) *coarse_columns = g.coarse_columns;
    if (coarse_rows) *coarse_rows = g.coarse_rows;
    if (coarse_step) *coarse_step = g.coarse_step;
    return CHIARO_OK;
}

int chiaro_refine_multiview_depth(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                                  size_t reference_index, const chiaro_depth_options *options, chiaro_warp *refined,
                                  chiaro_depth_report *reports, chiaro_depth_map *out_map,
                                  const chiaro_depth_debug *debug) {
    return refine(ctx, views, n_views, reference_index, options, refined, reports, out_map, debug, false);
}

int chiaro_refine_multiview_depth_device(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                                         size_t reference_index, const chiaro_depth_options *options,
                                         chiaro_warp *refined, chiaro_depth_report *reports,
                                         chiaro_depth_map *out_map) {
    return refine(ctx, views, n_views, reference_index, options, refined, reports, out_map, nullptr, true);
}

int chiaro_depth_set_stage_graph(chiaro_depth_ctx *ctx, int32_t enabled) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        if ((enabled != 0) == (ctx->stage_graph != 0)) return CHIARO_OK;  // unchanged: keep the graph
        ctx->stage_graph = enabled != 0;
        if (!ctx->stage_graph && ctx->stage_exec) {
            CK(cudaStreamSynchronize(ctx->stream));
            CK(cudaGraphExecDestroy(ctx->stage_exec));
            ctx->stage_exec = nullptr;
        }
        ctx->stage_key.clear();
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_depth_stage_graph_state(const chiaro_depth_ctx *ctx) { return ctx ? ctx->stage_graph_state : -1; }

int chiaro_depth_set_union_retry_limit(chiaro_depth_ctx *ctx, int32_t retries) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    ctx->union_retries = retries < 0 ? -1 : retries;
    return CHIARO_OK;
}

int chiaro_depth_set_memory_limit(chiaro_depth_ctx *ctx, uint64_t bytes) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    ctx->memory_limit = bytes;
    return CHIARO_OK;
}

uint64_t chiaro_depth_memory_held(const chiaro_depth_ctx *ctx) { return ctx ? ctx->memory_held : 0; }

int chiaro_depth_set_autotune(chiaro_depth_ctx *ctx, int32_t mode) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    bool shape = false;
    for (int t : COST_SHAPES) shape |= t == mode;
    if (mode != 0 && mode != 1 && !shape) return CHIARO_ERR_ARGUMENT;
    ctx->autotune = mode;
    if (mode != 1) ctx->cost_tuning.clear();
    return CHIARO_OK;
}

int chiaro_depth_tuning(const chiaro_depth_ctx *ctx, uint64_t *keys, int32_t *threads, int capacity) {
    if (!ctx) return 0;
    int n = 0;
    for (const auto &kv : ctx->cost_tuning) {
        if (n < capacity) {
            if (keys) keys[n] = kv.first;
            if (threads) threads[n] = kv.second;
        }
        ++n;
    }
    return n;
}

int chiaro_depth_last_timings(const chiaro_depth_ctx *ctx, float *ms, int capacity) {
    if (!ctx || !ms) return 0;
    int n = std::min(capacity, 7);
    for (int i = 0; i < n; ++i) ms[i] = ctx->timings[i];
    return n;
}

int chiaro_depth_last_launches(const chiaro_depth_ctx *ctx) { return ctx ? ctx->launches : 0; }

void *chiaro_depth_ctx_stream(const chiaro_depth_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int chiaro_sgm_aggregate_device(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                                uint64_t rows, uint64_t labels, float *out) {
    if (!ctx || !costs || !guidance || !out || columns < 1 || rows < 1 || labels < 1 || labels > MAX_LABELS)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        launch_sgm(ctx, costs, guidance, out, (int)columns, (int)rows, (int)labels);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_sgm_aggregate(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                         uint64_t rows, uint64_t labels, float *out) {
    if (!ctx || !costs || !guidance || !out || columns < 1 || rows < 1 || labels < 1 || labels > MAX_LABELS)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows, nl = n * labels;
        float *dc = dbuf<float>(ctx, "op.costs", nl), *dg = dbuf<float>(ctx, "op.guidance", n),
              *dout = dbuf<float>(ctx, "op.out", nl);
        upload(ctx, dc, costs, nl);
        upload(ctx, dg, guidance, n);
        launch_sgm(ctx, dc, dg, dout, (int)columns, (int)rows, (int)labels);
        download(ctx, out, dout, nl);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_select_depths(chiaro_depth_ctx *ctx, const double *labels, uint64_t n_labels, const float *scores,
                         const float *regularised, const uint8_t *tested, uint64_t n_nodes,
                         const chiaro_depth_options *options, uint8_t *has, double *depth, float *confidence,
                         float *improvement, uint8_t *regularized, uint8_t *fillable) {
    if (!ctx || !labels || !scores || !regularised || !tested || !options || n_labels < 2 || n_labels > MAX_LABELS)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t nl = n_nodes * n_labels;
        double *dl = dbuf<double>(ctx, "op.labels", n_labels);
        float *ds = dbuf<float>(ctx, "op.scores", nl), *dr = dbuf<float>(ctx, "op.reg", nl);
        uint8_t *dt = dbuf<uint8_t>(ctx, "op.tested", n_nodes);
        Field f = field_bufs(ctx, "op.field", n_nodes);
        uint8_t *dfill = dbuf<uint8_t>(ctx, "op.fillable", n_nodes);
        upload(ctx, dl, labels, n_labels);
        upload(ctx, ds, scores, nl);
        upload(ctx, dr, regularised, nl);
        upload(ctx, dt, tested, n_nodes);
        SelectParams p{};
        p.scores = ds;
        p.regularised = dr;
        p.tested = dt;
        p.label_depth = dl;
        p.nodes = (int)n_nodes;
        p.labels = (int)n_labels;
        p.minimum_score = options->minimum_score;
        p.minimum_margin = options->minimum_margin;
        p.minimum_improvement = options->minimum_improvement;
        p.field = f;
        p.fillable = dfill;
        select_depths_kernel<<<blocks_for(n_nodes * 32, 256), 256, 0, ctx->stream>>>(p);
        CK(cudaGetLastError());
        download_field(ctx, f, n_nodes, has, depth, confidence, improvement, regularized);
        download(ctx, fillable, dfill, n_nodes);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_reject_isolated(chiaro_depth_ctx *ctx, uint8_t *has, const double *depth, const float *confidence,
                           const float *guidance, uint64_t columns, uint64_t rows, double inverse_tolerance) {
    if (!ctx || !has || !depth || !confidence || !guidance) return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows;
        uint8_t *dh = dbuf<uint8_t>(ctx, "op.has", n), *dh2 = dbuf<uint8_t>(ctx, "op.has2", n);
        double *dd = dbuf<double>(ctx, "op.depth", n);
        float *dc = dbuf<float>(ctx, "op.conf", n), *dg = dbuf<float>(ctx, "op.guid", n);
        upload(ctx, dh, has, n);
        upload(ctx, dd, depth, n);
        upload(ctx, dc, confidence, n);
        upload(ctx, dg, guidance, n);
        reject_isolated_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(dh, dd, dc, dg, dh2, (int)columns,
                                                                           (int)rows, inverse_tolerance);
        CK(cudaGetLastError());
        download(ctx, has, dh2, n);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_reject_small_components(chiaro_depth_ctx *ctx, uint8_t *has, const double *depth, const float *guidance,
                                   uint64_t columns, uint64_t rows, double inverse_tolerance, uint64_t minimum_nodes) {
    if (!ctx || !has || !depth || !guidance || columns < 1 || rows < 1) return CHIARO_ERR_ARGUMENT;
    // node indices are 32-bit: refuse each side before the product can wrap
    if (columns >= (1ull << 31) || rows >= (1ull << 31) || columns * rows >= (1ull << 31)) return CHIARO_ERR_ARGUMENT;
    if (minimum_nodes <= 1) return CHIARO_OK;  // depth.rs:941-943
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows;
        cudaStream_t s = ctx->stream;
        uint8_t *dh = dbuf<uint8_t>(ctx, "op.has", n), *dh2 = dbuf<uint8_t>(ctx, "op.has2", n);
        double *dd = dbuf<double>(ctx, "op.depth", n);
        float *dg = dbuf<float>(ctx, "op.guid", n);
        int *parent = dbuf<int>(ctx, "op.parent", n), *size = dbuf<int>(ctx, "op.size", n);
        int *status = dbuf<int>(ctx, "op.status", 1);
        upload(ctx, dh, has, n);
        upload(ctx, dd, depth, n);
        upload(ctx, dg, guidance, n);
        CK(cudaMemsetAsync(status, 0, sizeof(int), s));
        components_init_kernel<<<blocks_for(n, 256), 256, 0, s>>>(parent, (int)n);
        CK(cudaMemsetAsync(size, 0, n * sizeof(int), s));
        components_union_kernel<<<blocks_for(n, 256), 256, 0, s>>>(dh, dd, dg, parent, (int)columns, (int)rows,
                                                                   inverse_tolerance, union_retries(ctx, n), status);
        components_size_kernel<<<blocks_for(n, 256), 256, 0, s>>>(dh, parent, size, (int)n);
        components_mark_kernel<<<blocks_for(n, 256), 256, 0, s>>>(dh, parent, size, dh2, (int)n,
                                                                  (int)std::min<uint64_t>(minimum_nodes, INT32_MAX));
        CK(cudaGetLastError());
        int h_status = 0;
        CK(cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (h_status & UNION_GAVE_UP) {
            ctx->error = "reject_small_components: a union-find join ran out of retries";
            return CHIARO_ERR_TIMEOUT;
        }
        download(ctx, has, dh2, n);
        CK(cudaStreamSynchronize(s));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_fit_local_planes(chiaro_depth_ctx *ctx, const uint8_t *has, double *depth, const float *confidence,
                            const float *guidance, uint64_t columns, uint64_t rows, double inverse_tolerance) {
    if (!ctx || !has || !depth || !confidence || !guidance) return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows;
        uint8_t *dh = dbuf<uint8_t>(ctx, "op.has", n);
        double *dd = dbuf<double>(ctx, "op.depth", n), *dd2 = dbuf<double>(ctx, "op.depth2", n);
        float *dc = dbuf<float>(ctx, "op.conf", n), *dg = dbuf<float>(ctx, "op.guid", n);
        std::vector<double> spatial25(25);
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx)
                spatial25[(dy + 2) * 5 + dx + 2] = std::exp((double)(-(dx * dx + dy * dy)) / 6.0);
        double *d25 = dbuf<double>(ctx, "op.sp25", 25);
        upload(ctx, d25, spatial25.data(), 25);
        upload(ctx, dh, has, n);
        upload(ctx, dd, depth, n);
        upload(ctx, dc, confidence, n);
        upload(ctx, dg, guidance, n);
        fit_local_planes_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(dh, dd, dc, dg, d25, dd2, (int)columns,
                                                                            (int)rows, inverse_tolerance);
        CK(cudaGetLastError());
        download(ctx, depth, dd2, n);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_warp_decisions_filter(chiaro_depth_ctx *ctx, uint8_t *kind, float *global, float *point,
                                 const uint8_t *measured, const float *guidance, uint64_t columns, uint64_t rows,
                                 int consensus, int boundaries) {
    if (!ctx || !kind || !global || !point || !measured || !guidance) return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows;
        cudaStream_t s = ctx->stream;
        Decisions a = decision_bufs(ctx, "op.dec", n), b = decision_bufs(ctx, "op.dec2", n);
        float *dg = dbuf<float>(ctx, "op.guid", n);
        upload(ctx, a.kind, kind, n);
        upload(ctx, a.global, reinterpret_cast<const float2 *>(global), n);
        upload(ctx, a.point, reinterpret_cast<const float2 *>(point), n);
        upload(ctx, a.measured, measured, n);
        CK(cudaMemsetAsync(a.confidence, 0, n * 4, s));
        upload(ctx, dg, guidance, n);
        if (consensus) {
            copy_decisions(ctx, b, a, n);
            warp_consensus_kernel<<<blocks_for(n, 256), 256, 0, s>>>(a, b, (int)columns, (int)rows);
            std::swap(a, b);
        }
        if (boundaries) {
            copy_decisions(ctx, b, a, n);
            warp_boundary_kernel<<<blocks_for(n, 256), 256, 0, s>>>(a, b, dg, (int)columns, (int)rows);
            std::swap(a, b);
        }
        CK(cudaGetLastError());
        download(ctx, kind, a.kind, n);
        download(ctx, reinterpret_cast<float2 *>(global), a.global, n);
        download(ctx, reinterpret_cast<float2 *>(point), a.point, n);
        CK(cudaStreamSynchronize(s));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_sgm_aggregate_u16_device(chiaro_depth_ctx *ctx, const float *costs, const float *guidance,
                                    uint64_t columns, uint64_t rows, uint64_t labels, uint16_t *aggregate,
                                    uint16_t *best) {
    if (!ctx || !costs || !guidance || (!aggregate && !best) || columns < 1 || rows < 1 || labels < 1 ||
        labels > MAX_LABELS || columns * rows > (1u << 30))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        launch_sgm_u16(ctx, costs, guidance, (int)columns, (int)rows, (int)labels, aggregate, best);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_sgm_aggregate_u16(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                             uint64_t rows, uint64_t labels, uint16_t *aggregate, uint16_t *best) {
    if (!ctx || !costs || !guidance || (!aggregate && !best) || columns < 1 || rows < 1 || labels < 1 ||
        labels > MAX_LABELS || columns * rows > (1u << 30))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        size_t n = columns * rows, nl = n * labels;
        float *dc = dbuf<float>(ctx, "op.costs", nl), *dg = dbuf<float>(ctx, "op.guidance", n);
        uint16_t *da = aggregate ? dbuf<uint16_t>(ctx, "op.aggregate16", nl) : nullptr;
        uint16_t *db = best ? dbuf<uint16_t>(ctx, "op.best16", n) : nullptr;
        upload(ctx, dc, costs, nl);
        upload(ctx, dg, guidance, n);
        launch_sgm_u16(ctx, dc, dg, (int)columns, (int)rows, (int)labels, da, db);
        download(ctx, aggregate, da, nl);
        download(ctx, best, db, n);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_sgm_aggregate_batch_device(chiaro_depth_ctx *ctx, const chiaro_sgm_instance *instances,
                                      uint64_t n_instances, uint64_t scratch_bytes, int flags) {
    if (!ctx || (!instances && n_instances) || (flags & ~(CHIARO_BATCH_GRAPH | CHIARO_BATCH_AUTOTUNE)))
        return CHIARO_ERR_ARGUMENT;
    if (n_instances == 0) return CHIARO_OK;
    try {
        CK(cudaSetDevice(ctx->device));
        return run_batch(ctx, instances, (size_t)n_instances, (size_t)scratch_bytes, flags);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

int chiaro_sgm_batch_report(const chiaro_depth_ctx *ctx, int *warps_per_cta, int *waves, int *replayed) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    if (warps_per_cta) *warps_per_cta = ctx->batch_warps;
    if (waves) *waves = ctx->batch_waves;
    if (replayed) *replayed = ctx->batch_replayed;
    return CHIARO_OK;
}

int chiaro_sgm_banded_report(const chiaro_depth_ctx *ctx, int *windows) {
    if (!ctx || !windows) return CHIARO_ERR_ARGUMENT;
    *windows = ctx->band_windows;
    return CHIARO_OK;
}

static int band_args(const void *ctx, const float *costs, const float *guidance, uint64_t columns, uint64_t rows,
                     uint64_t labels, const int32_t *offsets, uint64_t tile, uint64_t band, uint64_t margin,
                     const int32_t *winner, const uint8_t *fallback) {
    if (!ctx || !costs || !guidance || !offsets || !winner || !fallback || columns < 1 || rows < 1 || tile < 1 ||
        tile > 1024 || band < 1 || band > 32 || labels < band + 1 || labels > MAX_LABELS || margin > 4096 ||
        columns * rows > (1u << 26))
        return CHIARO_ERR_ARGUMENT;
    return CHIARO_OK;
}

int chiaro_sgm_banded_device(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                             uint64_t rows, uint64_t labels, const int32_t *tile_offsets, uint64_t tile,
                             uint64_t band, uint64_t margin, int32_t *winner, uint8_t *fallback) {
    if (int st = band_args(ctx, costs, guidance, columns, rows, labels, tile_offsets, tile, band, margin, winner,
                           fallback))
        return st;
    try {
        CK(cudaSetDevice(ctx->device));
        return run_band(ctx, costs, guidance, (int)columns, (int)rows, (int)labels, tile_offsets, (int)tile,
                        (int)band, (int)margin, winner, fallback);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

int chiaro_sgm_banded(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                      uint64_t rows, uint64_t labels, const int32_t *tile_offsets, uint64_t tile, uint64_t band,
                      uint64_t margin, int32_t *winner, uint8_t *fallback) {
    if (int st = band_args(ctx, costs, guidance, columns, rows, labels, tile_offsets, tile, band, margin, winner,
                           fallback))
        return st;
    try {
        CK(cudaSetDevice(ctx->device));
        const size_t n = columns * rows, nl = n * labels;
        const size_t tiles = ((columns + tile - 1) / tile) * ((rows + tile - 1) / tile);
        float *dc = dbuf<float>(ctx, "op.costs", nl), *dg = dbuf<float>(ctx, "op.guidance", n);
        int *doff = dbuf<int>(ctx, "op.band_offsets", tiles), *dw = dbuf<int>(ctx, "op.band_winner", n);
        uint8_t *df = dbuf<uint8_t>(ctx, "op.band_fallback", tiles);
        upload(ctx, dc, costs, nl);
        upload(ctx, dg, guidance, n);
        upload(ctx, doff, tile_offsets, tiles);
        int st = run_band(ctx, dc, dg, (int)columns, (int)rows, (int)labels, doff, (int)tile, (int)band, (int)margin,
                          dw, df);
        if (st) return st;
        download(ctx, winner, dw, n);
        download(ctx, fallback, df, tiles);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

// The coarse search's views: device-memory views as the device-buffer stage takes them.
static int coarse_views(const chiaro_view *views, size_t n_views, size_t reference_index,
                        const chiaro_depth_options *options, std::vector<DevView> &h_views) {
    int st = validate(views, n_views, reference_index, options);
    if (st != CHIARO_OK) return st;
    h_views.resize(n_views);
    for (size_t i = 0; i < n_views; ++i)
        h_views[i] = dev_view(views[i], views[i].luminance, reinterpret_cast<const float2 *>(views[i].warp.points));
    return CHIARO_OK;
}

int chiaro_coarse_depth_device(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                               size_t reference_index, const chiaro_depth_options *options,
                               const chiaro_band_options *band, int32_t *winner, uint8_t *tested,
                               int32_t *tile_offsets, uint8_t *tile_fallback, chiaro_band_report *report) {
    if (!ctx || !winner) return CHIARO_ERR_ARGUMENT;
    std::vector<DevView> h_views;
    int st = coarse_views(views, n_views, reference_index, options, h_views);
    if (st != CHIARO_OK) return st;
    BandSpec spec{};
    if (band) {
        if (band->tile < 1 || band->tile > (uint64_t)NAIVE_MAX_TILE || band->band < 1 || band->band > 32 ||
            band->band > options->planes || band->margin > 4096 ||
            !(band->contradicted_fraction >= 0.0f))
            return CHIARO_ERR_ARGUMENT;
        spec = BandSpec{band->params, (int)band->tile, (int)band->band, (int)band->margin,
                        band->contradicted_fraction};
    }
    try {
        CK(cudaSetDevice(ctx->device));
        return run_coarse(ctx, h_views, (int)reference_index, *options, band ? &spec : nullptr, winner, tested,
                          tile_offsets, tile_fallback, report, nullptr, nullptr);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

int chiaro_band_prepass_device(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                               size_t reference_index, const chiaro_depth_options *options, float *sampled_costs,
                               float *guidance, uint8_t *tested) {
    if (!ctx || !sampled_costs) return CHIARO_ERR_ARGUMENT;
    std::vector<DevView> h_views;
    int st = coarse_views(views, n_views, reference_index, options, h_views);
    if (st != CHIARO_OK) return st;
    if (options->planes + 1 < (uint64_t)PREPASS_SLOTS + 2) return CHIARO_ERR_ARGUMENT;
    BandSpec spec{nullptr, 4, 1, 0, 1.0f};
    try {
        CK(cudaSetDevice(ctx->device));
        int scratch = 0;
        return run_coarse(ctx, h_views, (int)reference_index, *options, &spec, &scratch, tested, nullptr, nullptr,
                          nullptr, sampled_costs, guidance);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

uint64_t chiaro_bandnet_parameter_count(void) { return NET_PARAMS; }

static int bandnet_args(const void *ctx, uint64_t images, uint64_t columns, uint64_t rows, uint64_t labels) {
    if (!ctx || images < 1 || columns < 1 || rows < 1 || labels < 1 + NET_BINS + 2 || labels > MAX_LABELS ||
        images * columns * rows > (1u << 26))
        return CHIARO_ERR_ARGUMENT;
    return CHIARO_OK;
}

// Batch setup shared by training and the gradient: features, targets, and
// 1 / (number of scored nodes) from the mask.
static float bandnet_batch(chiaro_depth_ctx *ctx, const NetState &s, const float *costs, const float *guidance,
                           const int32_t *winners, const uint8_t *mask, int labels, int stride, float **targets) {
    net_features(ctx, s, costs, guidance, labels, stride);
    *targets = dbuf<float>(ctx, "net.targets", (size_t)s.pixels);
    net_targets_kernel<<<(unsigned)div_ceil((size_t)s.pixels, 256), 256, 0, ctx->stream>>>(winners, s.pixels, labels,
                                                                                           *targets);
    CK(cudaGetLastError());
    std::vector<uint8_t> h(s.pixels);
    CK(cudaMemcpyAsync(h.data(), mask, s.pixels, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    size_t count = 0;
    for (uint8_t m : h) count += m != 0;
    return count ? 1.0f / (float)count : 0.0f;
}

int chiaro_bandnet_propose_device(chiaro_depth_ctx *ctx, const float *params, const float *costs,
                                  const float *guidance, uint64_t columns, uint64_t rows, uint64_t labels,
                                  uint64_t cost_stride, uint64_t tile, uint64_t band, int32_t *tile_offsets,
                                  float *centres) {
    if (bandnet_args(ctx, 1, columns, rows, labels) || !params || !costs || !guidance || !tile_offsets || tile < 1 ||
        band < 1 || band > 32 || labels < band + 1 || (cost_stride != labels && cost_stride != PREPASS_SLOTS))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        NetState s = net_state(ctx, 1, (int)rows, (int)columns);
        net_features(ctx, s, costs, guidance, (int)labels, (int)cost_stride);
        net_forward(ctx, s, params);
        const size_t tiles = ((columns + tile - 1) / tile) * ((rows + tile - 1) / tile);
        net_tile_offsets_kernel<<<(unsigned)div_ceil(tiles, 128), 128, 0, ctx->stream>>>(
            s.y, (int)columns, (int)rows, (int)labels, (int)tile, (int)band, tile_offsets);
        CK(cudaGetLastError());
        if (centres)
            CK(cudaMemcpyAsync(centres, s.y, sizeof(float) * columns * rows, cudaMemcpyDeviceToDevice, ctx->stream));
        if (int st = net_status(ctx, s)) return st;
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_bandnet_gradient_device(chiaro_depth_ctx *ctx, const float *params, const float *costs,
                                   const float *guidance, const int32_t *winners, const uint8_t *mask,
                                   uint64_t images, uint64_t columns, uint64_t rows, uint64_t labels,
                                   uint64_t cost_stride, float *grads, float *loss) {
    if (bandnet_args(ctx, images, columns, rows, labels) || !params || !costs || !guidance || !winners || !mask ||
        !grads || !loss || (cost_stride != labels && cost_stride != PREPASS_SLOTS))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        NetState s = net_state(ctx, (int)images, (int)rows, (int)columns);
        float *targets = nullptr;
        const float inverse =
            bandnet_batch(ctx, s, costs, guidance, winners, mask, (int)labels, (int)cost_stride, &targets);
        float *d_loss = dbuf<float>(ctx, "net.loss", 1);
        CK(cudaMemsetAsync(d_loss, 0, sizeof(float), ctx->stream));
        net_backward(ctx, s, params, targets, mask, inverse, grads, d_loss);
        CK(cudaMemcpyAsync(loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        if (int st = net_status(ctx, s)) return st;
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_bandnet_train_device(chiaro_depth_ctx *ctx, float *params, float *adam_m, float *adam_v,
                                uint64_t first_step, uint64_t steps, const float *costs, const float *guidance,
                                const int32_t *winners, const uint8_t *mask, uint64_t images, uint64_t columns,
                                uint64_t rows, uint64_t labels, uint64_t cost_stride, float learning_rate,
                                float *losses) {
    if (bandnet_args(ctx, images, columns, rows, labels) || !params || !adam_m || !adam_v || !costs || !guidance ||
        !winners || !mask || !(learning_rate > 0.0f) || steps > 100000 ||
        (cost_stride != labels && cost_stride != PREPASS_SLOTS))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        NetState s = net_state(ctx, (int)images, (int)rows, (int)columns);
        float *targets = nullptr;
        const float inverse =
            bandnet_batch(ctx, s, costs, guidance, winners, mask, (int)labels, (int)cost_stride, &targets);
        float *grads = dbuf<float>(ctx, "net.grads", NET_PARAMS);
        float *d_losses = dbuf<float>(ctx, "net.losses", std::max<uint64_t>(steps, 1));
        CK(cudaMemsetAsync(d_losses, 0, sizeof(float) * std::max<uint64_t>(steps, 1), ctx->stream));
        const float beta1 = 0.9f, beta2 = 0.999f;
        for (uint64_t k = 0; k < steps; ++k) {
            net_backward(ctx, s, params, targets, mask, inverse, grads, d_losses + k);
            const double t_step = (double)(first_step + k + 1);
            net_adam_kernel<<<(unsigned)div_ceil((size_t)NET_PARAMS, 256), 256, 0, ctx->stream>>>(
                params, grads, adam_m, adam_v, learning_rate, beta1, beta2, 1e-8f,
                (float)(1.0 - std::pow((double)beta1, t_step)), (float)(1.0 - std::pow((double)beta2, t_step)));
            CK(cudaGetLastError());
        }
        if (losses) CK(cudaMemcpyAsync(losses, d_losses, sizeof(float) * steps, cudaMemcpyDeviceToHost, ctx->stream));
        if (int st = net_status(ctx, s)) return st;
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

// ---- luminance_half (image.rs:401-428) -------------------------------------------------
namespace {

// Validation shared by both forms; the plane is (width / 2) x (height / 2).
int luminance_args(const uint16_t *samples, uint64_t width, uint64_t height, const chiaro_vignetting *mesh,
                   const float *out, bool device) {
    if (!samples || !out || width > (1u << 30) || height > (1u << 30)) return CHIARO_ERR_ARGUMENT;
    if (device && reinterpret_cast<uintptr_t>(samples) % 2 != 0) return CHIARO_ERR_ARGUMENT;
    if (mesh && mesh->columns >= 2 && mesh->rows >= 2 && !mesh->gains) return CHIARO_ERR_ARGUMENT;
    if (mesh && (mesh->columns > (1u << 20) || mesh->rows > (1u << 20))) return CHIARO_ERR_ARGUMENT;
    return CHIARO_OK;
}

void launch_luminance(chiaro_depth_ctx *ctx, const uint16_t *samples, uint64_t width, uint64_t height,
                      float black_q6, float white_q6, VignettingRef mesh, float *out) {
    const size_t n = (size_t)(width / 2) * (height / 2);
    if (n == 0) return;
    const unsigned blocks = (unsigned)std::min<size_t>(div_ceil(n, 256), (size_t)ctx->sm_count * 16);
    luminance_half_kernel<<<blocks, 256, 0, ctx->stream>>>(samples, (int)width, (int)height, black_q6, white_q6,
                                                          mesh, out);
    CK(cudaGetLastError());
}

}  // namespace

int chiaro_luminance_half_device(chiaro_depth_ctx *ctx, const uint16_t *samples, uint64_t width, uint64_t height,
                                 float black_q6, float white_q6, const chiaro_vignetting *mesh, float *out) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    if (int st = luminance_args(samples, width, height, mesh, out, true)) return st;
    try {
        CK(cudaSetDevice(ctx->device));
        VignettingRef m{nullptr, 0, 0};
        if (mesh && mesh->columns >= 2 && mesh->rows >= 2)
            m = VignettingRef{mesh->gains, (int)mesh->columns, (int)mesh->rows};
        launch_luminance(ctx, samples, width, height, black_q6, white_q6, m, out);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_luminance_half(chiaro_depth_ctx *ctx, const uint16_t *samples, uint64_t width, uint64_t height,
                          float black_q6, float white_q6, const chiaro_vignetting *mesh, float *out) {
    if (!ctx) return CHIARO_ERR_ARGUMENT;
    if (int st = luminance_args(samples, width, height, mesh, out, false)) return st;
    try {
        CK(cudaSetDevice(ctx->device));
        const size_t n_in = (size_t)width * height, n_out = (size_t)(width / 2) * (height / 2);
        if (n_out == 0) return CHIARO_OK;
        uint16_t *ds = dbuf<uint16_t>(ctx, "lum.samples", n_in);
        float *dout = dbuf<float>(ctx, "lum.out", n_out);
        upload(ctx, ds, samples, n_in);
        VignettingRef m{nullptr, 0, 0};
        if (mesh && mesh->columns >= 2 && mesh->rows >= 2) {
            const size_t ng = (size_t)mesh->columns * mesh->rows;
            float *dg = dbuf<float>(ctx, "lum.gains", ng);
            upload(ctx, dg, mesh->gains, ng);
            m = VignettingRef{dg, (int)mesh->columns, (int)mesh->rows};
        }
        launch_luminance(ctx, ds, width, height, black_q6, white_q6, m, dout);
        download(ctx, out, dout, n_out);
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_warp_sample_device(chiaro_depth_ctx *ctx, const chiaro_warp *warp, const float *xy, uint64_t n,
                              float *mapped, float *confidence) {
    if (!ctx || !warp || !warp->points || !mapped || (n && !xy)) return CHIARO_ERR_ARGUMENT;
    if (warp->step == 0 || warp->columns == 0 || warp->rows == 0 || warp->columns > INT32_MAX ||
        warp->rows > INT32_MAX || warp->step > INT32_MAX)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        if (n == 0) return CHIARO_OK;
        const WarpRef w{reinterpret_cast<const float2 *>(warp->points), (int)warp->step, (int)warp->columns,
                        (int)warp->rows};
        warp_sample_kernel<<<(unsigned)std::min<uint64_t>(div_ceil((size_t)n, 256), (uint64_t)ctx->sm_count * 16), 256,
                             0, ctx->stream>>>(w, warp->confidence, reinterpret_cast<const float2 *>(xy), (long)n,
                                               reinterpret_cast<float2 *>(mapped), confidence);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_depth_sample_nearest_device(chiaro_depth_ctx *ctx, const chiaro_depth_map *map, const float *xy,
                                       uint64_t n, double *depth, float *confidence, uint8_t *provenance,
                                       int64_t *node) {
    if (!ctx || !map || (n && !xy)) return CHIARO_ERR_ARGUMENT;
    if ((depth && !map->depth) || (confidence && !map->confidence) || (provenance && !map->provenance) ||
        map->columns > INT32_MAX || map->rows > INT32_MAX || map->step > INT32_MAX)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        if (n == 0) return CHIARO_OK;
        depth_sample_nearest_kernel<<<(unsigned)std::min<uint64_t>(div_ceil((size_t)n, 256), (uint64_t)ctx->sm_count * 16),
                                      256, 0, ctx->stream>>>(map->depth, map->confidence, map->provenance,
                                                             (int)map->columns, (int)map->rows, (int)map->step,
                                                             reinterpret_cast<const float2 *>(xy), (long)n, depth,
                                                             confidence, provenance,
                                                             reinterpret_cast<long long *>(node));
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->stream));
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
    return CHIARO_OK;
}

int chiaro_refine_resolution_warp_device(chiaro_depth_ctx *ctx, const float *reference, uint64_t reference_width,
                                         uint64_t reference_height, const float *target, uint64_t target_width,
                                         uint64_t target_height, const chiaro_warp *base, uint64_t width,
                                         uint64_t height, chiaro_warp *out, chiaro_resolution_report *report) {
    if (!ctx || !reference || !target || !base || !base->points || !out || !out->points || !report)
        return CHIARO_ERR_ARGUMENT;
    if (base->step == 0 || base->columns == 0 || base->rows == 0 || base->step > INT32_MAX ||
        base->columns > INT32_MAX || base->rows > INT32_MAX || reference_width > INT32_MAX ||
        reference_height > INT32_MAX || target_width > INT32_MAX || target_height > INT32_MAX ||
        width > INT32_MAX / 2 || height > INT32_MAX / 2)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        return run_resolution(ctx, reference, (int)reference_width, (int)reference_height, target, (int)target_width,
                              (int)target_height, *base, (int)width, (int)height, *out, *report);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

void chiaro_align_options_default(chiaro_align_options *options) {
    if (!options) return;
    *options = chiaro_align_options{32, 32, 12, 0.5f, 3.0f, 0.45f, 1};  // AlignOptions::default (align.rs:229-243)
}

int chiaro_align_module(chiaro_depth_ctx *ctx, const chiaro_align_input *reference, const chiaro_align_input *target,
                        int32_t target_is_reference, const chiaro_align_options *options, const chiaro_warp *seed,
                        chiaro_warp *out_warp, float *gain, chiaro_alignment_report *report) {
    if (!ctx || !reference || !target || !options || !out_warp || !out_warp->points || !gain || !report)
        return CHIARO_ERR_ARGUMENT;
    if (!reference->luminance || !target->luminance || options->grid_step == 0 || options->patch == 0 ||
        reference->width > INT32_MAX / 2 || reference->height > INT32_MAX / 2 || reference->luma_width > INT32_MAX ||
        reference->luma_height > INT32_MAX || target->luma_width > INT32_MAX || target->luma_height > INT32_MAX ||
        options->patch > 4096 || options->coarse_radius > 4096 || options->grid_step > INT32_MAX ||
        (seed && (!seed->points || seed->step == 0 || seed->columns == 0 || seed->rows == 0 ||
                  seed->step > INT32_MAX || seed->columns > INT32_MAX || seed->rows > INT32_MAX)))
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        return run_align(ctx, *reference, *target, target_is_reference != 0, *options, seed, *out_warp, *gain,
                         *report);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    } catch (const align_host::Failure &e) {
        ctx->error = e.message;
        return CHIARO_INVALID;
    }
}

int chiaro_refine_resolution_warp(chiaro_depth_ctx *ctx, const float *reference, uint64_t reference_width,
                                  uint64_t reference_height, const float *target, uint64_t target_width,
                                  uint64_t target_height, const chiaro_warp *base, uint64_t width, uint64_t height,
                                  chiaro_warp *out, chiaro_resolution_report *report) {
    if (!ctx || !reference || !target || !base || !base->points || !out || !out->points || !report)
        return CHIARO_ERR_ARGUMENT;
    if (base->step == 0 || base->columns == 0 || base->rows == 0 || base->step > INT32_MAX ||
        base->columns > INT32_MAX || base->rows > INT32_MAX || reference_width > INT32_MAX ||
        reference_height > INT32_MAX || target_width > INT32_MAX || target_height > INT32_MAX ||
        width > INT32_MAX / 2 || height > INT32_MAX / 2)
        return CHIARO_ERR_ARGUMENT;
    try {
        CK(cudaSetDevice(ctx->device));
        const size_t nr = (size_t)reference_width * reference_height, nt = (size_t)target_width * target_height;
        float *dr = dbuf<float>(ctx, "res.reference", std::max<size_t>(nr, 1));
        float *dt = dbuf<float>(ctx, "res.target", std::max<size_t>(nt, 1));
        if (nr) upload(ctx, dr, reference, nr);
        if (nt) upload(ctx, dt, target, nt);
        return run_resolution(ctx, dr, (int)reference_width, (int)reference_height, dt, (int)target_width,
                              (int)target_height, *base, (int)width, (int)height, *out, *report);
    } catch (const CudaError &e) {
        return fail(ctx, e);
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Allocation-free form of the connected-components filter.
//
// Some callers cannot allocate device memory: a host that hands this library a
// fixed memory budget (an embedded or real-time pipeline), a plugin running
// inside a framework that owns the allocator, or code building a CUDA graph
// around its own buffers. This entry point takes the caller's device buffers
// for inputs and output and keeps the union-find scratch (parent and component
// size per node) in a file-scope device array, so it calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// The array holds NOALLOC_MAX_NODES nodes (2 x 4 MiB, plus a status word); every
// GPU that loads the library keeps it until the process exits. All calls share
// it, so calls that overlap on the GPU (different streams, or host threads)
// race; the scratch keeps the previous call's contents and is reinitialised on
// every call. Its device address is looked up once per device index and kept:
// after cudaDeviceReset the kept address is stale, so the entry point must not
// be used across a device reset.
// ---------------------------------------------------------------------------------
namespace {

constexpr uint64_t NOALLOC_MAX_NODES = 1u << 20;

static __device__ __align__(256) int g_component_scratch[2 * NOALLOC_MAX_NODES + 64];  // [parent | size | status]

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_scratch_mutex;
int *g_scratch_address[NOALLOC_MAX_DEVICES] = {};

// Device address of g_component_scratch on the current device, looked up once
// per device with that device current (the host-side symbol is only a stand-in).
cudaError_t component_scratch(int **out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_component_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_address[device] = static_cast<int *>(p);
    }
    *out = g_scratch_address[device];
    return cudaSuccess;
}

}  // namespace

extern "C" int chiaro_reject_small_components_noalloc(void *stream, const uint8_t *has, const double *depth,
                                                      const float *guidance, uint64_t columns, uint64_t rows,
                                                      double inverse_tolerance, uint64_t minimum_nodes,
                                                      uint8_t *has_out) {
    if (!has || !depth || !guidance || !has_out || columns < 1 || rows < 1) return CHIARO_ERR_ARGUMENT;
    // each side first, so that the product below cannot wrap
    if (columns > NOALLOC_MAX_NODES || rows > NOALLOC_MAX_NODES) return CHIARO_ERR_CAPACITY;
    const uint64_t n = columns * rows;
    if (n > NOALLOC_MAX_NODES) return CHIARO_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (minimum_nodes <= 1) {  // depth.rs:941-943: nothing is removed
        return cudaMemcpyAsync(has_out, has, n, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? CHIARO_OK
                                                                                              : CHIARO_ERR_CUDA;
    }
    int *scratch = nullptr;
    if (component_scratch(&scratch) != cudaSuccess) return CHIARO_ERR_CUDA;
    int *parent = scratch, *size = scratch + NOALLOC_MAX_NODES, *status = scratch + 2 * NOALLOC_MAX_NODES;
    const unsigned blocks = blocks_for(n, 256);
    components_init_kernel<<<blocks, 256, 0, s>>>(parent, (int)n);
    if (cudaMemsetAsync(size, 0, n * sizeof(int), s) != cudaSuccess) return CHIARO_ERR_CUDA;
    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess) return CHIARO_ERR_CUDA;
    // n + 1 retries: a join cannot run out (see uf_union), so the status word stays clear
    components_union_kernel<<<blocks, 256, 0, s>>>(has, depth, guidance, parent, (int)columns, (int)rows,
                                                   inverse_tolerance, (int)n + 1, status);
    components_size_kernel<<<blocks, 256, 0, s>>>(has, parent, size, (int)n);
    components_mark_kernel<<<blocks, 256, 0, s>>>(has, parent, size, has_out, (int)n,
                                                  (int)std::min<uint64_t>(minimum_nodes, INT32_MAX));
    return cudaGetLastError() == cudaSuccess ? CHIARO_OK : CHIARO_ERR_CUDA;
}
