// bandnet.cuh — the learned band proposal of the banded SGM. The reference has no
// learned model; this is the design's small convolutional network, trained on
// the GPU from the exact SGM's winners.
//
// Layout: activations NHWC bf16 [images][H][W][32] over the coarse grid (one
// pixel per coarse node), weights bf16 [layer][tap][co][ci] (tap = 3 * (dy + 1) +
// dx + 1), fp32 master parameters and gradients. Six 3x3 convolutions 32 -> 32,
// ReLU after the first five; channel 0 of the last is the node's label centre,
// normalised to [0, 1] over the finite labels.
//
// The convolutions are implicit GEMMs on the 5th-generation tensor cores
// (net_conv_tc_kernel: tcgen05.mma, accumulator in tensor memory; below). The data
// gradient is the same kernel with the weights transposed and the taps mirrored,
// its epilogue masking by the previous layer's ReLU. The weight gradient is a GEMM
// over pixels (M = 32 output channels, N = 32 input channels, K = pixels) per tap,
// accumulated in fp32 with atomics, on mma.sync m16n8k16: its 32 rows are below the
// 64-row minimum of a tcgen05 tile.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace chiaro {

constexpr int NET_CH = 32;      // channels of every layer (inputs padded)
constexpr int NET_LAYERS = 6;
constexpr int NET_TAPS = 9;
constexpr int NET_W = NET_TAPS * NET_CH * NET_CH;  // weights per layer
constexpr int NET_PARAMS = NET_LAYERS * (NET_W + NET_CH);
constexpr int NET_BINS = 16;    // cost-summary bins
constexpr int NET_INPUTS = 1 + NET_BINS + 2;  // live input channels of layer 0

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                               unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&v);
}

// The band proposal's sampled labels: 16 finite labels spread evenly over
// 1..labels-1, the first and the last included.
__host__ __device__ inline int net_sample_label(int b, int labels) { return 1 + (b * (labels - 2) + 7) / 15; }

// Input features of one node: the reference luminance at the node (guidance / 8);
// the costs of the 16 sampled labels minus the lowest of them; the first sampled
// label holding that lowest cost, as (label - 1) / (labels - 2); and the lowest cost.
// Rows of `costs` hold `stride` values: the full volume (stride == labels, a label's
// cost at its index) or the pre-pass's compact rows (label 0, then the sampled labels
// in order). A warp per node: lane b < 16 reads sampled label b; the minimum and its
// first label come from shuffles; lane k writes channel k.
__global__ void net_features_kernel(const float *__restrict__ costs, int stride, const float *__restrict__ guidance,
                                    int nodes, int labels, __nv_bfloat16 *__restrict__ features) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int node = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (node >= nodes) return;  // whole warp
    const int label = lane < NET_BINS ? net_sample_label(lane, labels) : labels;
    const float v = lane < NET_BINS ? __ldg(costs + (size_t)node * stride + (stride == labels ? label : 1 + lane))
                                    : INFINITY;
    float lowest = v;
    int argmin = label;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(full, lowest, off);
        const int oa = __shfl_xor_sync(full, argmin, off);
        if (ov < lowest || (ov == lowest && oa < argmin)) {
            lowest = ov;
            argmin = oa;
        }
    }
    if (argmin == labels) argmin = 1;  // every sampled cost NaN: the first label
    const float bin = __shfl_sync(full, v, (lane + 31) & 31);  // lane 1 + b: sampled label b
    float value = 0.0f;
    if (lane == 0) value = guidance[node] * 0.125f;
    if (lane >= 1 && lane <= NET_BINS) value = bin - lowest;
    if (lane == NET_INPUTS - 2) value = (float)(argmin - 1) / (float)(labels - 2);
    if (lane == NET_INPUTS - 1) value = lowest;
    features[(size_t)node * NET_CH + lane] = __float2bfloat16_rn(value);
}

// ---- the convolution on the 5th-generation tensor cores (tcgen05) ------------------------
// An implicit GEMM per tile of 128 consecutive pixels of one image row: M = 128 pixels,
// N = 32 output channels, K = 9 taps x 32 input channels, as 18 tcgen05.mma of kind::f16
// (bf16 operands, fp32 accumulator in tensor memory, 128 lanes x 32 columns). Both operands
// sit in shared memory in the canonical K-major layout without swizzle: 16-byte rows of 8
// channels, 8-row groups 128 bytes apart (SBO), the two 8-channel halves of a 16-deep K step
// LBO apart. The staged input holds, per window row and 8-channel block, 130 pixels (the
// tile and one on each side) in consecutive 16-byte rows, so a tap's pixel shift moves the
// A descriptor's start by 16 bytes and no shifted copy is made. The layer's weights are
// staged once per persistent CTA as [tap][channel block][co][8]. One thread issues the MMAs
// and commits them to an mbarrier; the CTA waits on it (a bounded wait: a run-out sets the
// status word and the CTA frees its tensor memory and returns), then each warp reads its
// 32 accumulator lanes (tcgen05.ld 32x32b), adds the bias, applies ReLU or the mask and
// stores bf16 (and channel 0 in fp32 for the last layer).
constexpr int NET_TC_M = 128;   // pixels per tile (accumulator lanes)
constexpr int NET_TC_PP = 136;  // staged pixels per window row and channel block (130 used)
constexpr size_t NET_TC_W_BYTES = (size_t)NET_TAPS * 4 * NET_CH * 16;
constexpr size_t NET_TC_IN_BYTES = (size_t)3 * 4 * NET_TC_PP * 16;
constexpr size_t NET_TC_SMEM = NET_TC_W_BYTES + NET_TC_IN_BYTES;
// instruction descriptor: fp32 accumulator (bits 4-5), bf16 A and B (bits 7-9, 10-12),
// both K-major, N >> 3 (bits 17-22), M >> 4 (bits 24-28)
constexpr uint32_t NET_TC_IDESC =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NET_CH >> 3) << 17) | ((uint32_t)(NET_TC_M >> 4) << 24);
constexpr long NET_TC_SPIN = 1L << 22;  // polls of the MMA barrier (each a bounded try_wait) before giving up
constexpr int NET_TC_GAVE_UP = 1;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t address, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((address >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(NET_TC_IDESC), "r"(accumulate), "r"(0u));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

// Bounded wait for the MMA barrier's phase: true when it completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase) {
    for (long spin = 0; spin < NET_TC_SPIN; ++spin)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__global__ void __launch_bounds__(NET_TC_M) net_conv_tc_kernel(
    const __nv_bfloat16 *__restrict__ in, int images, int height, int width, const __nv_bfloat16 *__restrict__ w,
    const float *__restrict__ bias, int relu, const __nv_bfloat16 *__restrict__ mask, __nv_bfloat16 *__restrict__ out,
    float *__restrict__ out_f32, int *status) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned char *wsm = tc_smem, *insm = tc_smem + NET_TC_W_BYTES;
    const uint32_t w_addr = smem_u32(wsm), in_addr = smem_u32(insm), bar = smem_u32(&mma_bar);
    // the layer's weights w[tap][co][ci] as [tap][channel block][co][8 channels]
    for (int c = tid; c < NET_TAPS * NET_CH * 4; c += NET_TC_M) {
        const int row = c >> 2, j = c & 3, tap = row / NET_CH, co = row - tap * NET_CH;
        *reinterpret_cast<uint4 *>(wsm + (((size_t)tap * 4 + j) * NET_CH + co) * 16) =
            *reinterpret_cast<const uint4 *>(w + (size_t)row * NET_CH + j * 8);
    }
    if (warp == 0) {  // 32 columns of tensor memory: the 128 x 32 fp32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(32u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_slot;
    const int segments = (width + NET_TC_M - 1) / NET_TC_M;
    const long tiles = (long)images * height * segments;
    uint32_t phase = 0;
    bool failed = false;
    for (long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int n = (int)(tile / ((long)height * segments));
        const int rest = (int)(tile - (long)n * height * segments);
        const int y = rest / segments, x0 = (rest - y * segments) * NET_TC_M;
        const __nv_bfloat16 *image = in + (size_t)n * height * width * NET_CH;
        // the window: rows y - 1 .. y + 1, pixels x0 - 1 .. x0 + 128, zero outside the image
        for (int c = tid; c < 3 * 130 * 4; c += NET_TC_M) {
            const int j = c & 3, px = (c >> 2) % 130, r = (c >> 2) / 130;
            const int xx = x0 - 1 + px, yy = y - 1 + r;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < height && xx >= 0 && xx < width)
                v = *reinterpret_cast<const uint4 *>(image + ((size_t)yy * width + xx) * NET_CH + j * 8);
            *reinterpret_cast<uint4 *>(insm + (((size_t)r * 4 + j) * NET_TC_PP + px) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
            for (int tap = 0; tap < NET_TAPS; ++tap) {
                const int r = tap / 3, dx = tap % 3;
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    const uint64_t a = umma_desc(
                        in_addr + (uint32_t)((((r * 4 + 2 * half) * NET_TC_PP) + dx) * 16), NET_TC_PP * 16, 128);
                    const uint64_t b = umma_desc(w_addr + (uint32_t)(((tap * 4 + 2 * half) * NET_CH) * 16), NET_CH * 16,
                                                 128);
                    umma_bf16(tmem, a, b, (tap | half) != 0);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        // the MMAs are complete (their reads of the window too) once the barrier's phase flips
        failed = __syncthreads_or(!mbar_wait_bounded(bar, phase));
        if (failed) break;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint32_t acc[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(acc[0]), "=r"(acc[1]), "=r"(acc[2]), "=r"(acc[3]), "=r"(acc[4]), "=r"(acc[5]), "=r"(acc[6]),
              "=r"(acc[7]), "=r"(acc[8]), "=r"(acc[9]), "=r"(acc[10]), "=r"(acc[11]), "=r"(acc[12]), "=r"(acc[13]),
              "=r"(acc[14]), "=r"(acc[15]), "=r"(acc[16]), "=r"(acc[17]), "=r"(acc[18]), "=r"(acc[19]),
              "=r"(acc[20]), "=r"(acc[21]), "=r"(acc[22]), "=r"(acc[23]), "=r"(acc[24]), "=r"(acc[25]),
              "=r"(acc[26]), "=r"(acc[27]), "=r"(acc[28]), "=r"(acc[29]), "=r"(acc[30]), "=r"(acc[31])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int x = x0 + tid;  // this thread's accumulator lane is pixel x0 + tid
        if (x < width) {
            const size_t p = ((size_t)n * height + y) * width + x;
            unsigned packed[16];
#pragma unroll
            for (int co = 0; co < NET_CH; co += 2) {
                float v0 = __uint_as_float(acc[co]) + (bias ? bias[co] : 0.0f);
                float v1 = __uint_as_float(acc[co + 1]) + (bias ? bias[co + 1] : 0.0f);
                if (relu) {
                    v0 = fmaxf(v0, 0.0f);
                    v1 = fmaxf(v1, 0.0f);
                }
                if (mask) {
                    const __nv_bfloat16 *m = mask + p * NET_CH + co;
                    if (!(__bfloat162float(m[0]) > 0.0f)) v0 = 0.0f;
                    if (!(__bfloat162float(m[1]) > 0.0f)) v1 = 0.0f;
                }
                if (co == 0 && out_f32) out_f32[p] = v0;
                packed[co / 2] = pack_bf16(v0, v1);
            }
            uint4 *dst = reinterpret_cast<uint4 *>(out + p * NET_CH);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                dst[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();  // every warp has read the accumulator before the next tile's MMAs
    }
    if (failed) {
        if (tid == 0) atomicOr(status, NET_TC_GAVE_UP);
        mbar_wait_bounded(bar, phase);  // give MMAs still in flight a last bounded wait
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u));
}

// Shared-memory rows of the weight gradient: 32 bf16 channels padded to 40 (80 bytes), so
// the eight 16-byte rows an ldmatrix reads fall in distinct banks.
constexpr int NET_SROW = 40;

// dW[tap][co][ci] += sum_p dpre[p][co] * in[p + tap][ci] over a chunk of pixels (K):
// M = co (two m16 tiles), N = ci (four n8 tiles). A warp owns (tap, chunk of 16 x
// NET_WGRAD_STEPS pixels); pixels are the flattened (image, y, x) index.
constexpr int NET_WGRAD_STEPS = 16;

__device__ __forceinline__ void ldmatrix_x4_trans(unsigned (&r)[4], const __nv_bfloat16 *p) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// Per step, two lanes stage one of the 16 pixels: its gradient row dpre[q][*] and its
// tap neighbour's input row in[q + tap][*] (zero outside the image or past the last
// pixel), 16 bytes at a time, into shared rows of NET_SROW; ldmatrix.trans then reads
// both as k-major (pixel) fragments.
__global__ void __launch_bounds__(128) net_wgrad_kernel(const __nv_bfloat16 *__restrict__ in,
                                                        const __nv_bfloat16 *__restrict__ dpre, int images,
                                                        int height, int width, float *__restrict__ dw) {
    __shared__ __align__(16) __nv_bfloat16 stage[4][2][16 * NET_SROW];  // [warp][dpre, in][pixel][channel]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int group = lane >> 2, tig = lane & 3;
    const long total = (long)images * height * width;
    const long chunk_pixels = 16L * NET_WGRAD_STEPS;
    const long chunks = (total + chunk_pixels - 1) / chunk_pixels;
    const long job = (long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (job >= chunks * NET_TAPS) return;  // whole warp; no block barrier follows
    const int tap = (int)(job % NET_TAPS);
    const long q0 = (job / NET_TAPS) * chunk_pixels;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    __nv_bfloat16 *ds = stage[warp][0], *xs = stage[warp][1];
    const long hw = (long)height * width;
    const int mj = lane >> 3, mr = lane & 7;
    const int pixel = lane >> 1, part = (lane & 1) * 2;  // this lane's staged pixel and 16-byte parts
    float acc[2][4][4] = {};
    for (int step = 0; step < NET_WGRAD_STEPS; ++step) {
        const long q = q0 + step * 16 + pixel;
        uint4 d0 = make_uint4(0u, 0u, 0u, 0u), d1 = d0, x0 = d0, x1 = d0;
        if (q < total) {
            const __nv_bfloat16 *dp = dpre + q * NET_CH + part * 8;
            d0 = *reinterpret_cast<const uint4 *>(dp);
            d1 = *reinterpret_cast<const uint4 *>(dp + 8);
            const long n = q / hw;
            const int rem = (int)(q - n * hw), y = rem / width + dy, x = rem % width + dx;
            if (y >= 0 && y < height && x >= 0 && x < width) {
                const __nv_bfloat16 *xp = in + ((n * hw) + (long)y * width + x) * NET_CH + part * 8;
                x0 = *reinterpret_cast<const uint4 *>(xp);
                x1 = *reinterpret_cast<const uint4 *>(xp + 8);
            }
        }
        __syncwarp();  // the previous step's fragments are read
        *reinterpret_cast<uint4 *>(ds + pixel * NET_SROW + part * 8) = d0;
        *reinterpret_cast<uint4 *>(ds + pixel * NET_SROW + part * 8 + 8) = d1;
        *reinterpret_cast<uint4 *>(xs + pixel * NET_SROW + part * 8) = x0;
        *reinterpret_cast<uint4 *>(xs + pixel * NET_SROW + part * 8 + 8) = x1;
        __syncwarp();
        // A (co x pixels) of m-tile mt: matrices (pixels 0-7 | 8-15) x (co m0 | m0 + 8), a0..a3
        unsigned a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
            ldmatrix_x4_trans(a[mt], ds + ((mj >> 1) * 8 + mr) * NET_SROW + mt * 16 + (mj & 1) * 8);
#pragma unroll
        for (int np = 0; np < 2; ++np) {
            unsigned b[4];  // b0, b1 of n-tile 2 np, then of 2 np + 1 (pixels 0-7 | 8-15)
            ldmatrix_x4_trans(b, xs + ((mj & 1) * 8 + mr) * NET_SROW + (2 * np + (mj >> 1)) * 8);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                mma_bf16_16816(acc[mt][2 * np], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b[0], b[1]);
                mma_bf16_16816(acc[mt][2 * np + 1], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b[2], b[3]);
            }
        }
    }
    // C rows: co = mt * 16 + group (+ 8); columns: ci = nt * 8 + 2 tig (+ 1)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int co = mt * 16 + group + (r >= 2 ? 8 : 0), ci = nt * 8 + tig * 2 + (r & 1);
                atomicAdd(dw + ((size_t)tap * NET_CH + co) * NET_CH + ci, acc[mt][nt][r]);
            }
}

// db[co] += sum_p dpre[p][co]: a thread per (pixel, channel), a shared partial per block.
__global__ void net_bias_grad_kernel(const __nv_bfloat16 *__restrict__ dpre, long pixels, float *__restrict__ db) {
    __shared__ float partial[NET_CH];
    if (threadIdx.x < NET_CH) partial[threadIdx.x] = 0.0f;
    __syncthreads();
    const int ch = threadIdx.x % NET_CH;
    float s = 0.0f;
    for (long p = (long)blockIdx.x * (blockDim.x / NET_CH) + threadIdx.x / NET_CH; p < pixels;
         p += (long)gridDim.x * (blockDim.x / NET_CH))
        s += __bfloat162float(dpre[p * NET_CH + ch]);
    atomicAdd(&partial[ch], s);
    __syncthreads();
    if (threadIdx.x < NET_CH) atomicAdd(&db[threadIdx.x], partial[threadIdx.x]);
}

// Huber loss (delta) of channel 0 against the targets on the masked pixels, and
// its gradient into dout (channel 0; the other channels zero). loss_sum and count
// accumulate over the launch.
__global__ void net_loss_kernel(const float *__restrict__ y, const float *__restrict__ target,
                                const uint8_t *__restrict__ mask, long pixels, float inverse_count, float delta,
                                __nv_bfloat16 *__restrict__ dout, float *loss_sum) {
    float s = 0.0f;
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += (long)gridDim.x * blockDim.x) {
        float g = 0.0f;
        if (mask[p]) {
            const float e = y[p] - target[p], a = fabsf(e);
            s += a <= delta ? 0.5f * e * e : delta * (a - 0.5f * delta);
            g = (a <= delta ? e : copysignf(delta, e)) * inverse_count;
        }
        __nv_bfloat16 *d = dout + p * NET_CH;
        d[0] = __float2bfloat16_rn(g);
        for (int k = 1; k < NET_CH; ++k) d[k] = __float2bfloat16_rn(0.0f);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, s * inverse_count);
}

// Adam on the fp32 parameters, then the bf16 weights for the forward pass and the
// transposed, mirrored copy for the data gradient (wt[layer][8 - tap][ci][co]).
__global__ void net_adam_kernel(float *__restrict__ params, const float *__restrict__ grads, float *__restrict__ m,
                                float *__restrict__ v, float lr, float beta1, float beta2, float eps, float bias1,
                                float bias2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NET_PARAMS) return;
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.0f - beta1) * g, vi = beta2 * v[i] + (1.0f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / bias1) / (sqrtf(vi / bias2) + eps);
}

__global__ void net_pack_kernel(const float *__restrict__ params, __nv_bfloat16 *__restrict__ w,
                                __nv_bfloat16 *__restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NET_LAYERS * NET_W) return;
    const int layer = i / NET_W, r = i - layer * NET_W;
    const int tap = r / (NET_CH * NET_CH), co = (r / NET_CH) % NET_CH, ci = r % NET_CH;
    const __nv_bfloat16 b = __float2bfloat16_rn(params[layer * (NET_W + NET_CH) + r]);
    w[i] = b;
    wt[(size_t)layer * NET_W + ((size_t)(NET_TAPS - 1 - tap) * NET_CH + ci) * NET_CH + co] = b;
}

// Per tile of tile x tile nodes: the mean of the nodes' predicted centres (label units),
// and the offset that centres the band on it, clamped to [1, labels - band].
__global__ void net_tile_offsets_kernel(const float *__restrict__ y, int columns, int rows, int labels, int tile,
                                        int band, int *__restrict__ offsets) {
    const int tiles_x = (columns + tile - 1) / tile, tiles_y = (rows + tile - 1) / tile;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles_x * tiles_y) return;
    const int tx = t % tiles_x, ty = t / tiles_x;
    float s = 0.0f;
    int n = 0;
    for (int r = ty * tile; r < min(rows, (ty + 1) * tile); ++r)
        for (int c = tx * tile; c < min(columns, (tx + 1) * tile); ++c) {
            s += y[(size_t)r * columns + c];
            ++n;
        }
    const float centre = 1.0f + (s / (float)n) * (float)(labels - 2);
    const int o = (int)rintf(centre) - band / 2;
    offsets[t] = max(1, min(labels - band, o));
}

}  // namespace chiaro
