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
// The convolutions are implicit GEMMs on the tensor cores with mma.sync
// m16n8k16 (bf16 in, fp32 accumulate): a warp owns 16 consecutive pixels of a
// row and all 32 output channels (four n8 tiles), and walks K = 9 taps x 32
// input channels in 18 steps, gathering each A fragment straight from the NHWC
// input (zero outside the image) as 32-bit pairs of channels. The data gradient
// is the same kernel with the weights transposed and the taps mirrored, its
// epilogue masking by the previous layer's ReLU. The weight gradient is a GEMM
// over pixels (M = co, N = ci, K = pixels) per tap, accumulated in fp32 with
// atomics. These GEMMs are small (M ~ 10^4-10^5 pixels, N = 32, K = 288): a
// layer takes microseconds, bound by latency rather than by tensor throughput.
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

__device__ __forceinline__ unsigned ld_pair(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const unsigned *>(p);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&v);
}

__device__ __forceinline__ unsigned pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

// Input features of one node: the reference luminance at the node (guidance / 8);
// per bin of the finite labels, the bin's minimum cost minus the node's; the
// first cost argmin over the finite labels, as (argmin - 1) / (labels - 2); and
// the node's minimum cost.
__global__ void net_features_kernel(const float *__restrict__ costs, const float *__restrict__ guidance, int nodes,
                                    int labels, __nv_bfloat16 *__restrict__ features) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nodes) return;
    const float *c = costs + (size_t)node * labels;
    float bins[NET_BINS];
    float lowest = INFINITY;
    int argmin = 1;
    const int finite = labels - 1;
    for (int b = 0; b < NET_BINS; ++b) {
        const int l0 = 1 + b * finite / NET_BINS, l1 = 1 + (b + 1) * finite / NET_BINS;
        float m = INFINITY;
        for (int l = l0; l < l1; ++l) {
            const float v = c[l];
            if (v < lowest) {
                lowest = v;
                argmin = l;
            }
            m = fminf(m, v);
        }
        bins[b] = m;
    }
    __nv_bfloat16 *f = features + (size_t)node * NET_CH;
    f[0] = __float2bfloat16_rn(guidance[node] * 0.125f);
    for (int b = 0; b < NET_BINS; ++b) f[1 + b] = __float2bfloat16_rn(bins[b] - lowest);
    f[NET_INPUTS - 2] = __float2bfloat16_rn((float)(argmin - 1) / (float)(labels - 2));
    f[NET_INPUTS - 1] = __float2bfloat16_rn(lowest);
    for (int k = NET_INPUTS; k < NET_CH; ++k) f[k] = __float2bfloat16_rn(0.0f);
}

// out[p][co] = sum_{tap, ci} in[p + tap][ci] * w[tap][co][ci] + bias[co]; then ReLU
// (relu), or the mask of a previous activation (mask: zero where mask <= 0). out_f32,
// when given, receives channel 0 in fp32.
__global__ void __launch_bounds__(128) net_conv_kernel(const __nv_bfloat16 *__restrict__ in, int images, int height,
                                                       int width, const __nv_bfloat16 *__restrict__ w,
                                                       const float *__restrict__ bias, int relu,
                                                       const __nv_bfloat16 *__restrict__ mask,
                                                       __nv_bfloat16 *__restrict__ out, float *__restrict__ out_f32) {
    const int lane = threadIdx.x & 31;
    const int group = lane >> 2, tig = lane & 3;
    const int segments = (width + 15) / 16;
    const long tile = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile >= (long)images * height * segments) return;  // whole warp
    const int n = (int)(tile / ((long)height * segments));
    const int rest = (int)(tile - (long)n * height * segments);
    const int y = rest / segments, x0 = (rest - y * segments) * 16;
    const __nv_bfloat16 *image = in + (size_t)n * height * width * NET_CH;
    float acc[4][4] = {};
    for (int tap = 0; tap < NET_TAPS; ++tap) {
        const int yy = y + tap / 3 - 1, dx = tap % 3 - 1;
        const bool row_in = yy >= 0 && yy < height;
        const int xa = x0 + group + dx, xb = xa + 8;
        const bool in_a = row_in && xa >= 0 && xa < width, in_b = row_in && xb >= 0 && xb < width;
        const __nv_bfloat16 *pa = image + ((size_t)(row_in ? yy : 0) * width + (in_a ? xa : 0)) * NET_CH;
        const __nv_bfloat16 *pb = image + ((size_t)(row_in ? yy : 0) * width + (in_b ? xb : 0)) * NET_CH;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int ci = half * 16 + tig * 2;
            const unsigned a0 = in_a ? ld_pair(pa + ci) : 0u, a1 = in_b ? ld_pair(pb + ci) : 0u;
            const unsigned a2 = in_a ? ld_pair(pa + ci + 8) : 0u, a3 = in_b ? ld_pair(pb + ci + 8) : 0u;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const __nv_bfloat16 *wp = w + ((size_t)tap * NET_CH + nt * 8 + group) * NET_CH + ci;
                mma_bf16_16816(acc[nt], a0, a1, a2, a3, ld_pair(wp), ld_pair(wp + 8));
            }
        }
    }
    // epilogue: rows group (pixel x0 + group) and group + 8, columns co = nt * 8 + 2 tig + (0, 1)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int x = x0 + group + 8 * half;
        if (x >= width) continue;
        const size_t p = ((size_t)n * height + y) * width + x;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int co = nt * 8 + tig * 2;
            float v0 = acc[nt][2 * half] + (bias ? bias[co] : 0.0f);
            float v1 = acc[nt][2 * half + 1] + (bias ? bias[co + 1] : 0.0f);
            if (relu) {
                v0 = fmaxf(v0, 0.0f);
                v1 = fmaxf(v1, 0.0f);
            }
            if (mask) {
                const __nv_bfloat16 *m = mask + p * NET_CH + co;
                if (!(__bfloat162float(m[0]) > 0.0f)) v0 = 0.0f;
                if (!(__bfloat162float(m[1]) > 0.0f)) v1 = 0.0f;
            }
            *reinterpret_cast<unsigned *>(out + p * NET_CH + co) = pack_bf16(v0, v1);
            if (out_f32 && co == 0) out_f32[p] = v0;
        }
    }
}

// dW[tap][co][ci] += sum_p dpre[p][co] * in[p + tap][ci] over a chunk of pixels (K):
// M = co (two m16 tiles), N = ci (four n8 tiles). A warp owns (tap, chunk of 16 x
// NET_WGRAD_STEPS pixels); pixels are the flattened (image, y, x) index.
constexpr int NET_WGRAD_STEPS = 16;

__device__ __forceinline__ __nv_bfloat16 net_at(const __nv_bfloat16 *act, long q, int dy, int dx, int height,
                                                int width, long total, int ch) {
    if (q >= total) return __float2bfloat16_rn(0.0f);
    const long hw = (long)height * width;
    const long n = q / hw;
    const int rem = (int)(q - n * hw), y = rem / width + dy, x = rem % width + dx;
    if (y < 0 || y >= height || x < 0 || x >= width) return __float2bfloat16_rn(0.0f);
    return act[((n * hw) + (long)y * width + x) * NET_CH + ch];
}

__global__ void __launch_bounds__(128) net_wgrad_kernel(const __nv_bfloat16 *__restrict__ in,
                                                        const __nv_bfloat16 *__restrict__ dpre, int images,
                                                        int height, int width, float *__restrict__ dw) {
    const int lane = threadIdx.x & 31;
    const int group = lane >> 2, tig = lane & 3;
    const long total = (long)images * height * width;
    const long chunk_pixels = 16L * NET_WGRAD_STEPS;
    const long chunks = (total + chunk_pixels - 1) / chunk_pixels;
    const long job = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (job >= chunks * NET_TAPS) return;  // whole warp
    const int tap = (int)(job % NET_TAPS);
    const long q0 = (job / NET_TAPS) * chunk_pixels;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    float acc[2][4][4] = {};
    for (int step = 0; step < NET_WGRAD_STEPS; ++step) {
        const long qa = q0 + step * 16 + tig * 2;  // k = 2 tig, 2 tig + 1; then + 8
        unsigned a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int co = mt * 16 + group;
            a[mt][0] = pack_raw(net_at(dpre, qa, 0, 0, height, width, total, co),
                                net_at(dpre, qa + 1, 0, 0, height, width, total, co));
            a[mt][1] = pack_raw(net_at(dpre, qa, 0, 0, height, width, total, co + 8),
                                net_at(dpre, qa + 1, 0, 0, height, width, total, co + 8));
            a[mt][2] = pack_raw(net_at(dpre, qa + 8, 0, 0, height, width, total, co),
                                net_at(dpre, qa + 9, 0, 0, height, width, total, co));
            a[mt][3] = pack_raw(net_at(dpre, qa + 8, 0, 0, height, width, total, co + 8),
                                net_at(dpre, qa + 9, 0, 0, height, width, total, co + 8));
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int ci = nt * 8 + group;
            const unsigned b0 = pack_raw(net_at(in, qa, dy, dx, height, width, total, ci),
                                         net_at(in, qa + 1, dy, dx, height, width, total, ci));
            const unsigned b1 = pack_raw(net_at(in, qa + 8, dy, dx, height, width, total, ci),
                                         net_at(in, qa + 9, dy, dx, height, width, total, ci));
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma_bf16_16816(acc[mt][nt], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b0, b1);
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
