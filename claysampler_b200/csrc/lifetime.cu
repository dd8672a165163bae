// Note-lifetime predictor: inference, fused training step and the label reduction
// over rendered single-note mixes (include/claysampler_lifetime.h).
//
// The network is small (16 -> 64 -> 64 -> 2, about 5.3k multiply-adds per
// sample), so a kernel is bound by its launch and by shared-memory traffic, not by
// the FP32 pipe: inference is one thread per sample with the BF16-rounded weights
// staged once per CTA in shared memory (every thread reads the same weight at the
// same time, a broadcast), and the gradient keeps a CTA's 128 samples' activations
// and deltas in shared memory, where the weight gradients are formed as fixed-order
// sums over the samples (one partial row per CTA, added in CTA order by the
// update kernel: deterministic, no atomics).
#include "../../include/claysampler_lifetime.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <stdexcept>
#include <string>

namespace {

constexpr int F = CS_LIFETIME_FEATURES;
constexpr int H = CS_LIFETIME_HIDDEN;
constexpr int O = CS_LIFETIME_OUTPUTS;
constexpr int P = CS_LIFETIME_PARAMS;
constexpr int kRow = P + 1;                        // partial row: gradient, then loss
constexpr int kSamples = CS_LIFETIME_BLOCK_SAMPLES; // threads (= samples) per CTA
constexpr int kXStride = F + 1;                    // padded rows: no bank conflicts
constexpr int kHStride = H + 1;                    // when a thread walks its own row
static_assert(P == H * F + H + H * H + H + O * H + O, "parameter layout");

thread_local std::string lastError;

// Weights as the kernels use them: BF16 values (nearest-even) held as float.
struct Staged {
    float w1[H * F];
    float w2[H * H];
    float w3[O * H];
    float b1[H], b2[H], b3[O];
    float mean[F], invStd[F], targetMean[O], targetStd[O];
};

__device__ __forceinline__ float bf16(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }

__device__ void stage(Staged& s, const float* __restrict__ params, const float* __restrict__ norm)
{
    for (int i = threadIdx.x; i < H * F; i += blockDim.x)
        s.w1[i] = bf16(params[CS_LIFETIME_W1_AT + i]);
    for (int i = threadIdx.x; i < H * H; i += blockDim.x)
        s.w2[i] = bf16(params[CS_LIFETIME_W2_AT + i]);
    for (int i = threadIdx.x; i < O * H; i += blockDim.x)
        s.w3[i] = bf16(params[CS_LIFETIME_W3_AT + i]);
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        s.b1[i] = params[CS_LIFETIME_B1_AT + i];
        s.b2[i] = params[CS_LIFETIME_B2_AT + i];
    }
    if (threadIdx.x < O) {
        s.b3[threadIdx.x] = params[CS_LIFETIME_B3_AT + threadIdx.x];
        s.targetMean[threadIdx.x] = norm[2 * F + threadIdx.x];
        s.targetStd[threadIdx.x] = norm[2 * F + O + threadIdx.x];
    }
    if (threadIdx.x < F) {
        s.mean[threadIdx.x] = norm[threadIdx.x];
        s.invStd[threadIdx.x] = norm[F + threadIdx.x];
    }
}

// Standardised input row of sample `i` (16 floats = four 128-bit loads).
__device__ __forceinline__ void loadInput(const Staged& s, const float* __restrict__ x, int i, float (&in)[F])
{
    const float4* row = reinterpret_cast<const float4*>(x + size_t(i) * F);
#pragma unroll
    for (int q = 0; q < F / 4; ++q) {
        const float4 v = row[q];
        in[4 * q + 0] = (v.x - s.mean[4 * q + 0]) * s.invStd[4 * q + 0];
        in[4 * q + 1] = (v.y - s.mean[4 * q + 1]) * s.invStd[4 * q + 1];
        in[4 * q + 2] = (v.z - s.mean[4 * q + 2]) * s.invStd[4 * q + 2];
        in[4 * q + 3] = (v.w - s.mean[4 * q + 3]) * s.invStd[4 * q + 3];
    }
}

// Every sum starts from the bias and adds its terms in index order.
__global__ void __launch_bounds__(kSamples) forwardKernel(const float* __restrict__ params,
                                                          const float* __restrict__ norm,
                                                          const float* __restrict__ x, int n,
                                                          float* __restrict__ y)
{
    __shared__ Staged s;
    stage(s, params, norm);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float in[F];
    loadInput(s, x, i, in);
    float h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float a = s.b1[j];
#pragma unroll
        for (int f = 0; f < F; ++f)
            a = fmaf(s.w1[j * F + f], in[f], a);
        h1[j] = fmaxf(a, 0.f);
    }
    float out0 = s.b3[0], out1 = s.b3[1];
    for (int j = 0; j < H; ++j) {
        float a = s.b2[j];
#pragma unroll
        for (int k = 0; k < H; ++k)
            a = fmaf(s.w2[j * H + k], h1[k], a);
        a = fmaxf(a, 0.f);
        out0 = fmaf(s.w3[j], a, out0);
        out1 = fmaf(s.w3[H + j], a, out1);
    }
    y[2 * size_t(i) + 0] = fmaf(out0, s.targetStd[0], s.targetMean[0]);
    y[2 * size_t(i) + 1] = fmaf(out1, s.targetStd[1], s.targetMean[1]);
}

// ---- inference on the tensor cores --------------------------------------------------
//
// A warp takes 16 samples.  Layer 1 (16 -> 64) and layer 2 (64 -> 64) run as
// mma.sync m16n8k16 with BF16 operands and FP32 accumulation: the standardised
// inputs and the first layer's activations are rounded to BF16 where they enter a
// tensor-core product (the weights already are BF16).  The accumulator fragments of
// two neighbouring 8-column tiles of one layer hold exactly the A fragment of the
// next layer's 16-column step, so activations never leave registers.  Layer 3
// (64 -> 2) is a dot product per sample over the warp's fragments, reduced across
// the four lanes that share a row.

__device__ __forceinline__ uint32_t packBf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);     // .x = lo (low half)
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mmaBf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                 "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kTensorWarps = 4;                     // 64 samples per CTA

__global__ void __launch_bounds__(kTensorWarps * 32) forwardTensorKernel(const float* __restrict__ params,
                                                                         const float* __restrict__ norm,
                                                                         const float* __restrict__ x, int n,
                                                                         float* __restrict__ y)
{
    __shared__ Staged s;
    stage(s, params, norm);
    __syncthreads();
    const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
    const int group = lane >> 2, quad = lane & 3;   // fragment row group and column pair
    const int rowBase = (blockIdx.x * kTensorWarps + warp) * 16;
    const int rows[2] = {rowBase + group, rowBase + group + 8};
    // Layer-1 A fragment: inputs (rows g, g+8; columns 2q, 2q+1, 2q+8, 2q+9).
    float in[2][4];
    for (int r = 0; r < 2; ++r) {
        const bool live = rows[r] < n;
        const float* row = x + size_t(live ? rows[r] : 0) * F;
        const int cols[4] = {2 * quad, 2 * quad + 1, 2 * quad + 8, 2 * quad + 9};
        for (int c = 0; c < 4; ++c)
            in[r][c] = live ? (row[cols[c]] - s.mean[cols[c]]) * s.invStd[cols[c]] : 0.f;
    }
    const uint32_t a1[4] = {packBf16(in[0][0], in[0][1]), packBf16(in[1][0], in[1][1]),
                            packBf16(in[0][2], in[0][3]), packBf16(in[1][2], in[1][3])};
    // Layer 1: 8 column tiles of 8 outputs.
    float h1[8][4];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int out = 8 * t + group;              // B column = output index
        const uint32_t b0 = packBf16(s.w1[out * F + 2 * quad], s.w1[out * F + 2 * quad + 1]);
        const uint32_t b1 = packBf16(s.w1[out * F + 2 * quad + 8], s.w1[out * F + 2 * quad + 9]);
        const float bias0 = s.b1[8 * t + 2 * quad], bias1 = s.b1[8 * t + 2 * quad + 1];
        h1[t][0] = bias0;
        h1[t][1] = bias1;
        h1[t][2] = bias0;
        h1[t][3] = bias1;
        mmaBf16(h1[t], a1, b0, b1);
#pragma unroll
        for (int c = 0; c < 4; ++c)
            h1[t][c] = fmaxf(h1[t][c], 0.f);
    }
    // Layer 2: 4 steps of 16 inputs (two layer-1 tiles each) x 8 output tiles.
    float h2[8][4];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const float bias0 = s.b2[8 * t + 2 * quad], bias1 = s.b2[8 * t + 2 * quad + 1];
        h2[t][0] = bias0;
        h2[t][1] = bias1;
        h2[t][2] = bias0;
        h2[t][3] = bias1;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t a[4] = {packBf16(h1[2 * k][0], h1[2 * k][1]), packBf16(h1[2 * k][2], h1[2 * k][3]),
                               packBf16(h1[2 * k + 1][0], h1[2 * k + 1][1]),
                               packBf16(h1[2 * k + 1][2], h1[2 * k + 1][3])};
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int out = 8 * t + group;
            const float* w = s.w2 + out * H + 16 * k;
            mmaBf16(h2[t], a, packBf16(w[2 * quad], w[2 * quad + 1]), packBf16(w[2 * quad + 8], w[2 * quad + 9]));
        }
    }
    // Layer 3: the lane's partial sums for rows g and g+8, then across the quad.
    float part[2][O] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = 8 * t + 2 * quad + (c & 1);
            const float a = fmaxf(h2[t][c], 0.f);
            part[c >> 1][0] = fmaf(s.w3[j], a, part[c >> 1][0]);
            part[c >> 1][1] = fmaf(s.w3[H + j], a, part[c >> 1][1]);
        }
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int o = 0; o < O; ++o) {
            part[r][o] += __shfl_xor_sync(0xffffffffu, part[r][o], 1);
            part[r][o] += __shfl_xor_sync(0xffffffffu, part[r][o], 2);
        }
    if (quad == 0)
        for (int r = 0; r < 2; ++r)
            if (rows[r] < n)
                for (int o = 0; o < O; ++o)
                    y[2 * size_t(rows[r]) + o] = fmaf(part[r][o] + s.b3[o], s.targetStd[o], s.targetMean[o]);
}

constexpr size_t kGradientSmem =
    sizeof(Staged) + sizeof(float) * (size_t(kSamples) * (kXStride + 4 * kHStride + O) + kSamples);

// Forward and backward for one CTA of 128 samples; writes the CTA's partial row
// (dL/dparams summed over its samples in sample order, then its loss).
__global__ void __launch_bounds__(kSamples) gradientKernel(const float* __restrict__ params,
                                                           const float* __restrict__ norm,
                                                           const float* __restrict__ x,
                                                           const float* __restrict__ t, int n, float invCount,
                                                           float* __restrict__ partials)
{
    extern __shared__ __align__(16) float smem[];
    Staged& s = *reinterpret_cast<Staged*>(smem);
    float* X = smem + sizeof(Staged) / sizeof(float);   // [128][17] standardised inputs
    float* A1 = X + kSamples * kXStride;                // [128][65] first-layer activations
    float* A2 = A1 + kSamples * kHStride;               // [128][65] second-layer activations
    float* D2 = A2 + kSamples * kHStride;               // [128][65] dL/dz2
    float* D1 = D2 + kSamples * kHStride;               // [128][65] dL/dz1
    float* DY = D1 + kSamples * kHStride;               // [128][2]  dL/dy
    float* lossOf = DY + kSamples * O;                  // [128]
    stage(s, params, norm);
    __syncthreads();

    const int me = threadIdx.x;
    const int i = blockIdx.x * kSamples + me;
    const bool live = i < n;
    float in[F];
    if (live) {
        loadInput(s, x, i, in);
    } else {
#pragma unroll
        for (int f = 0; f < F; ++f)
            in[f] = 0.f;
    }
#pragma unroll
    for (int f = 0; f < F; ++f)
        X[me * kXStride + f] = in[f];
    for (int j = 0; j < H; ++j) {
        float a = s.b1[j];
#pragma unroll
        for (int f = 0; f < F; ++f)
            a = fmaf(s.w1[j * F + f], in[f], a);
        A1[me * kHStride + j] = fmaxf(a, 0.f);
    }
    float out0 = s.b3[0], out1 = s.b3[1];
    for (int j = 0; j < H; ++j) {
        float a = s.b2[j];
        for (int k = 0; k < H; ++k)
            a = fmaf(s.w2[j * H + k], A1[me * kHStride + k], a);
        a = fmaxf(a, 0.f);
        A2[me * kHStride + j] = a;
        out0 = fmaf(s.w3[j], a, out0);
        out1 = fmaf(s.w3[H + j], a, out1);
    }
    float d0 = 0.f, d1 = 0.f, loss = 0.f;
    if (live) {
        const float t0 = (t[2 * size_t(i) + 0] - s.targetMean[0]) / s.targetStd[0];
        const float t1 = (t[2 * size_t(i) + 1] - s.targetMean[1]) / s.targetStd[1];
        const float e0 = out0 - t0, e1 = out1 - t1;
        d0 = e0 * invCount;
        d1 = e1 * invCount;
        loss = (e0 * e0 + e1 * e1) * (0.5f * invCount);
    }
    DY[me * O + 0] = d0;
    DY[me * O + 1] = d1;
    lossOf[me] = loss;
    for (int j = 0; j < H; ++j) {
        const float g = s.w3[j] * d0 + s.w3[H + j] * d1;
        D2[me * kHStride + j] = A2[me * kHStride + j] > 0.f ? g : 0.f;
    }
    for (int k = 0; k < H; ++k) {
        float a = 0.f;
        for (int j = 0; j < H; ++j)
            a = fmaf(s.w2[j * H + k], D2[me * kHStride + j], a);
        D1[me * kHStride + k] = A1[me * kHStride + k] > 0.f ? a : 0.f;
    }
    __syncthreads();

    // Weight gradients: entry e of the parameter vector, summed over the CTA's
    // samples in order.  Dead samples contribute exact zeros.
    float* row = partials + size_t(blockIdx.x) * kRow;
    for (int e = me; e < P; e += kSamples) {
        float g = 0.f;
        if (e < CS_LIFETIME_B1_AT) {
            const int j = (e - CS_LIFETIME_W1_AT) / F, f = (e - CS_LIFETIME_W1_AT) % F;
            for (int q = 0; q < kSamples; ++q)
                g = fmaf(D1[q * kHStride + j], X[q * kXStride + f], g);
        } else if (e < CS_LIFETIME_W2_AT) {
            const int j = e - CS_LIFETIME_B1_AT;
            for (int q = 0; q < kSamples; ++q)
                g += D1[q * kHStride + j];
        } else if (e < CS_LIFETIME_B2_AT) {
            const int j = (e - CS_LIFETIME_W2_AT) / H, k = (e - CS_LIFETIME_W2_AT) % H;
            for (int q = 0; q < kSamples; ++q)
                g = fmaf(D2[q * kHStride + j], A1[q * kHStride + k], g);
        } else if (e < CS_LIFETIME_W3_AT) {
            const int j = e - CS_LIFETIME_B2_AT;
            for (int q = 0; q < kSamples; ++q)
                g += D2[q * kHStride + j];
        } else if (e < CS_LIFETIME_B3_AT) {
            const int o = (e - CS_LIFETIME_W3_AT) / H, j = (e - CS_LIFETIME_W3_AT) % H;
            for (int q = 0; q < kSamples; ++q)
                g = fmaf(DY[q * O + o], A2[q * kHStride + j], g);
        } else {
            const int o = e - CS_LIFETIME_B3_AT;
            for (int q = 0; q < kSamples; ++q)
                g += DY[q * O + o];
        }
        row[e] = g;
    }
    if (me == 0) {
        float total = 0.f;
        for (int q = 0; q < kSamples; ++q)
            total += lossOf[q];
        row[P] = total;
    }
}

// Adds the partial rows in CTA order; optionally writes the gradient (+ loss) and
// applies one Adam step to the parameters.
__global__ void updateKernel(const float* __restrict__ partials, int blocks, float* __restrict__ gradient,
                             float* __restrict__ loss, float* __restrict__ params, float* __restrict__ m,
                             float* __restrict__ v, float rate, float correction1, float correction2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > P)
        return;
    float g = 0.f;
    for (int b = 0; b < blocks; ++b)
        g += partials[size_t(b) * kRow + p];
    if (gradient)
        gradient[p] = g;
    if (p == P) {
        if (loss)
            *loss = g;
        return;
    }
    if (params) {
        constexpr float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
        const float m1 = beta1 * m[p] + (1.f - beta1) * g;
        const float m2 = beta2 * v[p] + (1.f - beta2) * g * g;
        m[p] = m1;
        v[p] = m2;
        params[p] -= rate * (m1 / correction1) / (sqrtf(m2 / correction2) + eps);
    }
}

constexpr int kLabelThreads = 256;

// One CTA per window: the largest magnitude and the last frame at or above the
// threshold (max reductions, so the result does not depend on the order).
__global__ void __launch_bounds__(kLabelThreads) labelKernel(const float2* __restrict__ mix,
                                                             const long long* __restrict__ windows,
                                                             float threshold, float* __restrict__ peak,
                                                             int* __restrict__ last)
{
    const long long first = windows[2 * size_t(blockIdx.x)];
    const long long end = windows[2 * size_t(blockIdx.x) + 1];
    float top = 0.f;
    long long lastFrame = -1;
    for (long long f = first + threadIdx.x; f < end; f += kLabelThreads) {
        const float2 v = mix[f];
        const float m = fmaxf(fabsf(v.x), fabsf(v.y));
        top = fmaxf(top, m);
        if (m >= threshold)
            lastFrame = f;
    }
    for (int offset = 16; offset; offset >>= 1) {
        top = fmaxf(top, __shfl_xor_sync(0xffffffffu, top, offset));
        lastFrame = max(lastFrame, __shfl_xor_sync(0xffffffffu, lastFrame, offset));
    }
    __shared__ float tops[kLabelThreads / 32];
    __shared__ long long lasts[kLabelThreads / 32];
    const int warp = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
        tops[warp] = top;
        lasts[warp] = lastFrame;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kLabelThreads / 32; ++w) {
            top = fmaxf(top, tops[w]);
            lastFrame = max(lastFrame, lasts[w]);
        }
        peak[blockIdx.x] = top;
        last[blockIdx.x] = lastFrame < 0 ? -1 : int(lastFrame - first);
    }
}

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(status));
}

template <class Body>
int guarded(Body&& body)
{
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        lastError = e.what();
        return 1;
    }
}

void requireAligned(const void* pointer, const char* what)
{
    if (!pointer)
        throw std::runtime_error(std::string(what) + " is null");
    if (reinterpret_cast<uintptr_t>(pointer) % 16)
        throw std::runtime_error(std::string(what) + " must be 16-byte aligned");
}

int blocksFor(int count) { return (count + kSamples - 1) / kSamples; }

void launchGradient(const float* params, const float* norm, const float* features, const float* targets,
                    int count, float* partials, cudaStream_t stream)
{
    if (count <= 0)
        throw std::runtime_error("no samples");
    requireAligned(params, "params");
    requireAligned(norm, "norm");
    requireAligned(features, "features");
    requireAligned(targets, "targets");
    requireAligned(partials, "partials");
    // Set on every call: the attribute belongs to the current device's context.
    check(cudaFuncSetAttribute(gradientKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGradientSmem)),
          "gradient kernel shared memory");
    gradientKernel<<<blocksFor(count), kSamples, kGradientSmem, stream>>>(params, norm, features, targets, count,
                                                                          1.f / float(count), partials);
    check(cudaGetLastError(), "gradient kernel launch");
}

} // namespace

extern "C" {

int cs_lifetime_forward(const float* params, const float* norm, const float* features, int count,
                        float* predictions, void* stream)
{
    return guarded([&] {
        if (count < 0)
            throw std::runtime_error("negative count");
        if (!count)
            return;
        requireAligned(params, "params");
        requireAligned(norm, "norm");
        requireAligned(features, "features");
        requireAligned(predictions, "predictions");
        const int warpsRows = kTensorWarps * 16;
        forwardTensorKernel<<<(count + warpsRows - 1) / warpsRows, kTensorWarps * 32, 0, cudaStream_t(stream)>>>(
            params, norm, features, count, predictions);
        check(cudaGetLastError(), "forward kernel launch");
    });
}

size_t cs_lifetime_partial_floats(int count)
{
    return count <= 0 ? 0 : size_t(blocksFor(count)) * kRow;
}

int cs_lifetime_gradient(const float* params, const float* norm, const float* features, const float* targets,
                         int count, float* partials, float* gradient, void* stream)
{
    return guarded([&] {
        requireAligned(gradient, "gradient");
        launchGradient(params, norm, features, targets, count, partials, cudaStream_t(stream));
        updateKernel<<<(kRow + 255) / 256, 256, 0, cudaStream_t(stream)>>>(
            partials, blocksFor(count), gradient, nullptr, nullptr, nullptr, nullptr, 0.f, 1.f, 1.f);
        check(cudaGetLastError(), "update kernel launch");
    });
}

int cs_lifetime_train_step(float* params, float* moment1, float* moment2, const float* norm,
                           const float* features, const float* targets, int count, float* partials, int step,
                           float learning_rate, float* loss, void* stream)
{
    return guarded([&] {
        if (step < 1)
            throw std::runtime_error("Adam steps count from 1");
        requireAligned(moment1, "moment1");
        requireAligned(moment2, "moment2");
        launchGradient(params, norm, features, targets, count, partials, cudaStream_t(stream));
        const float c1 = float(1.0 - std::pow(0.9, double(step)));
        const float c2 = float(1.0 - std::pow(0.999, double(step)));
        updateKernel<<<(kRow + 255) / 256, 256, 0, cudaStream_t(stream)>>>(
            partials, blocksFor(count), nullptr, loss, params, moment1, moment2, learning_rate, c1, c2);
        check(cudaGetLastError(), "update kernel launch");
    });
}

int cs_note_labels(const float* mix, const int64_t* windows, int count, float threshold, float* peak,
                   int32_t* last, void* stream)
{
    return guarded([&] {
        if (count < 0)
            throw std::runtime_error("negative count");
        if (!count)
            return;
        if (!mix || !windows || !peak || !last)
            throw std::runtime_error("null pointer");
        if (reinterpret_cast<uintptr_t>(mix) % 8)
            throw std::runtime_error("mix must be 8-byte aligned");
        labelKernel<<<count, kLabelThreads, 0, cudaStream_t(stream)>>>(
            reinterpret_cast<const float2*>(mix), reinterpret_cast<const long long*>(windows), threshold, peak,
            last);
        check(cudaGetLastError(), "label kernel launch");
    });
}

const char* cs_lifetime_last_error(void) { return lastError.c_str(); }

} // extern "C"
