// mlp.cu -- the learned format selector: a 32 -> 64 -> 64 -> 5 MLP (ReLU)
// predicting log2 of each candidate's compressed size from the block's
// sampled statistics.  BF16 weights (FP32 master copy for Adam), FP32
// accumulation everywhere.
//
// Every matrix product runs on the tensor cores (mma.sync m16n8k16, BF16
// operands, FP32 accumulators), one warp per 16 samples.  A layer's FP32
// accumulators are turned into the next layer's BF16 A operand in registers
// (the m16n8 accumulator layout of two adjacent column tiles is the m16k16
// A layout), so activations never leave the warp in the forward pass.
//
// Training step (batch B, one CTA of 4 warps per 64 samples, deterministic):
//   k_mlp_step  : forward, loss and backward through the hidden layers per
//                 warp; the BF16 activations and deltas are stored transposed
//                 in shared memory and the CTA's weight gradients (sums over
//                 its 64 samples) are tensor-core products of those tiles;
//                 bias gradients are FP32 sums; per-CTA partials out;
//   k_mlp_adam  : one thread per parameter sums the partials in fixed order,
//                 applies Adam and refreshes the BF16 copy;
//   k_mlp_tick  : advances the device step counter.
// The three launches are captured once as a CUDA graph and replayed for
// every step, so a 2000-step run issues 2000 graph launches and no host
// synchronisation.
//
// Rounding points (the CPU restatement follows them): features, hidden
// activations and backward deltas are rounded to BF16 where they enter a
// product; biases are added and ReLU masks taken in FP32.
#include <cuda_bf16.h>

#include "internal.h"

namespace ms {

constexpr unsigned kIn = 32, kH = 64, kOut = 5;
constexpr unsigned kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
                   kB3 = kW3 + kOut * kH, kP = kB3 + kOut;
constexpr unsigned kStepThreads = 128;  // 4 warps x 16 samples
constexpr unsigned kStepSamples = 64;

}  // namespace ms

struct ms_mlp {
    float *params;          // FP32 master weights [kP]
    __nv_bfloat16 *wbf;     // BF16 copy used by forward/backward [kP]
    float *m, *v;           // Adam moments
    float *partials;        // per-CTA gradients [max_ctas][kP]
    float *grads;           // reduced gradients [kP]
    unsigned max_ctas;
    unsigned long long *step;  // device step counter
    float *loss;               // device loss of the last step
};

namespace ms {
namespace {

__device__ __forceinline__ uint64_t mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
    return v;
}

__global__ void k_mlp_init(float *p, __nv_bfloat16 *wbf, float *m, float *v, uint64_t seed) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < kP; i += gridDim.x * blockDim.x) {
        float fan = 0.f;
        if (i < kB1) fan = float(kIn);
        else if (i >= kW2 && i < kB2) fan = float(kH);
        else if (i >= kW3 && i < kB3) fan = float(kH);
        float w = 0.f;
        if (fan > 0.f) {  // He-uniform
            const float u = float(mix(seed ^ (uint64_t(i) << 20)) >> 40) / float(1 << 24);
            w = (2.f * u - 1.f) * sqrtf(6.f / fan);
        }
        if (i >= kB3) w = 10.f;  // output bias near typical log2 sizes
        p[i] = w;
        wbf[i] = __float2bfloat16_rn(w);
        m[i] = 0.f;
        v[i] = 0.f;
    }
}

// label j of block b: log2(size in bytes)
__device__ __forceinline__ float label(const uint32_t *sizes, uint64_t b, unsigned j) {
    return log2f(float(sizes[b * kOut + j]));
}

// ---------------------------------------------------------------------------
// tensor-core helpers: D = A (16x16, row) * B (16x8, col) + C, BF16 in, FP32
// accumulate.  Fragment of lane (g = lane/4, t = lane%4):
//   A regs {a0,a1} row g, k 2t..2t+1 | {a2,a3} row g+8 | {a4,a5} row g, k 8+2t
//     | {a6,a7} row g+8, k 8+2t          (low half = lower column)
//   B regs {b0,b1} k 2t..2t+1, col g | {b2,b3} k 8+2t..
//   C/D    c0,c1 row g, cols 2t,2t+1 | c2,c3 row g+8
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// Shared-memory row strides (BF16 elements; +8 breaks bank conflicts).
constexpr unsigned kLdIn = kIn + 8, kLdH = kH + 8, kLdS = kStepSamples + 8, kLdO = 16 + 8;

// The weights as the products read them: W1 [64][32], W2 [64][64] and
// W3 [8][64] (rows 5..7 zero) in their own layout (B operand of the forward
// products), W2T [64][64] and W3T [64][16] (columns 5..15 zero) transposed
// (B operand of the backward products), biases in FP32.
struct MlpSmemW {
    __nv_bfloat16 w1[kH * kLdIn], w2[kH * kLdH], w3[8 * kLdH], w2t[kH * kLdH], w3t[kH * kLdO];
    float b1[kH], b2[kH], b3[8];
};

__device__ void load_weights(MlpSmemW &w, const __nv_bfloat16 *__restrict__ wbf, bool transposed) {
    for (unsigned i = threadIdx.x; i < kH * kIn; i += blockDim.x) w.w1[(i / kIn) * kLdIn + i % kIn] = wbf[kW1 + i];
    for (unsigned i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const __nv_bfloat16 v = wbf[kW2 + i];
        w.w2[(i / kH) * kLdH + i % kH] = v;
        if (transposed) w.w2t[(i % kH) * kLdH + i / kH] = v;
    }
    for (unsigned i = threadIdx.x; i < 8 * kH; i += blockDim.x) {
        const unsigned j = i / kH, h = i % kH;
        const __nv_bfloat16 v = j < kOut ? wbf[kW3 + j * kH + h] : __float2bfloat16_rn(0.f);
        w.w3[j * kLdH + h] = v;
    }
    if (transposed)
        for (unsigned i = threadIdx.x; i < kH * 16; i += blockDim.x) {
            const unsigned h = i / 16, j = i % 16;
            w.w3t[h * kLdO + j] = j < kOut ? wbf[kW3 + j * kH + h] : __float2bfloat16_rn(0.f);
        }
    for (unsigned i = threadIdx.x; i < kH; i += blockDim.x) {
        w.b1[i] = __bfloat162float(wbf[kB1 + i]);
        w.b2[i] = __bfloat162float(wbf[kB2 + i]);
    }
    if (threadIdx.x < 8) w.b3[threadIdx.x] = threadIdx.x < kOut ? __bfloat162float(wbf[kB3 + threadIdx.x]) : 0.f;
}

// A fragments (two 16-column slices) of 16 samples' features; rows whose
// sample is absent (valid bit clear) are zero.
__device__ __forceinline__ void load_x(const float *__restrict__ feats, uint64_t b_lo, uint64_t b_hi, bool v_lo,
                                       bool v_hi, unsigned t, uint32_t (&ax)[2][4], float (&xf)[2][8]) {
#pragma unroll
    for (unsigned j = 0; j < 2; j++) {
#pragma unroll
        for (unsigned h = 0; h < 2; h++) {  // k 16j + 8h + 2t
            const unsigned k = 16 * j + 8 * h + 2 * t;
            const float2 lo = v_lo ? __ldg(reinterpret_cast<const float2 *>(feats + b_lo * kIn + k)) : make_float2(0, 0);
            const float2 hi = v_hi ? __ldg(reinterpret_cast<const float2 *>(feats + b_hi * kIn + k)) : make_float2(0, 0);
            ax[j][2 * h] = pack_bf16(lo.x, lo.y);
            ax[j][2 * h + 1] = pack_bf16(hi.x, hi.y);
            xf[j][4 * h] = lo.x;
            xf[j][4 * h + 1] = lo.y;
            xf[j][4 * h + 2] = hi.x;
            xf[j][4 * h + 3] = hi.y;
        }
    }
}

// Forward through the hidden layers for one warp's 16 samples: acc1/acc2
// hold z1/z2 (FP32, 8 column tiles), a2/a3 the BF16 A fragments of
// relu(z1)/relu(z2), out the 16 x 8 output tile (columns 5..7 zero).
__device__ __forceinline__ void mlp_forward(const MlpSmemW &w, unsigned g, unsigned t, const uint32_t (&ax)[2][4],
                                            float (&acc1)[8][4], float (&acc2)[8][4], uint32_t (&a2)[4][4],
                                            uint32_t (&a3)[4][4], float (&out)[4]) {
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++) {
        acc1[nt][0] = acc1[nt][2] = w.b1[8 * nt + 2 * t];
        acc1[nt][1] = acc1[nt][3] = w.b1[8 * nt + 2 * t + 1];
#pragma unroll
        for (unsigned j = 0; j < 2; j++) {
            const __nv_bfloat16 *row = w.w1 + (8 * nt + g) * kLdIn + 16 * j + 2 * t;
            mma_bf16(acc1[nt], ax[j], lds32(row), lds32(row + 8));
        }
    }
#pragma unroll
    for (unsigned j = 0; j < 4; j++) {
        a2[j][0] = pack_bf16(fmaxf(acc1[2 * j][0], 0.f), fmaxf(acc1[2 * j][1], 0.f));
        a2[j][1] = pack_bf16(fmaxf(acc1[2 * j][2], 0.f), fmaxf(acc1[2 * j][3], 0.f));
        a2[j][2] = pack_bf16(fmaxf(acc1[2 * j + 1][0], 0.f), fmaxf(acc1[2 * j + 1][1], 0.f));
        a2[j][3] = pack_bf16(fmaxf(acc1[2 * j + 1][2], 0.f), fmaxf(acc1[2 * j + 1][3], 0.f));
    }
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++) {
        acc2[nt][0] = acc2[nt][2] = w.b2[8 * nt + 2 * t];
        acc2[nt][1] = acc2[nt][3] = w.b2[8 * nt + 2 * t + 1];
#pragma unroll
        for (unsigned j = 0; j < 4; j++) {
            const __nv_bfloat16 *row = w.w2 + (8 * nt + g) * kLdH + 16 * j + 2 * t;
            mma_bf16(acc2[nt], a2[j], lds32(row), lds32(row + 8));
        }
    }
#pragma unroll
    for (unsigned j = 0; j < 4; j++) {
        a3[j][0] = pack_bf16(fmaxf(acc2[2 * j][0], 0.f), fmaxf(acc2[2 * j][1], 0.f));
        a3[j][1] = pack_bf16(fmaxf(acc2[2 * j][2], 0.f), fmaxf(acc2[2 * j][3], 0.f));
        a3[j][2] = pack_bf16(fmaxf(acc2[2 * j + 1][0], 0.f), fmaxf(acc2[2 * j + 1][1], 0.f));
        a3[j][3] = pack_bf16(fmaxf(acc2[2 * j + 1][2], 0.f), fmaxf(acc2[2 * j + 1][3], 0.f));
    }
    out[0] = out[2] = w.b3[2 * t];
    out[1] = out[3] = w.b3[2 * t + 1];
#pragma unroll
    for (unsigned j = 0; j < 4; j++) {
        const __nv_bfloat16 *row = w.w3 + g * kLdH + 16 * j + 2 * t;
        mma_bf16(out, a3[j], lds32(row), lds32(row + 8));
    }
}


// The CTA's activations and deltas, transposed ([feature][sample], BF16).
struct MlpSmemA {
    __nv_bfloat16 xt[kIn * kLdS], h1t[kH * kLdS], h2t[kH * kLdS], d1t[kH * kLdS], d2t[kH * kLdS], dot[16 * kLdS];
    float gb[kH + kH + 8][4];  // bias-gradient partial sums per warp
    float ls[4];               // loss per warp
};

// Stores a 16 x (8 * NT) FP32 tile (C layout) transposed as BF16 columns
// 16 w .. 16 w + 15 of dst [feature][sample].
template <unsigned NT>
__device__ __forceinline__ void store_t(__nv_bfloat16 *dst, const float (&c)[NT][4], unsigned w, unsigned g,
                                        unsigned t, bool relu) {
#pragma unroll
    for (unsigned nt = 0; nt < NT; nt++) {
#pragma unroll
        for (unsigned e = 0; e < 4; e++) {
            const unsigned col = 8 * nt + 2 * t + (e & 1), row = 16 * w + g + 8 * (e >> 1);
            dst[col * kLdS + row] = __float2bfloat16_rn(relu ? fmaxf(c[nt][e], 0.f) : c[nt][e]);
        }
    }
}

// Sum over the warp's 16 samples of a C-layout tile, per column: lanes of
// equal t hold the same columns (rows g and g + 8).
__device__ __forceinline__ float colsum(float v) {
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 4);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 8);
    v += __shfl_xor_sync(0xFFFFFFFFu, v, 16);
    return v;
}

// One training step for 64 samples per CTA: forward, backward, per-CTA
// gradients.  idx: explicit sample indices (gradient checks) or nullptr =
// sample by hash.
__global__ void __launch_bounds__(kStepThreads) k_mlp_step(const float *__restrict__ feats,
                                                          const uint32_t *__restrict__ sizes, uint64_t n,
                                                          const uint32_t *__restrict__ idx, unsigned batch,
                                                          const __nv_bfloat16 *__restrict__ wbf,
                                                          float *__restrict__ partials,
                                                          const unsigned long long *__restrict__ step,
                                                          uint64_t seed, float *__restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmemW &W = *reinterpret_cast<MlpSmemW *>(smem_raw);
    MlpSmemA &S = *reinterpret_cast<MlpSmemA *>(smem_raw + sizeof(MlpSmemW));
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    load_weights(W, wbf, true);
    for (unsigned i = threadIdx.x; i < 16 * kLdS; i += blockDim.x) S.dot[i] = __float2bfloat16_rn(0.f);
    // this warp's samples: rows g and g + 8 of its tile
    const unsigned s_lo = blockIdx.x * kStepSamples + 16 * w + g, s_hi = s_lo + 8;
    const bool v_lo = s_lo < batch, v_hi = s_hi < batch;
    const unsigned long long st = *step;
    const uint64_t b_lo = v_lo ? (idx ? idx[s_lo] : mix(seed ^ (st << 32) ^ s_lo) % n) : 0;
    const uint64_t b_hi = v_hi ? (idx ? idx[s_hi] : mix(seed ^ (st << 32) ^ s_hi) % n) : 0;
    __syncthreads();
    uint32_t ax[2][4];
    float xf[2][8];
    load_x(feats, b_lo, b_hi, v_lo, v_hi, t, ax, xf);
    float acc1[8][4], acc2[8][4], out[4];
    uint32_t a2[4][4], a3[4][4];
    mlp_forward(W, g, t, ax, acc1, acc2, a2, a3, out);
    // transposed BF16 copies of the product inputs for the weight gradients
#pragma unroll
    for (unsigned j = 0; j < 2; j++)
#pragma unroll
        for (unsigned e = 0; e < 8; e++) {
            const unsigned col = 16 * j + 8 * (e >> 2) + 2 * t + (e & 1), row = 16 * w + g + 8 * ((e >> 1) & 1);
            S.xt[col * kLdS + row] = __float2bfloat16_rn(xf[j][e]);
        }
    store_t<8>(S.h1t, acc1, w, g, t, true);
    store_t<8>(S.h2t, acc2, w, g, t, true);
    // loss and d(mean squared error)/d(out)
    float dout[4], ls = 0.f;
    const float scale = 2.f / float(batch * kOut);
#pragma unroll
    for (unsigned e = 0; e < 4; e++) {
        const unsigned j = 2 * t + (e & 1);
        const bool hi = e >> 1, valid = (hi ? v_hi : v_lo) && j < kOut;
        const float err = valid ? out[e] - label(sizes, hi ? b_hi : b_lo, j) : 0.f;
        ls += err * err;
        dout[e] = err * scale;
    }
    ls = warp_sum_f(ls);
    if (lane == 0) S.ls[w] = ls;
    uint32_t ado[4] = {pack_bf16(dout[0], dout[1]), pack_bf16(dout[2], dout[3]), 0u, 0u};
    if (t < 3) {  // columns 0..5 of the output tile (5 unused, zero)
#pragma unroll
        for (unsigned e = 0; e < 4; e++) {
            const unsigned j = 2 * t + (e & 1), row = 16 * w + g + 8 * (e >> 1);
            S.dot[j * kLdS + row] = __float2bfloat16_rn(dout[e]);
        }
    }
    // backward: dz2 = (dout W3) * (z2 > 0), dz1 = (dz2 W2) * (z1 > 0)
    float d2[8][4], d1[8][4];
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++) {
        d2[nt][0] = d2[nt][1] = d2[nt][2] = d2[nt][3] = 0.f;
        const __nv_bfloat16 *row = W.w3t + (8 * nt + g) * kLdO + 2 * t;
        mma_bf16(d2[nt], ado, lds32(row), lds32(row + 8));
#pragma unroll
        for (unsigned e = 0; e < 4; e++) d2[nt][e] = acc2[nt][e] > 0.f ? d2[nt][e] : 0.f;
    }
    uint32_t ad2[4][4];
#pragma unroll
    for (unsigned j = 0; j < 4; j++) {
        ad2[j][0] = pack_bf16(d2[2 * j][0], d2[2 * j][1]);
        ad2[j][1] = pack_bf16(d2[2 * j][2], d2[2 * j][3]);
        ad2[j][2] = pack_bf16(d2[2 * j + 1][0], d2[2 * j + 1][1]);
        ad2[j][3] = pack_bf16(d2[2 * j + 1][2], d2[2 * j + 1][3]);
    }
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++) {
        d1[nt][0] = d1[nt][1] = d1[nt][2] = d1[nt][3] = 0.f;
#pragma unroll
        for (unsigned j = 0; j < 4; j++) {
            const __nv_bfloat16 *row = W.w2t + (8 * nt + g) * kLdH + 16 * j + 2 * t;
            mma_bf16(d1[nt], ad2[j], lds32(row), lds32(row + 8));
        }
#pragma unroll
        for (unsigned e = 0; e < 4; e++) d1[nt][e] = acc1[nt][e] > 0.f ? d1[nt][e] : 0.f;
    }
    store_t<8>(S.d2t, d2, w, g, t, false);
    store_t<8>(S.d1t, d1, w, g, t, false);
    // bias gradients: FP32 sums of the deltas over this warp's samples
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++)
#pragma unroll
        for (unsigned c = 0; c < 2; c++) {
            const float s1 = colsum(d1[nt][c] + d1[nt][c + 2]), s2 = colsum(d2[nt][c] + d2[nt][c + 2]);
            if (g == 0) {
                S.gb[8 * nt + 2 * t + c][w] = s1;
                S.gb[kH + 8 * nt + 2 * t + c][w] = s2;
            }
        }
#pragma unroll
    for (unsigned c = 0; c < 2; c++) {
        const float s3 = colsum(dout[c] + dout[c + 2]);
        if (g == 0) S.gb[2 * kH + 2 * t + c][w] = s3;
    }
    __syncthreads();
    // weight gradients over the CTA's 64 samples: dW = dZ^T A, K = samples
    float *outp = partials + size_t(blockIdx.x) * kP;
    auto gemm_tile = [&](const __nv_bfloat16 *dt, const __nv_bfloat16 *at, unsigned m0, unsigned n0, unsigned ncols,
                         unsigned rows_valid, unsigned base) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (unsigned k0 = 0; k0 < kStepSamples; k0 += 16) {
            const uint32_t a[4] = {lds32(dt + (m0 + g) * kLdS + k0 + 2 * t), lds32(dt + (m0 + g + 8) * kLdS + k0 + 2 * t),
                                   lds32(dt + (m0 + g) * kLdS + k0 + 8 + 2 * t),
                                   lds32(dt + (m0 + g + 8) * kLdS + k0 + 8 + 2 * t)};
            const __nv_bfloat16 *bp = at + (n0 + g) * kLdS + k0 + 2 * t;
            mma_bf16(c, a, lds32(bp), lds32(bp + 8));
        }
#pragma unroll
        for (unsigned e = 0; e < 4; e++) {
            const unsigned row = m0 + g + 8 * (e >> 1), col = n0 + 2 * t + (e & 1);
            if (row < rows_valid) outp[base + row * ncols + col] = c[e];
        }
    };
    // W1: 64 x 32 (warp w: rows 16w.., 4 column tiles); W2: 64 x 64 (8 tiles);
    // W3: 5 x 64 (warp w: column tiles 2w, 2w+1)
#pragma unroll
    for (unsigned nt = 0; nt < 4; nt++) gemm_tile(S.d1t, S.xt, 16 * w, 8 * nt, kIn, kH, kW1);
#pragma unroll
    for (unsigned nt = 0; nt < 8; nt++) gemm_tile(S.d2t, S.h1t, 16 * w, 8 * nt, kH, kH, kW2);
#pragma unroll
    for (unsigned nt = 2 * w; nt < 2 * w + 2; nt++) gemm_tile(S.dot, S.h2t, 0, 8 * nt, kH, kOut, kW3);
    for (unsigned i = threadIdx.x; i < kH + kH + kOut; i += blockDim.x) {
        const float v = S.gb[i][0] + S.gb[i][1] + S.gb[i][2] + S.gb[i][3];
        outp[i < kH ? kB1 + i : i < 2 * kH ? kB2 + i - kH : kB3 + i - 2 * kH] = v;
    }
    if (threadIdx.x == 0 && loss) atomicAdd(loss, (S.ls[0] + S.ls[1] + S.ls[2] + S.ls[3]) / float(batch * kOut));
}

__global__ void k_mlp_reduce(const float *__restrict__ partials, unsigned nparts, float *__restrict__ grads) {
    for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < kP; p += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (unsigned c = 0; c < nparts; c++) g += partials[size_t(c) * kP + p];
        grads[p] = g;
    }
}

__global__ void k_mlp_adam(float *__restrict__ p, __nv_bfloat16 *__restrict__ wbf, float *__restrict__ m,
                           float *__restrict__ v, const float *__restrict__ partials, unsigned nparts,
                           const unsigned long long *__restrict__ step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float tt = float(*step + 1);
    const float c1 = 1.f - powf(b1, tt), c2 = 1.f - powf(b2, tt);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < kP; i += gridDim.x * blockDim.x) {
        float g = 0.f;
        for (unsigned c = 0; c < nparts; c++) g += partials[size_t(c) * kP + i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = w;
        wbf[i] = __float2bfloat16_rn(w);
    }
}

__global__ void k_mlp_tick(unsigned long long *step, float *loss, float *curve, unsigned long long first,
                           unsigned steps) {
    const unsigned long long s = *step;
    if (curve && s >= first && s - first < steps) curve[s - first] = *loss;
    *step = s + 1;
    *loss = 0.f;
}

// Inference: one warp per 16 blocks on the tensor cores; predicted log2
// sizes, the argmin and whether the margin to the runner-up is below
// `margin` (then 255: let the exhaustive pass decide).
__global__ void __launch_bounds__(128) k_mlp_choose(const float *__restrict__ feats, uint64_t n,
                                                   const __nv_bfloat16 *__restrict__ wbf, float margin,
                                                   float *__restrict__ pred, uint8_t *__restrict__ choice,
                                                   unsigned long long *__restrict__ nfallback) {
    __shared__ __align__(16) MlpSmemW W;
    load_weights(W, wbf, false);
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    unsigned fb = 0;
    for (uint64_t tile = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n;
         tile += warps) {
        const uint64_t b_lo = tile * 16 + g, b_hi = b_lo + 8;
        const bool v_lo = b_lo < n, v_hi = b_hi < n;
        uint32_t ax[2][4];
        float xf[2][8];
        load_x(feats, b_lo, b_hi, v_lo, v_hi, t, ax, xf);
        float acc1[8][4], acc2[8][4], out[4];
        uint32_t a2[4][4], a3[4][4];
        mlp_forward(W, g, t, ax, acc1, acc2, a2, a3, out);
        // gather the five outputs of row g into lane t = 0, of row g + 8 into t = 1
        float o[kOut];
        const unsigned q = lane & ~3u;
#pragma unroll
        for (unsigned j = 0; j < kOut; j++) {
            const float lo = __shfl_sync(0xFFFFFFFFu, out[j & 1], q + j / 2);
            const float hi = __shfl_sync(0xFFFFFFFFu, out[2 + (j & 1)], q + j / 2);
            o[j] = t == 0 ? lo : hi;
        }
        const uint64_t b = t == 0 ? b_lo : b_hi;
        if (t < 2 && b < n) {
            unsigned best = 0;
            for (unsigned j = 1; j < kOut; j++)
                if (o[j] < o[best]) best = j;
            float second = 1e30f;
            for (unsigned j = 0; j < kOut; j++)
                if (j != best) second = fminf(second, o[j]);
            const bool unsure = second - o[best] < margin;
            if (pred)
                for (unsigned j = 0; j < kOut; j++) pred[b * kOut + j] = o[j];
            if (choice) choice[b] = unsure ? uint8_t(255) : uint8_t(best);
            fb += unsure;
        }
    }
    fb = __reduce_add_sync(0xFFFFFFFFu, fb);
    if ((threadIdx.x & 31u) == 0 && nfallback && fb) atomicAdd(nfallback, (unsigned long long)fb);
}

size_t step_smem() { return sizeof(MlpSmemW) + sizeof(MlpSmemA); }

}  // namespace
}  // namespace ms

using namespace ms;

extern "C" uint64_t ms_gpu_mlp_param_count(void) { return kP; }

extern "C" int ms_gpu_mlp_create(uint64_t seed, unsigned max_batch, ms_mlp **out) {
    if (!out || max_batch == 0) return ms_fail(MS_ERR_INVALID, "mlp_create: bad argument");
    ms_mlp *m = new ms_mlp();
    m->max_ctas = (max_batch + kStepSamples - 1) / kStepSamples;
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&m->params, sizeof(float) * kP);
    e = e ? e : cudaMalloc(&m->wbf, sizeof(__nv_bfloat16) * kP);
    e = e ? e : cudaMalloc(&m->m, sizeof(float) * kP);
    e = e ? e : cudaMalloc(&m->v, sizeof(float) * kP);
    e = e ? e : cudaMalloc(&m->partials, sizeof(float) * kP * m->max_ctas);
    e = e ? e : cudaMalloc(&m->grads, sizeof(float) * kP);
    e = e ? e : cudaMalloc(&m->step, sizeof(unsigned long long));
    e = e ? e : cudaMalloc(&m->loss, sizeof(float));
    if (e != cudaSuccess) {
        delete m;
        return ms_fail_cuda(e, "mlp_create");
    }
    k_mlp_init<<<8, 256>>>(m->params, m->wbf, m->m, m->v, seed);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY(cudaMemset(m->step, 0, sizeof(unsigned long long)));
    MS_CUDA_TRY(cudaMemset(m->loss, 0, sizeof(float)));
    MS_CUDA_TRY(cudaDeviceSynchronize());
    MS_CUDA_TRY(cudaFuncSetAttribute(k_mlp_step, cudaFuncAttributeMaxDynamicSharedMemorySize, int(step_smem())));
    *out = m;
    return MS_OK;
}

extern "C" int ms_gpu_mlp_destroy(ms_mlp *m) {
    if (!m) return MS_OK;
    cudaFree(m->params);
    cudaFree(m->wbf);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->partials);
    cudaFree(m->grads);
    cudaFree(m->step);
    cudaFree(m->loss);
    delete m;
    return MS_OK;
}

// Gradient of the mean squared error over an explicit batch (no update):
// d_grads receives kP floats in parameter order, *d_loss the loss.
extern "C" int ms_gpu_mlp_grads(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n,
                                const uint32_t *d_idx, unsigned batch, float *d_grads, float *d_loss, void *stream) {
    if (!m || !d_feats || !d_sizes || !d_idx || !d_grads || batch == 0 || batch > m->max_ctas * kStepSamples)
        return ms_fail(MS_ERR_INVALID, "mlp_grads: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned ctas = (batch + kStepSamples - 1) / kStepSamples;
    if (d_loss) MS_CUDA_TRY(cudaMemsetAsync(d_loss, 0, sizeof(float), st));
    k_mlp_step<<<ctas, kStepThreads, step_smem(), st>>>(d_feats, d_sizes, n, d_idx, batch, m->wbf, m->partials,
                                                        m->step, 0, d_loss);
    MS_CUDA_TRY(cudaGetLastError());
    k_mlp_reduce<<<8, 256, 0, st>>>(m->partials, ctas, d_grads);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// `steps` Adam steps of `batch` samples drawn from n labelled blocks.  The
// step is captured once as a CUDA graph and replayed.  d_loss_curve
// (optional, device, `steps` floats) receives the training loss per step.
extern "C" int ms_gpu_mlp_train(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n, unsigned steps,
                                unsigned batch, float lr, uint64_t seed, float *d_loss_curve, void *stream) {
    if (!m || !d_feats || !d_sizes || n == 0 || batch == 0 || batch > m->max_ctas * kStepSamples)
        return ms_fail(MS_ERR_INVALID, "mlp_train: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned ctas = (batch + kStepSamples - 1) / kStepSamples;
    unsigned long long first = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&first, m->step, 8, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(float), st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    cudaStream_t cap;
    MS_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g;
    cudaGraphExec_t ge;
    MS_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    k_mlp_step<<<ctas, kStepThreads, step_smem(), cap>>>(d_feats, d_sizes, n, nullptr, batch, m->wbf, m->partials,
                                                         m->step, seed, m->loss);
    k_mlp_adam<<<(kP + 255) / 256, 256, 0, cap>>>(m->params, m->wbf, m->m, m->v, m->partials, ctas, m->step, lr);
    k_mlp_tick<<<1, 1, 0, cap>>>(m->step, m->loss, d_loss_curve, first, steps);
    cudaError_t ce = cudaStreamEndCapture(cap, &g);
    if (ce != cudaSuccess) {
        cudaStreamDestroy(cap);
        return ms_fail_cuda(ce, "mlp_train capture");
    }
    ce = cudaGraphInstantiate(&ge, g, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        return ms_fail_cuda(ce, "mlp_train instantiate");
    }
    for (unsigned s = 0; s < steps && ce == cudaSuccess; s++) ce = cudaGraphLaunch(ge, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    if (ce != cudaSuccess) return ms_fail_cuda(ce, "mlp_train");
    return MS_OK;
}

// Mean loss over an explicit set (evaluation), no update.
extern "C" int ms_gpu_mlp_eval_loss(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n,
                                    const uint32_t *d_idx, unsigned batch, float *d_loss, void *stream) {
    if (!m) return ms_fail(MS_ERR_INVALID, "mlp_eval_loss: null");
    return ms_gpu_mlp_grads(m, d_feats, d_sizes, n, d_idx, batch, m->grads, d_loss, stream);
}

extern "C" int ms_gpu_mlp_choose(ms_mlp *m, const float *d_feats, uint64_t n, float margin_log2, float *d_pred,
                                 uint8_t *d_choice, uint64_t *d_nfallback, void *stream) {
    if (!m || (!d_feats && n)) return ms_fail(MS_ERR_INVALID, "mlp_choose: bad argument");
    if (reinterpret_cast<uintptr_t>(d_feats) % 16)
        return ms_fail(MS_ERR_INVALID, "mlp_choose: features must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    if (d_nfallback) MS_CUDA_TRY(cudaMemsetAsync(d_nfallback, 0, 8, st));
    if (!n) return MS_OK;
    const unsigned grid = unsigned(minu((n + 63) / 64, uint64_t(persistent_grid(128, 8))));
    k_mlp_choose<<<grid, 128, 0, st>>>(d_feats, n, m->wbf, margin_log2, d_pred, d_choice,
                                       (unsigned long long *)d_nfallback);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// Checkpoint: parameters (FP32 master), Adam moments and the step counter.
// h_state holds 3*kP floats followed by the 8-byte step.
extern "C" uint64_t ms_gpu_mlp_state_bytes(void) { return 3 * sizeof(float) * kP + 8; }

extern "C" int ms_gpu_mlp_save(ms_mlp *m, void *h_state) {
    if (!m || !h_state) return ms_fail(MS_ERR_INVALID, "mlp_save: null");
    float *f = static_cast<float *>(h_state);
    MS_CUDA_TRY(cudaDeviceSynchronize());
    MS_CUDA_TRY(cudaMemcpy(f, m->params, sizeof(float) * kP, cudaMemcpyDeviceToHost));
    MS_CUDA_TRY(cudaMemcpy(f + kP, m->m, sizeof(float) * kP, cudaMemcpyDeviceToHost));
    MS_CUDA_TRY(cudaMemcpy(f + 2 * kP, m->v, sizeof(float) * kP, cudaMemcpyDeviceToHost));
    MS_CUDA_TRY(cudaMemcpy(f + 3 * kP, m->step, 8, cudaMemcpyDeviceToHost));
    return MS_OK;
}

__global__ void k_mlp_refresh_bf16(const float *p, __nv_bfloat16 *w) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < kP; i += gridDim.x * blockDim.x)
        w[i] = __float2bfloat16_rn(p[i]);
}

extern "C" int ms_gpu_mlp_load(ms_mlp *m, const void *h_state) {
    if (!m || !h_state) return ms_fail(MS_ERR_INVALID, "mlp_load: null");
    const float *f = static_cast<const float *>(h_state);
    MS_CUDA_TRY(cudaMemcpy(m->params, f, sizeof(float) * kP, cudaMemcpyHostToDevice));
    MS_CUDA_TRY(cudaMemcpy(m->m, f + kP, sizeof(float) * kP, cudaMemcpyHostToDevice));
    MS_CUDA_TRY(cudaMemcpy(m->v, f + 2 * kP, sizeof(float) * kP, cudaMemcpyHostToDevice));
    MS_CUDA_TRY(cudaMemcpy(m->step, f + 3 * kP, 8, cudaMemcpyHostToDevice));
    k_mlp_refresh_bf16<<<8, 256>>>(m->params, m->wbf);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY(cudaDeviceSynchronize());
    return MS_OK;
}
