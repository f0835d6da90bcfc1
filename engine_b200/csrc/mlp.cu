// mlp.cu -- the learned format selector: a 32 -> 64 -> 64 -> 5 MLP (ReLU)
// predicting log2 of each candidate's compressed size from the block's
// sampled statistics.  BF16 weights (FP32 master copy for Adam), FP32
// accumulation everywhere.
//
// Training step (batch B, one CTA per 64 samples, no atomics, deterministic):
//   k_mlp_step  : each thread runs one sample forward and backward with the
//                 BF16 weights, keeps activations and deltas in shared
//                 memory, then the CTA reduces its 64 samples into per-CTA
//                 partial gradients (plain FP32 dot products over samples);
//   k_mlp_adam  : one thread per parameter sums the partials in fixed order,
//                 applies Adam and refreshes the BF16 copy;
//   k_mlp_tick  : advances the device step counter.
// The three launches are captured once as a CUDA graph and replayed for
// every step, so a 2000-step run issues 2000 graph launches and no host
// synchronisation.
#include <cuda_bf16.h>

#include "internal.h"

namespace ms {

constexpr unsigned kIn = 32, kH = 64, kOut = 5;
constexpr unsigned kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
                   kB3 = kW3 + kOut * kH, kP = kB3 + kOut;
constexpr unsigned kStepThreads = 64;
constexpr unsigned kSX = kIn + 1, kSH = kH + 1;  // padded shared-memory rows (no bank conflicts)

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

// One training step's forward + backward for 64 samples per CTA.
// idx: explicit sample indices (gradient checks) or nullptr = sample by hash.
__global__ void __launch_bounds__(kStepThreads) k_mlp_step(const float *__restrict__ feats,
                                                          const uint32_t *__restrict__ sizes, uint64_t n,
                                                          const uint32_t *__restrict__ idx, unsigned batch,
                                                          const __nv_bfloat16 *__restrict__ wbf,
                                                          float *__restrict__ partials,
                                                          const unsigned long long *__restrict__ step,
                                                          uint64_t seed, float *__restrict__ loss) {
    extern __shared__ float sm[];
    float *W = sm;                        // kP weights as float
    float *X = W + kP;                    // [64][kSX]
    float *H1 = X + kStepThreads * kSX;   // [64][kSH] activations (post ReLU)
    float *H2 = H1 + kStepThreads * kSH;
    float *D1 = H2 + kStepThreads * kSH;  // [64][kSH] dz1
    float *D2 = D1 + kStepThreads * kSH;  // [64][kSH] dz2
    float *DO = D2 + kStepThreads * kSH;  // [64][kOut]
    float *LS = DO + kStepThreads * kOut; // [64] per-sample loss
    const unsigned t = threadIdx.x;
    for (unsigned i = t; i < kP; i += blockDim.x) W[i] = __bfloat162float(wbf[i]);
    const unsigned s_glob = blockIdx.x * kStepThreads + t;
    const bool act = s_glob < batch;
    uint64_t b = 0;
    if (act) b = idx ? idx[s_glob] : mix(seed ^ (*step << 32) ^ s_glob) % n;
    __syncthreads();
    float x[kIn];
    for (unsigned k = 0; k < kIn; k++) x[k] = act ? feats[b * kIn + k] : 0.f;
    for (unsigned k = 0; k < kIn; k++) X[t * kSX + k] = x[k];
    // forward
    for (unsigned i = 0; i < kH; i++) {
        float z = W[kB1 + i];
        for (unsigned k = 0; k < kIn; k++) z = fmaf(W[kW1 + i * kIn + k], x[k], z);
        H1[t * kSH + i] = fmaxf(z, 0.f);
    }
    for (unsigned i = 0; i < kH; i++) {
        float z = W[kB2 + i];
        for (unsigned k = 0; k < kH; k++) z = fmaf(W[kW2 + i * kH + k], H1[t * kSH + k], z);
        H2[t * kSH + i] = fmaxf(z, 0.f);
    }
    float ls = 0.f;
    for (unsigned j = 0; j < kOut; j++) {
        float z = W[kB3 + j];
        for (unsigned k = 0; k < kH; k++) z = fmaf(W[kW3 + j * kH + k], H2[t * kSH + k], z);
        const float e = act ? z - label(sizes, b, j) : 0.f;
        ls += e * e;
        DO[t * kOut + j] = 2.f * e / float(batch * kOut);  // d(mean squared error)/dz3
    }
    LS[t] = ls;
    // backward through the hidden layers
    for (unsigned i = 0; i < kH; i++) {
        float g = 0.f;
        for (unsigned j = 0; j < kOut; j++) g = fmaf(W[kW3 + j * kH + i], DO[t * kOut + j], g);
        D2[t * kSH + i] = H2[t * kSH + i] > 0.f ? g : 0.f;
    }
    for (unsigned i = 0; i < kH; i++) {
        float g = 0.f;
        for (unsigned j = 0; j < kH; j++) g = fmaf(W[kW2 + j * kH + i], D2[t * kSH + j], g);
        D1[t * kSH + i] = H1[t * kSH + i] > 0.f ? g : 0.f;
    }
    __syncthreads();
    // per-CTA gradients: sums over the 64 samples, fixed order
    float *out = partials + size_t(blockIdx.x) * kP;
    for (unsigned p = t; p < kP; p += blockDim.x) {
        float g = 0.f;
        if (p < kB1) {
            const unsigned i = p / kIn, k = p % kIn;
            for (unsigned s = 0; s < kStepThreads; s++) g = fmaf(D1[s * kSH + i], X[s * kSX + k], g);
        } else if (p < kW2) {
            const unsigned i = p - kB1;
            for (unsigned s = 0; s < kStepThreads; s++) g += D1[s * kSH + i];
        } else if (p < kB2) {
            const unsigned i = (p - kW2) / kH, k = (p - kW2) % kH;
            for (unsigned s = 0; s < kStepThreads; s++) g = fmaf(D2[s * kSH + i], H1[s * kSH + k], g);
        } else if (p < kW3) {
            const unsigned i = p - kB2;
            for (unsigned s = 0; s < kStepThreads; s++) g += D2[s * kSH + i];
        } else if (p < kB3) {
            const unsigned j = (p - kW3) / kH, k = (p - kW3) % kH;
            for (unsigned s = 0; s < kStepThreads; s++) g = fmaf(DO[s * kOut + j], H2[s * kSH + k], g);
        } else {
            const unsigned j = p - kB3;
            for (unsigned s = 0; s < kStepThreads; s++) g += DO[s * kOut + j];
        }
        out[p] = g;
    }
    if (t == 0 && loss) {
        float l = 0.f;
        for (unsigned s = 0; s < kStepThreads; s++) l += LS[s];
        atomicAdd(loss, l / float(batch * kOut));
    }
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

// Inference: one thread per block; predicted log2 sizes, the argmin and
// whether the margin to the runner-up is below `margin` (then 255: let the
// exhaustive pass decide).
__global__ void __launch_bounds__(128) k_mlp_choose(const float *__restrict__ feats, uint64_t n,
                                                   const __nv_bfloat16 *__restrict__ wbf, float margin,
                                                   float *__restrict__ pred, uint8_t *__restrict__ choice,
                                                   unsigned long long *__restrict__ nfallback) {
    __shared__ __align__(16) float W[kP];
    for (unsigned i = threadIdx.x; i < kP; i += blockDim.x) W[i] = __bfloat162float(wbf[i]);
    __syncthreads();
    unsigned fb = 0;
    // The loops are unrolled so x and h1 stay in registers, and the weights
    // are read four at a time; the order of every sum is the plain loop's.
    for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < n; b += uint64_t(gridDim.x) * blockDim.x) {
        float x[kIn], h1[kH];
        const float4 *fx = reinterpret_cast<const float4 *>(feats + b * kIn);
#pragma unroll
        for (unsigned k = 0; k < kIn / 4; k++) {
            const float4 t = __ldg(fx + k);
            x[4 * k] = t.x;
            x[4 * k + 1] = t.y;
            x[4 * k + 2] = t.z;
            x[4 * k + 3] = t.w;
        }
#pragma unroll
        for (unsigned i = 0; i < kH; i++) {
            float z = W[kB1 + i];
            const float4 *w = reinterpret_cast<const float4 *>(W + kW1 + i * kIn);
#pragma unroll
            for (unsigned k = 0; k < kIn / 4; k++) {
                const float4 t = w[k];
                z = fmaf(t.x, x[4 * k], z);
                z = fmaf(t.y, x[4 * k + 1], z);
                z = fmaf(t.z, x[4 * k + 2], z);
                z = fmaf(t.w, x[4 * k + 3], z);
            }
            h1[i] = fmaxf(z, 0.f);
        }
        float o[kOut];
#pragma unroll
        for (unsigned j = 0; j < kOut; j++) o[j] = W[kB3 + j];
#pragma unroll 4
        for (unsigned i = 0; i < kH; i++) {
            float z = W[kB2 + i];
            const float4 *w = reinterpret_cast<const float4 *>(W + kW2 + i * kH);
#pragma unroll
            for (unsigned k = 0; k < kH / 4; k++) {
                const float4 t = w[k];
                z = fmaf(t.x, h1[4 * k], z);
                z = fmaf(t.y, h1[4 * k + 1], z);
                z = fmaf(t.z, h1[4 * k + 2], z);
                z = fmaf(t.w, h1[4 * k + 3], z);
            }
            z = fmaxf(z, 0.f);
#pragma unroll
            for (unsigned j = 0; j < kOut; j++) o[j] = fmaf(W[kW3 + j * kH + i], z, o[j]);
        }
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
    fb = __reduce_add_sync(0xFFFFFFFFu, fb);
    if ((threadIdx.x & 31u) == 0 && nfallback) atomicAdd(nfallback, (unsigned long long)fb);
}

size_t step_smem() {
    return sizeof(float) * (kP + kStepThreads * (kSX + 4 * kSH + kOut + 1));
}

}  // namespace
}  // namespace ms

using namespace ms;

extern "C" uint64_t ms_gpu_mlp_param_count(void) { return kP; }

extern "C" int ms_gpu_mlp_create(uint64_t seed, unsigned max_batch, ms_mlp **out) {
    if (!out || max_batch == 0) return ms_fail(MS_ERR_INVALID, "mlp_create: bad argument");
    ms_mlp *m = new ms_mlp();
    m->max_ctas = (max_batch + kStepThreads - 1) / kStepThreads;
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
    if (!m || !d_feats || !d_sizes || !d_idx || !d_grads || batch == 0 || batch > m->max_ctas * kStepThreads)
        return ms_fail(MS_ERR_INVALID, "mlp_grads: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned ctas = (batch + kStepThreads - 1) / kStepThreads;
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
    if (!m || !d_feats || !d_sizes || n == 0 || batch == 0 || batch > m->max_ctas * kStepThreads)
        return ms_fail(MS_ERR_INVALID, "mlp_train: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned ctas = (batch + kStepThreads - 1) / kStepThreads;
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
    const unsigned grid = unsigned(minu((n + 127) / 128, uint64_t(persistent_grid(128, 8))));
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
