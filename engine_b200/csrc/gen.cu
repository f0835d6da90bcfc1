// gen.cu -- seeded synthetic data on the device.  Value i is a function of
// (seed, i) only: the i-th output of a splitmix64 stream started at `seed`
// (counter form), so host and device produce identical columns.
#include "internal.h"

namespace ms {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_uniform_bits(uint64_t seed, unsigned bits, uint64_t row0, uint64_t n,
                               uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t z = mix64(seed, row0 + i);
        out[i] = bits >= 64 ? z : (bits == 0 ? 0 : z >> (64 - bits));
    }
}

// Inverse-CDF draw: smallest k with u < table[k] (table[n_tab-1] = 2^64-1).
__global__ void k_from_table(uint64_t seed, const uint64_t *__restrict__ table, uint64_t n_tab, uint64_t n,
                             uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t u = mix64(seed, i);
        uint64_t lo = 0, hi = n_tab - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (u < table[mid]) hi = mid;
            else lo = mid + 1;
        }
        out[i] = lo;
    }
}

}  // namespace
}  // namespace ms

extern "C" int ms_gpu_gen_uniform_bits_at(uint64_t seed, unsigned bits, uint64_t row0, uint64_t n, uint64_t *d_out,
                                          void *stream) {
    if (!d_out && n) return ms_fail(MS_ERR_INVALID, "gen_uniform_bits: null output");
    if (!n) return MS_OK;
    ms::k_uniform_bits<<<ms::persistent_grid(256, 8), 256, 0, (cudaStream_t)stream>>>(seed, bits, row0, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_gen_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *d_out, void *stream) {
    return ms_gpu_gen_uniform_bits_at(seed, bits, 0, n, d_out, stream);
}

extern "C" int ms_gpu_gen_from_table(uint64_t seed, const uint64_t *d_table, uint64_t n_table, uint64_t n,
                                     uint64_t *d_out, void *stream) {
    if ((!d_out || !d_table || !n_table) && n) return ms_fail(MS_ERR_INVALID, "gen_from_table: bad argument");
    if (!n) return MS_OK;
    ms::k_from_table<<<ms::persistent_grid(256, 8), 256, 0, (cudaStream_t)stream>>>(seed, d_table, n_table, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// ---------------------------------------------------------------------------
// Sorted column with random gaps and run-structured column (the same values
// as the oracle's orc_gen_sorted_gaps / orc_gen_runs).
// ---------------------------------------------------------------------------
#include "scan.cuh"

namespace ms {
namespace {

__global__ void k_gap_draws(uint64_t seed, const uint64_t *__restrict__ table, uint64_t n_tab, uint64_t n,
                            uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t u = mix64(seed, i);
        uint64_t lo = 0, hi = n_tab - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (u < table[mid]) hi = mid;
            else lo = mid + 1;
        }
        out[i] = 1 + lo;
    }
}

__global__ void k_add_inclusive(const uint64_t *__restrict__ inc, uint64_t n, uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] += inc[i];
}

__global__ void k_run_heads(uint64_t seed, unsigned log2_len, uint64_t n, uint32_t *__restrict__ head) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        head[i] = (i > 0 && (mix64(seed, i) >> (64 - log2_len)) == 0) ? 1u : 0u;
}

__global__ void k_run_values(uint64_t seed, unsigned value_bits, const uint32_t *__restrict__ head,
                             const uint64_t *__restrict__ excl, uint64_t n, uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t run = excl[i] + head[i];
        const uint64_t z = mix64(seed ^ 0xD1B54A32D192ED03ull, run);
        out[i] = value_bits >= 64 ? z : z >> (64 - value_bits);
    }
}

}  // namespace
}  // namespace ms

extern "C" int ms_gpu_gen_sorted_gaps(uint64_t seed, const uint64_t *d_gap_table, uint64_t n_table, uint64_t n,
                                      uint64_t *d_out, ms_arena *a, void *stream) {
    using namespace ms;
    if (!a || (!d_out && n) || !d_gap_table || !n_table) return ms_fail(MS_ERR_INVALID, "gen_sorted_gaps: bad argument");
    if (!n) return MS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t mark = a->used;
    uint64_t *gaps = arena_take_t<uint64_t>(a, n);
    uint64_t *tot = arena_take_t<uint64_t>(a, 1);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(n, 1));
    if (!gaps || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (gen_sorted_gaps)");
    k_gap_draws<<<persistent_grid(256, 8), 256, 0, st>>>(seed, d_gap_table, n_table, n, gaps);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint64_t, 1>(gaps, n, d_out, tot, scr, st)));
    k_add_inclusive<<<persistent_grid(256, 8), 256, 0, st>>>(gaps, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    a->used = mark;
    return MS_OK;
}

extern "C" int ms_gpu_gen_runs(uint64_t seed, unsigned log2_mean_len, unsigned value_bits, uint64_t n, uint64_t *d_out,
                               ms_arena *a, void *stream) {
    using namespace ms;
    if (!a || (!d_out && n) || log2_mean_len < 1 || log2_mean_len > 63)
        return ms_fail(MS_ERR_INVALID, "gen_runs: bad argument");
    if (!n) return MS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t mark = a->used;
    uint32_t *head = arena_take_t<uint32_t>(a, n);
    uint64_t *excl = arena_take_t<uint64_t>(a, n);
    uint64_t *tot = arena_take_t<uint64_t>(a, 1);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(n, 1));
    if (!head || !excl || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (gen_runs)");
    k_run_heads<<<persistent_grid(256, 8), 256, 0, st>>>(seed, log2_mean_len, n, head);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(head, n, excl, tot, scr, st)));
    k_run_values<<<persistent_grid(256, 8), 256, 0, st>>>(seed, value_bits, head, excl, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    a->used = mark;
    return MS_OK;
}
