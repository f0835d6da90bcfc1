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

__global__ void k_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t z = mix64(seed, i);
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

extern "C" int ms_gpu_gen_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *d_out, void *stream) {
    if (!d_out && n) return ms_fail(MS_ERR_INVALID, "gen_uniform_bits: null output");
    if (!n) return MS_OK;
    ms::k_uniform_bits<<<ms::persistent_grid(256, 8), 256, 0, (cudaStream_t)stream>>>(seed, bits, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_gen_from_table(uint64_t seed, const uint64_t *d_table, uint64_t n_table, uint64_t n,
                                     uint64_t *d_out, void *stream) {
    if ((!d_out || !d_table || !n_table) && n) return ms_fail(MS_ERR_INVALID, "gen_from_table: bad argument");
    if (!n) return MS_OK;
    ms::k_from_table<<<ms::persistent_grid(256, 8), 256, 0, (cudaStream_t)stream>>>(seed, d_table, n_table, n, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}
