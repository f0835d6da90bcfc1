// ms_common.cuh -- shared definitions of the B200 compression-aware path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ms_gpu.h"

namespace ms {

// Reference layout constants (AVX-512 defaults, default_formats.h:35-82).
constexpr unsigned kStep = 8;             // vbp_l<bw,8>: 8 interleaved lanes
constexpr unsigned kBlock = 512;          // values per vbp block (64 * step)
constexpr unsigned kPageBlocks = 64;      // dynamic_vbp_f<512,64,8> page
constexpr unsigned kMeta = 64;            // dvbp page header bytes
constexpr unsigned kNoBlock = 0xFF;       // VBP_BW_NOBLOCK (vbp_commons.h:54)
constexpr unsigned kCascBlock = 1024;     // delta_f / for_f block
constexpr unsigned kForPageBlocks = 8;    // for_f page
constexpr unsigned kWiBuffer = 2048;      // write iterator buffer (write_iterator.h:78-80)

// Device error flags (set by kernels, read by the host after the launch).
enum : unsigned { kErrNone = 0, kErrCorrupt = 1, kErrTimeout = 2, kErrCapacity = 4 };

// Block-index entry: byte offset (low 56 bits) | bit width (high 8 bits).
__host__ __device__ inline uint64_t idx_pack(uint64_t off, unsigned bw) {
    return off | (uint64_t(bw) << 56);
}
__host__ __device__ inline uint64_t idx_off(uint64_t e) { return e & ((uint64_t(1) << 56) - 1); }
__host__ __device__ inline unsigned idx_bw(uint64_t e) { return unsigned(e >> 56); }

__host__ __device__ inline unsigned effective_bitwidth(uint64_t v) {
#ifdef __CUDA_ARCH__
    return 64u - unsigned(__clzll((long long)(v | 1u)));
#else
    return 64u - unsigned(__builtin_clzll(v | 1u));
#endif
}

__host__ __device__ inline uint64_t minu(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ inline uint64_t maxu(uint64_t a, uint64_t b) { return a > b ? a : b; }

__host__ __device__ inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// F::get_size_max_byte(m_BlockSize): the size of one maximal block
// (vbp_format_rndaccess.h:71-73, dynamic_vbp.h:106-118, delta.h:91-101,
// for.h:99-111).
__host__ __device__ inline uint64_t max_block_bytes(int fmt, unsigned bw) {
    switch (fmt) {
    case MS_FMT_STATIC_VBP: return uint64_t(64) * bw;
    case MS_FMT_DYNAMIC_VBP: return 8 * 512 + 64;
    case MS_FMT_DELTA_DVBP: return 8 * 1024 + 2 * 64;
    case MS_FMT_FOR_DVBP: return 64 + 8 * 1024 + 2 * 64;
    default: return 0;
    }
}

__host__ __device__ inline uint64_t block_size(int fmt) {
    switch (fmt) {
    case MS_FMT_UNCOMPR: return 1;
    case MS_FMT_STATIC_VBP:
    case MS_FMT_DYNAMIC_VBP: return 512;
    case MS_FMT_DELTA_DVBP:
    case MS_FMT_FOR_DVBP: return 1024;
    default: return 0;
    }
}

// column<F>::create_data_uncompr_start (column.h:182-196) as an offset.
__host__ __device__ inline uint64_t rest_offset(int fmt, unsigned bw, uint64_t compr) {
    if (fmt == MS_FMT_UNCOMPR) return align_up(compr, 64);
    return align_up(compr + 2 * max_block_bytes(fmt, bw), 64);
}

// Number of values in the uncompressed rest (column.h:205-214).
__host__ __device__ inline uint64_t count_rest(const ms_col &c) {
    if (c.format == MS_FMT_UNCOMPR) return c.count_values;
    if (c.format == MS_FMT_RLE) return 0;
    if (c.size_compr_byte == c.size_used_byte) return 0;
    return (c.size_used_byte - rest_offset(c.format, c.bw, c.size_compr_byte)) / 8;
}

// Index of the first value handled by an operator's scalar remainder loop
// (select_compr.h:206-250): the rest values beyond its last full vector.
__host__ __device__ inline uint64_t scalar_from(const ms_col &c) {
    uint64_t nrest = count_rest(c);
    return c.count_values - nrest % kStep;
}

// Bounded spin: iterations before a device-side wait gives up.
constexpr unsigned kSpinLimit = 1u << 22;

}  // namespace ms

#define MS_CUDA_TRY(expr)                                  \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) return ms_fail_cuda(_e, #expr); \
    } while (0)

int ms_fail_cuda(cudaError_t e, const char *what);
int ms_fail(int status, const char *what);
