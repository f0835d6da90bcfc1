// stream.cuh -- a column seen as a run of 512-row vbp blocks laid out one
// after another in memory (page headers in between), for kernels that stage
// consecutive blocks into shared memory with one bulk copy per column.
#pragma once

#include "colview.cuh"

namespace ms {
namespace {

struct StreamCol {
    const uint8_t *base;
    const uint64_t *index;  // nullptr: fixed width
    unsigned fixed_bw;
    uint64_t nb;            // blocks available to the pipeline
};

__device__ __forceinline__ void blk_loc(const StreamCol &c, uint64_t b, uint64_t &off, unsigned &bw) {
    if (c.index) {
        const uint64_t e = __ldg(c.index + b);
        off = idx_off(e);
        bw = idx_bw(e);
    } else {
        bw = c.fixed_bw;
        off = b * 64ull * bw;
    }
}

// The block stream of a column: an uncompressed column's 512-row blocks are
// laid out as vbp_l<64,8> blocks of width 64.
inline StreamCol stream_of(const ColView &v) {
    StreamCol s{};
    if (v.fmt == MS_FMT_UNCOMPR) {
        s.base = reinterpret_cast<const uint8_t *>(v.rest);
        s.fixed_bw = 64;  // an uncompressed 512-row block is laid out as vbp_l<64,8>
        s.nb = v.n / kBlock;
    } else if (v.fmt == MS_FMT_STATIC_VBP) {
        s.base = v.data;
        s.fixed_bw = v.bw;
        s.nb = v.nb();
    } else {
        s.base = v.data;
        s.index = v.index;
        s.nb = v.nb();
    }
    return s;
}

// uncompr_f, static_vbp and dynamic_vbp blocks decode without a cascade
inline bool plain(const ColView &v) {
    return v.fmt == MS_FMT_UNCOMPR || v.fmt == MS_FMT_STATIC_VBP || v.fmt == MS_FMT_DYNAMIC_VBP;
}

}  // namespace
}  // namespace ms
