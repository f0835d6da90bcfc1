// colview.cuh -- a kernel-side view of a device column and the warp-level
// block decoder shared by every fused operator.
//
// A column is seen as a sequence of 512-row "blocks":
//   * blocks [0, nb) lie in the compressed main part and are vbp blocks
//     (static_vbp: fixed bw at b*64*bw; dynamic_vbp/delta/for: entry b of the
//     block index gives byte offset and bw; for_f adds the 1024-block
//     reference value, delta_f a per-block lane-wise carry-in);
//   * the remaining rows [n_compr, n) are the uncompressed rest, read row by
//     row (uncompr_f columns are all "rest", read 512 rows per block).
// Decompression is thereby fused into the consumer: decoded values only live
// in registers (decompress_and_process_batch, format.h:164-195).
#pragma once

#include "ms_common.cuh"
#include "vbp.cuh"

namespace ms {

struct ColView {
    int fmt;
    unsigned bw;               // static_vbp width
    const uint8_t *data;       // compressed main part
    const uint64_t *index;     // per-block (offset | bw << 56), dvbp family
    const uint64_t *aux;       // for_f: reference value per 1024-block
    const uint64_t *carry;     // delta_f: 8 lane carries per 512-block (exclusive)
    const uint64_t *rest;      // uncompressed rows [n_compr, n)
    uint64_t n;                // count_values
    uint64_t n_compr;          // rows in the compressed part (multiple of 512)
    uint64_t sfrom;            // first row of the scalar remainder
    __host__ __device__ uint64_t nb() const { return n_compr / kBlock; }
    __host__ __device__ uint64_t nblocks_total() const { return (n + kBlock - 1) / kBlock; }
};

// Cascade step after unpacking block b of the compressed part: for_f adds
// the 1024-block reference (for.h:385-467); delta_f turns the deltas into
// values with a lane-wise running sum -- thread-local over its 16 slots,
// across the four quarters of the lane by shuffles, plus the block's
// carry-in (delta.h:285-347).
// `side` is the block's reference (for_f) or this lane's carry-in (delta_f),
// loaded by cascade_side before the unpack so that its latency overlaps it.
__device__ __forceinline__ uint64_t cascade_side(const ColView &c, uint64_t b, unsigned l) {
    if (c.fmt == MS_FMT_FOR_DVBP) return __ldg(c.aux + (b >> 1));
    if (c.fmt == MS_FMT_DELTA_DVBP) return __ldg(c.carry + b * 8 + l);
    return 0;
}

__device__ __forceinline__ void apply_cascade(const ColView &c, uint64_t b, unsigned l, unsigned q,
                                              uint64_t (&v)[16], uint64_t side) {
    if (c.fmt == MS_FMT_FOR_DVBP) {
        const uint64_t ref = side;
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] += ref;
    } else if (c.fmt == MS_FMT_DELTA_DVBP) {
#pragma unroll
        for (int k = 1; k < 16; k++) v[k] += v[k - 1];
        const uint64_t tot = v[15];
        const uint64_t up = __shfl_up_sync(0xFFFFFFFFu, tot, 8);
        uint64_t pre = q >= 1 ? up : 0;
        const uint64_t up2 = __shfl_up_sync(0xFFFFFFFFu, tot + pre, 16);
        pre += q >= 2 ? up2 : 0;
        pre += side;
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] += pre;
    }
}

// Decode rows of block b for thread (l, q): v[k] = row b*512 + (16q+k)*8 + l.
// Rows >= n are returned as 0; `valid` gets bit k set for rows < n.
// Returns false (and sets *err) for a corrupt bit width.
__device__ __forceinline__ bool decode_block(const ColView &c, uint64_t b, unsigned l, unsigned q, uint64_t (&v)[16],
                                             unsigned &valid) {
    const uint64_t row0 = b * kBlock;
    if (b < c.nb()) {
        valid = 0xFFFFu;
        uint64_t off;
        unsigned bw;
        if (c.fmt == MS_FMT_STATIC_VBP) {
            bw = c.bw;
            off = b * uint64_t(64) * bw;
        } else {
            const uint64_t e = __ldg(c.index + b);
            off = idx_off(e);
            bw = idx_bw(e);
        }
        const uint64_t side = cascade_side(c, b, l);
        const bool ok = vbp_decode16_rt(bw, reinterpret_cast<const uint64_t *>(c.data + off), l, q, v);
        apply_cascade(c, b, l, q, v, side);
        return ok;
    }
    // uncompressed rows
    valid = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const uint64_t r = row0 + (16u * q + k) * 8u + l;
        if (r < c.n) {
            v[k] = __ldg(c.rest + (r - c.n_compr));
            valid |= 1u << k;
        } else {
            v[k] = 0;
        }
    }
    return true;
}

// Select comparison: signed before the scalar remainder, unsigned after
// (compare_avx512.h:35-111 vs compare_scalar.h:17-77).
__device__ __forceinline__ bool cmp_eval(int cmp, uint64_t a, uint64_t b, bool sgn) {
    const int64_t x = (int64_t)a, y = (int64_t)b;
    switch (cmp) {
    case MS_CMP_EQ: return a == b;
    case MS_CMP_LT: return sgn ? x < y : a < b;
    case MS_CMP_LE: return sgn ? x <= y : a <= b;
    case MS_CMP_GT: return sgn ? x > y : a > b;
    default: return sgn ? x >= y : a >= b;
    }
}

// Hit mask of thread (l, q) in block b: bit k set if row (16q+k)*8+l passes.
__device__ __forceinline__ unsigned select_mask(const ColView &c, uint64_t b, unsigned l, unsigned q,
                                                const uint64_t (&v)[16], unsigned valid, int cmp, uint64_t val) {
    unsigned m = 0;
    const uint64_t row0 = b * kBlock;
    // rows of this block all precede the scalar remainder in the common case
    if (row0 + kBlock <= c.sfrom) {
#pragma unroll
        for (int k = 0; k < 16; k++) m |= unsigned(cmp_eval(cmp, v[k], val, true)) << k;
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint64_t r = row0 + (16u * q + k) * 8u + l;
            m |= unsigned(cmp_eval(cmp, v[k], val, r < c.sfrom)) << k;
        }
    }
    return m & valid;
}

// Rank of each hit of thread (l, q) within its block, in row order
// (q, k, l).  base[k] receives the in-block rank of slot k's row (valid only
// where the hit bit is set); returns the block's total hit count.
__device__ __forceinline__ unsigned block_ranks(unsigned hits, unsigned l, unsigned q, unsigned (&rank)[16]) {
    const unsigned qmask = 0xFFu << (8u * q);
    const unsigned below_q = (1u << (8u * q)) - 1u;
    const unsigned lane_lt = (1u << l) - 1u;
    unsigned before = 0, run = 0, total = 0;
    unsigned b[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        b[k] = __ballot_sync(0xFFFFFFFFu, (hits >> k) & 1u);
        before += __popc(b[k] & below_q);
        total += __popc(b[k]);
    }
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const unsigned byte = (b[k] & qmask) >> (8u * q);
        rank[k] = before + run + __popc(byte & lane_lt);
        run += __popc(byte);
    }
    return total;
}

}  // namespace ms
