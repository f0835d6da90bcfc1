// vbp.cuh -- device bit-(un)packing of the vertical layout vbp_l<bw,8>.
//
// Layout (vbp_format_rndaccess.h:61-87; generated pack/unpack routines,
// vbp_routine_gen.py:61-180): a block holds 512 values; value j sits in lane
// j % 8 at slot j / 8; a lane's values are concatenated LSB-first in a stream
// of bw 64-bit words, and stream word w of lane l is stored at word index
// w * 8 + l.  A block occupies 64 * bw bytes.
//
// Decoding maps one warp to one block: thread t handles lane l = t & 7 and
// the quarter q = t >> 3 of that lane's stream, i.e. slots 16q .. 16q+15,
// which are the rows (16q + k) * 8 + l of the block (k = 0..15).  Within a
// quarter the first value starts at bit 16*q*bw of the stream; the thread
// loads the covering words, shifts them by the (runtime) start offset
// s0 in {0,16,32,48} and then extracts its 16 values at compile-time bit
// positions.  All bit widths are template instances, so every shift and mask
// is an immediate.
#pragma once

#include "ms_common.cuh"

namespace ms {

template <unsigned BW>
struct vbp_traits {
    static constexpr uint64_t mask = BW == 64 ? ~uint64_t(0) : ((uint64_t(1) << BW) - 1);
    static constexpr unsigned nr = (16 * BW + 63) / 64;  // normalised words per quarter
    static constexpr unsigned nw = nr + 1;                // raw words loaded per quarter
};

// Load helper: streaming read-only load.
__device__ __forceinline__ uint64_t ld_stream(const uint64_t *p) { return __ldg(p); }

// Decode the 16 values of quarter q of lane l from a block at `blk`
// (global or shared memory).  v[k] = value of row (16q + k) * 8 + l.
template <unsigned BW, bool kShared = false>
__device__ __forceinline__ void vbp_decode16(const uint64_t *__restrict__ blk, unsigned l, unsigned q,
                                             uint64_t (&v)[16]) {
    using T = vbp_traits<BW>;
    const unsigned sbit = 16u * q * BW;
    const unsigned w0 = sbit >> 6;
    const unsigned s0 = sbit & 63u;
    uint64_t w[T::nw];
#pragma unroll
    for (unsigned i = 0; i < T::nw; i++) {
        const unsigned wi = w0 + i;
        if (kShared) w[i] = wi < BW ? blk[wi * 8 + l] : 0;
        else w[i] = wi < BW ? ld_stream(blk + wi * 8 + l) : 0;
    }
    uint64_t r[T::nr];
    if (BW % 4 == 0) {
#pragma unroll
        for (unsigned i = 0; i < T::nr; i++) r[i] = w[i];
    } else {
#pragma unroll
        for (unsigned i = 0; i < T::nr; i++)
            r[i] = s0 ? ((w[i] >> s0) | (w[i + 1] << (64 - s0))) : w[i];
    }
#pragma unroll
    for (unsigned k = 0; k < 16; k++) {
        const unsigned p = k * BW, wi = p >> 6, sh = p & 63u;
        uint64_t x = r[wi] >> sh;
        if (sh + BW > 64) x |= r[wi + 1] << (64 - sh);
        v[k] = x & T::mask;
    }
}

// Runtime bit-width dispatch for a warp-uniform bw (1..64).  `fn` is called
// as fn(v) after the 16 values are decoded; returns false for an invalid bw.
template <bool kShared = false>
__device__ __forceinline__ bool vbp_decode16_rt(unsigned bw, const uint64_t *__restrict__ blk, unsigned l, unsigned q,
                                                uint64_t (&v)[16]) {
    switch (bw) {
#define MS_CASE(B) \
    case B: vbp_decode16<B, kShared>(blk, l, q, v); return true;
        MS_CASE(1) MS_CASE(2) MS_CASE(3) MS_CASE(4) MS_CASE(5) MS_CASE(6) MS_CASE(7) MS_CASE(8)
        MS_CASE(9) MS_CASE(10) MS_CASE(11) MS_CASE(12) MS_CASE(13) MS_CASE(14) MS_CASE(15) MS_CASE(16)
        MS_CASE(17) MS_CASE(18) MS_CASE(19) MS_CASE(20) MS_CASE(21) MS_CASE(22) MS_CASE(23) MS_CASE(24)
        MS_CASE(25) MS_CASE(26) MS_CASE(27) MS_CASE(28) MS_CASE(29) MS_CASE(30) MS_CASE(31) MS_CASE(32)
        MS_CASE(33) MS_CASE(34) MS_CASE(35) MS_CASE(36) MS_CASE(37) MS_CASE(38) MS_CASE(39) MS_CASE(40)
        MS_CASE(41) MS_CASE(42) MS_CASE(43) MS_CASE(44) MS_CASE(45) MS_CASE(46) MS_CASE(47) MS_CASE(48)
        MS_CASE(49) MS_CASE(50) MS_CASE(51) MS_CASE(52) MS_CASE(53) MS_CASE(54) MS_CASE(55) MS_CASE(56)
        MS_CASE(57) MS_CASE(58) MS_CASE(59) MS_CASE(60) MS_CASE(61) MS_CASE(62) MS_CASE(63) MS_CASE(64)
#undef MS_CASE
    default:
#pragma unroll
        for (unsigned k = 0; k < 16; k++) v[k] = 0;
        return false;
    }
}

// Pack lane l of one block: the 64 values in[v*8 + l] (v = 0..63, read
// through `get(v)`) are written as bw stream words out[w*8 + l].  Inputs are
// not masked, as in the reference's generated pack routine.
template <unsigned BW, class Get>
__device__ __forceinline__ void vbp_pack_lane(Get get, uint64_t *__restrict__ out, unsigned l) {
    uint64_t acc = 0;
    unsigned w = 0;
#pragma unroll
    for (unsigned v = 0; v < 64; v++) {
        const unsigned bit = v * BW, sh = bit & 63u;
        const uint64_t x = get(v);
        acc |= x << sh;
        if (sh + BW >= 64) {
            out[w * 8 + l] = acc;
            w++;
            acc = (sh + BW > 64) ? (x >> (64 - sh)) : 0;
        }
    }
}

template <class Get>
__device__ __forceinline__ bool vbp_pack_lane_rt(unsigned bw, Get get, uint64_t *__restrict__ out, unsigned l) {
    switch (bw) {
#define MS_CASE(B) \
    case B: vbp_pack_lane<B>(get, out, l); return true;
        MS_CASE(1) MS_CASE(2) MS_CASE(3) MS_CASE(4) MS_CASE(5) MS_CASE(6) MS_CASE(7) MS_CASE(8)
        MS_CASE(9) MS_CASE(10) MS_CASE(11) MS_CASE(12) MS_CASE(13) MS_CASE(14) MS_CASE(15) MS_CASE(16)
        MS_CASE(17) MS_CASE(18) MS_CASE(19) MS_CASE(20) MS_CASE(21) MS_CASE(22) MS_CASE(23) MS_CASE(24)
        MS_CASE(25) MS_CASE(26) MS_CASE(27) MS_CASE(28) MS_CASE(29) MS_CASE(30) MS_CASE(31) MS_CASE(32)
        MS_CASE(33) MS_CASE(34) MS_CASE(35) MS_CASE(36) MS_CASE(37) MS_CASE(38) MS_CASE(39) MS_CASE(40)
        MS_CASE(41) MS_CASE(42) MS_CASE(43) MS_CASE(44) MS_CASE(45) MS_CASE(46) MS_CASE(47) MS_CASE(48)
        MS_CASE(49) MS_CASE(50) MS_CASE(51) MS_CASE(52) MS_CASE(53) MS_CASE(54) MS_CASE(55) MS_CASE(56)
        MS_CASE(57) MS_CASE(58) MS_CASE(59) MS_CASE(60) MS_CASE(61) MS_CASE(62) MS_CASE(63) MS_CASE(64)
#undef MS_CASE
    default: return false;
    }
}

}  // namespace ms
