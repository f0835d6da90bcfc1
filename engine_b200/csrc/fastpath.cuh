// fastpath.cuh -- predicate and sum evaluated inside the bit-width switch.
//
// For plain vbp blocks (static_vbp, dynamic_vbp, uncompressed viewed as
// vbp_l<64,8>) the value range of a block is known at compile time inside
// each switch case: values of a bw-bit block are < 2^bw.  The select
// predicate therefore reduces to one unsigned threshold test, and for
// bw <= 32 decoding, comparing and summing run on 32-bit registers (one
// funnel shift + one mask per value) instead of 64-bit pairs.
//
// Predicate reduction (values v < 2^63, compared as signed 64-bit integers
// as the reference's AVX-512 primitives do, compare_avx512.h:35-111):
//   less c      : v <  T, T = c if (int64)c > 0 else 0
//   lessequal c : v <  T, T = c+1 if (int64)c >= 0 else 0
//   greater c   : !(v < T) with T of lessequal;  greaterequal: !(v < T) of less
//   equal c     : v == c
// 64-bit blocks (values may reach 2^63) use the signed compare directly.
#pragma once

#include "colview.cuh"

namespace ms {

struct Pred {
    int cmp;        // original comparison (64-bit blocks)
    uint64_t val;   // original constant
    int is_eq;      // equal
    uint64_t T;     // threshold (v < T), in [0, 2^63]
    int flip;       // negate the threshold test
};

inline Pred make_pred(int cmp, uint64_t c) {
    Pred p{cmp, c, cmp == MS_CMP_EQ, 0, 0};
    const int64_t cs = (int64_t)c;
    switch (cmp) {
    case MS_CMP_LT: p.T = cs > 0 ? c : 0; break;
    case MS_CMP_LE: p.T = cs >= 0 ? c + 1 : 0; break;
    case MS_CMP_GT: p.T = cs >= 0 ? c + 1 : 0; p.flip = 1; break;
    case MS_CMP_GE: p.T = cs > 0 ? c : 0; p.flip = 1; break;
    default: break;
    }
    return p;
}

// 16 values of quarter q of lane l as 32-bit integers (bw <= 32).
template <unsigned BW>
__device__ __forceinline__ void vbp_decode16_u32(const uint64_t *__restrict__ blk, unsigned l, unsigned q,
                                                 uint32_t (&v)[16]) {
    static_assert(BW <= 32, "32-bit decode");
    constexpr unsigned NW = (16 * BW + 63) / 64 + 1;  // 64-bit words covering the quarter (+1 for the shift)
    constexpr unsigned NH = (16 * BW + 31) / 32 + 1;  // 32-bit words after normalisation (+1 spare)
    const unsigned sbit = 16u * q * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t h[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        h[2 * i] = uint32_t(w);
        h[2 * i + 1] = uint32_t(w >> 32);
    }
    // start inside the loaded words: o whole 32-bit words, then t bits (0 or 16)
    const unsigned o = (sbit >> 5) & 1u;
    const unsigned t = sbit & 31u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        const uint32_t a = (i + 1 < 2 * NW) ? (o ? h[i + 1] : h[i]) : 0;
        const uint32_t b = (i + 2 < 2 * NW) ? (o ? h[i + 2] : h[i + 1]) : ((i + 1 < 2 * NW && !o) ? h[i + 1] : 0);
        n[i] = (BW % 2 == 0) ? a : __funnelshift_r(a, b, t);
    }
    constexpr uint32_t M = BW == 32 ? 0xFFFFFFFFu : ((1u << BW) - 1u);
#pragma unroll
    for (unsigned k = 0; k < 16; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        uint32_t x = (sh + BW <= 32) ? (n[wi] >> sh) : __funnelshift_r(n[wi], n[wi + 1], sh);
        v[k] = x & M;
    }
}

// v < T for the 16 values of quarter q of lane l (BW <= 32, T < 2^BW) on
// top-aligned fields: the bits below a field shifted to the top of a 32-bit
// word are less than 2^(32-BW), so  v < T  <=>  top < T * 2^(32-BW).
template <unsigned BW>
__device__ __forceinline__ unsigned vbp_lt16_top(const uint64_t *__restrict__ blk, unsigned l, unsigned q,
                                                 uint32_t T) {
    static_assert(BW <= 32, "32-bit fields");
    constexpr unsigned NW = (16 * BW + 63) / 64 + 1;
    constexpr unsigned NH = (16 * BW + 31) / 32 + 1;
    const unsigned sbit = 16u * q * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t h[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        h[2 * i] = uint32_t(w);
        h[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;
    const unsigned t = sbit & 31u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        const uint32_t a = (i + 1 < 2 * NW) ? (o ? h[i + 1] : h[i]) : 0;
        const uint32_t b = (i + 2 < 2 * NW) ? (o ? h[i + 2] : h[i + 1]) : ((i + 1 < 2 * NW && !o) ? h[i + 1] : 0);
        n[i] = (BW % 2 == 0) ? a : __funnelshift_r(a, b, t);
    }
    const uint32_t Tt = BW == 32 ? T : (T << (32u - BW));
    unsigned m = 0;
#pragma unroll
    for (unsigned k = 0; k < 16; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t top = (sh + BW <= 32) ? (n[wi] << (32u - sh - BW)) : __funnelshift_r(n[wi], n[wi + 1], sh + BW - 32u);
        m |= unsigned(top < Tt) << k;
    }
    return m;
}

template <unsigned BW>
__device__ __forceinline__ unsigned mask_block(const uint64_t *blk, unsigned l, unsigned q, const Pred &p) {
    unsigned m = 0;
    if (BW <= 32 && !p.is_eq && p.T < (uint64_t(1) << (BW <= 32 ? BW : 32))) {
        m = vbp_lt16_top<(BW <= 32 ? BW : 32)>(blk, l, q, uint32_t(p.T));
        if (p.flip) m ^= 0xFFFFu;
    } else if (BW <= 32) {
        uint32_t v[16];
        vbp_decode16_u32<(BW <= 32 ? BW : 32)>(blk, l, q, v);
        if (p.is_eq) {
            const bool in = p.val < (uint64_t(1) << 32);
            const uint32_t c = uint32_t(p.val);
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(in && v[k] == c) << k;
        } else {
            const bool big = p.T > 0xFFFFFFFFull;  // every value is below T
            const uint32_t T = uint32_t(p.T);
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(big || v[k] < T) << k;
            if (p.flip) m ^= 0xFFFFu;
        }
    } else {
        uint64_t v[16];
        vbp_decode16<BW, true>(blk, l, q, v);
        if (BW == 64) {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(cmp_eval(p.cmp, v[k], p.val, true)) << k;
        } else if (p.is_eq) {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(v[k] == p.val) << k;
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(v[k] < p.T) << k;
            if (p.flip) m ^= 0xFFFFu;
        }
    }
    return m;
}

template <unsigned BW>
__device__ __forceinline__ uint64_t sum_block(const uint64_t *blk, unsigned l, unsigned q, unsigned m) {
    if (BW <= 27) {  // 16 values of < 2^27 fit a 32-bit partial sum
        uint32_t v[16];
        vbp_decode16_u32<(BW <= 27 ? BW : 27)>(blk, l, q, v);
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
        return s;
    } else {
        uint64_t v[16];
        vbp_decode16<BW, true>(blk, l, q, v);
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0;
        return s;
    }
}

#define MS_BW_CASES(X)                                                                                  \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) \
    X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32) X(33) X(34)   \
    X(35) X(36) X(37) X(38) X(39) X(40) X(41) X(42) X(43) X(44) X(45) X(46) X(47) X(48) X(49) X(50)   \
    X(51) X(52) X(53) X(54) X(55) X(56) X(57) X(58) X(59) X(60) X(61) X(62) X(63) X(64)

// Hit mask of a plain vbp block (bit k = row (16q+k)*8+l); bw 0 or > 64
// sets *bad.
__device__ __forceinline__ unsigned mask_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned q,
                                                  const Pred &p, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return mask_block<B>(blk, l, q, p);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; return 0;
    }
}

__device__ __forceinline__ uint64_t sum_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned q,
                                                 unsigned m, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return sum_block<B>(blk, l, q, m);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; return 0;
    }
}

}  // namespace ms

namespace ms {

// ---------------------------------------------------------------------------
// 32 values per thread: thread (l, h) of a half-warp decodes slots 32h..32h+31
// of lane l, i.e. rows (32h + k) * 8 + l.  The half starts at bit 32*h*bw,
// always on a 32-bit word boundary, so even widths need no realignment and
// odd widths only a word select.
// ---------------------------------------------------------------------------
template <unsigned BW>
__device__ __forceinline__ void vbp_decode32_u32(const uint64_t *__restrict__ blk, unsigned l, unsigned h,
                                                 uint32_t (&v)[32]) {
    static_assert(BW <= 32, "32-bit decode");
    constexpr unsigned NW = (32 * BW + 63) / 64 + 1;
    constexpr unsigned NH = BW + 1;
    const unsigned sbit = 32u * h * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t hw[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        hw[2 * i] = uint32_t(w);
        hw[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;  // 0 for even widths
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        if (BW % 2 == 0) n[i] = (i < 2 * NW) ? hw[i] : 0;
        else n[i] = (i + 1 < 2 * NW) ? (o ? hw[i + 1] : hw[i]) : ((i < 2 * NW && !o) ? hw[i] : 0);
    }
    constexpr uint32_t M = BW == 32 ? 0xFFFFFFFFu : ((1u << BW) - 1u);
#pragma unroll
    for (unsigned k = 0; k < 32; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t x = (sh + BW <= 32) ? (n[wi] >> sh) : __funnelshift_r(n[wi], n[wi + 1], sh);
        v[k] = x & M;
    }
}

// Threshold test v < T for the 32 values of half h of lane l (BW <= 32,
// T < 2^BW) without isolating the values: each field is shifted to the top
// of a 32-bit word, where the bits below it (the next fields) are less than
// 2^(32-BW), so  v < T  <=>  top < T * 2^(32-BW).  One shift and one compare
// per value.
template <unsigned BW>
__device__ __forceinline__ unsigned vbp_lt32_top(const uint64_t *__restrict__ blk, unsigned l, unsigned h,
                                                 uint32_t T) {
    static_assert(BW <= 32, "32-bit fields");
    constexpr unsigned NW = (32 * BW + 63) / 64 + 1;
    constexpr unsigned NH = BW + 1;
    const unsigned sbit = 32u * h * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t hw[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        hw[2 * i] = uint32_t(w);
        hw[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        if (BW % 2 == 0) n[i] = (i < 2 * NW) ? hw[i] : 0;
        else n[i] = (i + 1 < 2 * NW) ? (o ? hw[i + 1] : hw[i]) : ((i < 2 * NW && !o) ? hw[i] : 0);
    }
    const uint32_t Tt = BW == 32 ? T : (T << (32u - BW));
    unsigned m = 0;
#pragma unroll
    for (unsigned k = 0; k < 32; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t top = (sh + BW <= 32) ? (n[wi] << (32u - sh - BW)) : __funnelshift_r(n[wi], n[wi + 1], sh + BW - 32u);
        m |= unsigned(top < Tt) << k;
    }
    return m;
}

template <unsigned BW>
__device__ __forceinline__ unsigned mask32_block(const uint64_t *blk, unsigned l, unsigned h, const Pred &p) {
    unsigned m = 0;
    if (BW <= 32 && !p.is_eq && p.T < (uint64_t(1) << (BW <= 32 ? BW : 32))) {
        m = vbp_lt32_top<(BW <= 32 ? BW : 32)>(blk, l, h, uint32_t(p.T));
        if (p.flip) m = ~m;
    } else if (BW <= 32) {
        uint32_t v[32];
        vbp_decode32_u32<(BW <= 32 ? BW : 32)>(blk, l, h, v);
        if (p.is_eq) {
            const bool in = p.val < (uint64_t(1) << 32);
            const uint32_t c = uint32_t(p.val);
#pragma unroll
            for (int k = 0; k < 32; k++) m |= unsigned(in && v[k] == c) << k;
        } else {
            const bool big = p.T > 0xFFFFFFFFull;
            const uint32_t T = uint32_t(p.T);
#pragma unroll
            for (int k = 0; k < 32; k++) m |= unsigned(big || v[k] < T) << k;
            if (p.flip) m = ~m;
        }
    } else {
        m = mask_block<BW>(blk, l, 2 * h, p) | (mask_block<BW>(blk, l, 2 * h + 1, p) << 16);
    }
    return m;
}

template <unsigned BW>
__device__ __forceinline__ uint64_t sum32_block(const uint64_t *blk, unsigned l, unsigned h, unsigned m) {
    if (BW <= 26) {  // 32 values of < 2^26 fit a 32-bit partial sum
        uint32_t v[32];
        vbp_decode32_u32<(BW <= 26 ? BW : 26)>(blk, l, h, v);
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < 32; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
        return s;
    } else {
        return sum_block<BW>(blk, l, 2 * h, m & 0xFFFFu) + sum_block<BW>(blk, l, 2 * h + 1, m >> 16);
    }
}

__device__ __forceinline__ unsigned mask32_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned h,
                                                    const Pred &p, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return mask32_block<B>(blk, l, h, p);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; return 0;
    }
}

__device__ __forceinline__ uint64_t sum32_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned h,
                                                   unsigned m, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return sum32_block<B>(blk, l, h, m);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; return 0;
    }
}

}  // namespace ms

namespace ms {

// ---------------------------------------------------------------------------
// Selection flags: the predicate of x and the sum over y meet in 32 flags
// (0 or 1, one register per value of the half) instead of a bit mask, so
// the y side multiplies-and-adds (s += v * flag, an integer multiply-add)
// rather than testing a mask bit and adding under a predicate, and fields are
// isolated as (w << a) >> b.  Both moves take work off the integer ALU,
// which bounds the fused kernel.
// ---------------------------------------------------------------------------
template <unsigned BW, bool kFlip>
__device__ __forceinline__ unsigned vbp_sel32_top(const uint64_t *__restrict__ blk, unsigned l, unsigned h,
                                                  uint32_t T, uint32_t (&sel)[32]) {
    static_assert(BW <= 32, "32-bit fields");
    constexpr unsigned NW = (32 * BW + 63) / 64 + 1;
    constexpr unsigned NH = BW + 1;
    const unsigned sbit = 32u * h * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t hw[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        hw[2 * i] = uint32_t(w);
        hw[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        if (BW % 2 == 0) n[i] = (i < 2 * NW) ? hw[i] : 0;
        else n[i] = (i + 1 < 2 * NW) ? (o ? hw[i + 1] : hw[i]) : ((i < 2 * NW && !o) ? hw[i] : 0);
    }
    const uint32_t Tt = BW == 32 ? T : (T << (32u - BW));
    unsigned c0 = 0, c1 = 0;
#pragma unroll
    for (unsigned k = 0; k < 32; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t top = (sh + BW <= 32) ? (n[wi] << (32u - sh - BW)) : __funnelshift_r(n[wi], n[wi + 1], sh + BW - 32u);
        const bool lt = top < Tt;
        sel[k] = (kFlip ? !lt : lt) ? 1u : 0u;
        if (k & 1) c1 += sel[k];
        else c0 += sel[k];
    }
    return c0 + c1;
}

// Flags of the 32 values of half h of lane l of a plain vbp block of width
// bw; returns how many are set.  bw 0 or > 64 sets *bad.
__device__ __forceinline__ unsigned sel32_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned h,
                                                   const Pred &p, uint32_t (&sel)[32], bool &bad) {
    if (bw >= 1 && bw <= 32 && !p.is_eq && p.T < (uint64_t(1) << bw)) {
        switch (bw) {
#define MS_X(B)                                                                                              \
    case B:                                                                                                  \
        return p.flip ? vbp_sel32_top<(B <= 32 ? B : 32), true>(blk, l, h, uint32_t(p.T), sel)               \
                      : vbp_sel32_top<(B <= 32 ? B : 32), false>(blk, l, h, uint32_t(p.T), sel);
            MS_X(1) MS_X(2) MS_X(3) MS_X(4) MS_X(5) MS_X(6) MS_X(7) MS_X(8) MS_X(9) MS_X(10) MS_X(11) MS_X(12)
            MS_X(13) MS_X(14) MS_X(15) MS_X(16) MS_X(17) MS_X(18) MS_X(19) MS_X(20) MS_X(21) MS_X(22) MS_X(23)
            MS_X(24) MS_X(25) MS_X(26) MS_X(27) MS_X(28) MS_X(29) MS_X(30) MS_X(31) MS_X(32)
#undef MS_X
        default: break;
        }
    }
    const unsigned m = mask32_block_rt(bw, blk, l, h, p, bad);
#pragma unroll
    for (unsigned k = 0; k < 32; k++) sel[k] = (m >> k) & 1u;
    return __popc(m);
}

// Sum of the flagged values among the 32 of half h of lane l (BW <= 26, so
// the 32-bit partial cannot overflow).
template <unsigned BW>
__device__ __forceinline__ uint32_t sum32_sel(const uint64_t *__restrict__ blk, unsigned l, unsigned h,
                                              const uint32_t (&sel)[32]) {
    static_assert(BW <= 26, "32-bit partial sums");
    constexpr unsigned NW = (32 * BW + 63) / 64 + 1;
    constexpr unsigned NH = BW + 1;
    const unsigned sbit = 32u * h * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t hw[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        hw[2 * i] = uint32_t(w);
        hw[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        if (BW % 2 == 0) n[i] = (i < 2 * NW) ? hw[i] : 0;
        else n[i] = (i + 1 < 2 * NW) ? (o ? hw[i + 1] : hw[i]) : ((i < 2 * NW && !o) ? hw[i] : 0);
    }
    uint32_t s0 = 0, s1 = 0;
#pragma unroll
    for (unsigned k = 0; k < 32; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t top = (sh + BW <= 32) ? (n[wi] << (32u - sh - BW)) : __funnelshift_r(n[wi], n[wi + 1], sh + BW - 32u);
        const uint32_t v = top >> (32u - BW);
        if (k & 1) s1 += v * sel[k];
        else s0 += v * sel[k];
    }
    return s0 + s1;
}

__device__ __forceinline__ uint64_t sum32_sel_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned h,
                                                 const uint32_t (&sel)[32], bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return sum32_sel<(B <= 26 ? B : 26)>(blk, l, h, sel);
        MS_X(1) MS_X(2) MS_X(3) MS_X(4) MS_X(5) MS_X(6) MS_X(7) MS_X(8) MS_X(9) MS_X(10) MS_X(11) MS_X(12) MS_X(13)
        MS_X(14) MS_X(15) MS_X(16) MS_X(17) MS_X(18) MS_X(19) MS_X(20) MS_X(21) MS_X(22) MS_X(23) MS_X(24) MS_X(25)
        MS_X(26)
#undef MS_X
    default: break;
    }
    unsigned m = 0;
#pragma unroll
    for (unsigned k = 0; k < 32; k++) m |= sel[k] << k;
    return sum32_block_rt(bw, blk, l, h, m, bad);
}

}  // namespace ms

namespace ms {

// Select and sum over the same plain vbp block, decoded once: cnt gets the
// number of rows of thread (l, q) that pass, the return value their sum.
template <unsigned BW>
__device__ __forceinline__ uint64_t self_sum_block(const uint64_t *blk, unsigned l, unsigned q, const Pred &p,
                                                   unsigned &cnt) {
    unsigned m = 0;
    if (BW <= 32) {
        uint32_t v[16];
        vbp_decode16_u32<(BW <= 32 ? BW : 32)>(blk, l, q, v);
        if (p.is_eq) {
            const bool in = p.val < (uint64_t(1) << 32);
            const uint32_t c = uint32_t(p.val);
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(in && v[k] == c) << k;
        } else {
            const bool big = p.T > 0xFFFFFFFFull;
            const uint32_t T = uint32_t(p.T);
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(big || v[k] < T) << k;
            if (p.flip) m ^= 0xFFFFu;
        }
        cnt = __popc(m);
        if (BW <= 27) {
            uint32_t s = 0;
#pragma unroll
            for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
            return s;
        }
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
        return s;
    } else {
        uint64_t v[16];
        vbp_decode16<BW, true>(blk, l, q, v);
        if (BW == 64) {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(cmp_eval(p.cmp, v[k], p.val, true)) << k;
        } else if (p.is_eq) {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(v[k] == p.val) << k;
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(v[k] < p.T) << k;
            if (p.flip) m ^= 0xFFFFu;
        }
        cnt = __popc(m);
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0;
        return s;
    }
}

__device__ __forceinline__ uint64_t self_sum_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned q,
                                                      const Pred &p, unsigned &cnt, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return self_sum_block<B>(blk, l, q, p, cnt);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; cnt = 0; return 0;
    }
}

}  // namespace ms

namespace ms {

// self_sum_block with 32 values per thread: thread (l, h) of a half-warp
// takes slots 32h..32h+31 of lane l (word-aligned half streams); wider
// blocks fall back to the 16-value form on quarters 2h and 2h+1.
// Threshold select + sum of the same 32 values on top-aligned fields: the
// test is `top < T * 2^(32-BW)` (see vbp_lt32_top), the value
// `top >> (32-BW)`; the hit becomes a 0/1 flag that multiplies the value into
// the sum and adds to the count (integer multiply-adds instead of predicated
// adds on the ALU).
template <unsigned BW, bool kFlip>
__device__ __forceinline__ uint64_t vbp_ltsum32_top(const uint64_t *__restrict__ blk, unsigned l, unsigned h,
                                                    uint32_t T, unsigned &cnt) {
    static_assert(BW <= 32, "32-bit fields");
    constexpr unsigned NW = (32 * BW + 63) / 64 + 1;
    constexpr unsigned NH = BW + 1;
    const unsigned sbit = 32u * h * BW;
    const unsigned w0 = sbit >> 6;
    uint32_t hw[2 * NW];
#pragma unroll
    for (unsigned i = 0; i < NW; i++) {
        const uint64_t w = (w0 + i < BW) ? blk[(w0 + i) * 8 + l] : 0;
        hw[2 * i] = uint32_t(w);
        hw[2 * i + 1] = uint32_t(w >> 32);
    }
    const unsigned o = (sbit >> 5) & 1u;
    uint32_t n[NH];
#pragma unroll
    for (unsigned i = 0; i < NH; i++) {
        if (BW % 2 == 0) n[i] = (i < 2 * NW) ? hw[i] : 0;
        else n[i] = (i + 1 < 2 * NW) ? (o ? hw[i + 1] : hw[i]) : ((i < 2 * NW && !o) ? hw[i] : 0);
    }
    const uint32_t Tt = BW == 32 ? T : (T << (32u - BW));
    uint32_t c0 = 0, c1 = 0, s0 = 0, s1 = 0;
    uint64_t s64 = 0;
#pragma unroll
    for (unsigned k = 0; k < 32; k++) {
        const unsigned p = k * BW, wi = p >> 5, sh = p & 31u;
        const uint32_t top = (sh + BW <= 32) ? (n[wi] << (32u - sh - BW)) : __funnelshift_r(n[wi], n[wi + 1], sh + BW - 32u);
        const bool lt = top < Tt;
        const uint32_t f = (kFlip ? !lt : lt) ? 1u : 0u;
        const uint32_t v = BW == 32 ? top : (top >> (32u - BW));
        if (k & 1) c1 += f;
        else c0 += f;
        if (BW <= 26) {  // 32 values of < 2^26 fit a 32-bit partial sum
            if (k & 1) s1 += v * f;
            else s0 += v * f;
        } else {
            s64 += uint64_t(v) * f;
        }
    }
    cnt = c0 + c1;
    return BW <= 26 ? uint64_t(s0) + s1 : s64;
}

template <unsigned BW>
__device__ __forceinline__ uint64_t self_sum32_block(const uint64_t *blk, unsigned l, unsigned h, const Pred &p,
                                                     unsigned &cnt) {
    if (BW <= 32 && !p.is_eq && p.T < (uint64_t(1) << (BW <= 32 ? BW : 32))) {
        return p.flip ? vbp_ltsum32_top<(BW <= 32 ? BW : 32), true>(blk, l, h, uint32_t(p.T), cnt)
                      : vbp_ltsum32_top<(BW <= 32 ? BW : 32), false>(blk, l, h, uint32_t(p.T), cnt);
    } else if (BW <= 32) {
        uint32_t v[32];
        vbp_decode32_u32<(BW <= 32 ? BW : 32)>(blk, l, h, v);
        unsigned m = 0;
        if (p.is_eq) {
            const bool in = p.val < (uint64_t(1) << 32);
            const uint32_t c = uint32_t(p.val);
#pragma unroll
            for (int k = 0; k < 32; k++) m |= unsigned(in && v[k] == c) << k;
        } else {
            const bool big = p.T > 0xFFFFFFFFull;
            const uint32_t T = uint32_t(p.T);
#pragma unroll
            for (int k = 0; k < 32; k++) m |= unsigned(big || v[k] < T) << k;
            if (p.flip) m = ~m;
        }
        cnt = __popc(m);
        if (BW <= 26) {  // 32 values of < 2^26 fit a 32-bit partial sum
            uint32_t s = 0;
#pragma unroll
            for (int k = 0; k < 32; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
            return s;
        }
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 32; k++) s += ((m >> k) & 1u) ? v[k] : 0u;
        return s;
    } else {
        unsigned c0 = 0, c1 = 0;
        const uint64_t s = self_sum_block<BW>(blk, l, 2 * h, p, c0) + self_sum_block<BW>(blk, l, 2 * h + 1, p, c1);
        cnt = c0 + c1;
        return s;
    }
}

__device__ __forceinline__ uint64_t self_sum32_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned h,
                                                        const Pred &p, unsigned &cnt, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return self_sum32_block<B>(blk, l, h, p, cnt);
        MS_BW_CASES(MS_X)
#undef MS_X
    default: bad = true; cnt = 0; return 0;
    }
}

}  // namespace ms
