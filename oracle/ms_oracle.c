/*
 * ms_oracle.c -- CPU oracle (test infrastructure only; see ms_oracle.h).
 *
 * Each function names the reference code it restates.  Reference paths are
 * relative to the MorphStore/Engine source tree.
 */
#include "ms_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define STEP 8u
#define VBP_BLOCK 512u          /* vbp_l<bw,8>::m_BlockSize = 8 * 64 */
#define DVBP_PAGE_BLOCKS 64u    /* dynamic_vbp_f<512,64,8> */
#define DVBP_META 64u
#define DVBP_NOBLOCK 0xFFu      /* VBP_BW_NOBLOCK, include/core/morphing/vbp_commons.h:54 */
#define CASC_BLOCK 1024u        /* delta_f<1024,..>, for_f<1024,8,..> */
#define FOR_PAGE_BLOCKS 8u
#define WI_BUFFER 2048u         /* write_iterator.h:78-80: round_up(m_BlockSize, 2048) */

static uint64_t align64(uint64_t x) { return (x + 63u) & ~(uint64_t)63u; }

/* include/core/utils/math.h:108-113 */
unsigned orc_effective_bitwidth(uint64_t v) {
    return 64u - (unsigned)__builtin_clzll(v | 1u);
}

/* m_BlockSize of each format (format.h:95, vbp_format_rndaccess.h:76,
 * dynamic_vbp.h:121, delta.h:104, for.h:163); rle_f has none (rle.h:42-49). */
uint64_t orc_block_size(int fmt) {
    switch (fmt) {
    case ORC_FMT_UNCOMPR: return 1;
    case ORC_FMT_STATIC_VBP: return VBP_BLOCK;
    case ORC_FMT_DYNAMIC_VBP: return VBP_BLOCK;
    case ORC_FMT_DELTA_DVBP: return CASC_BLOCK;
    case ORC_FMT_FOR_DVBP: return CASC_BLOCK;
    default: return 0;
    }
}

/* F::get_size_max_byte(n), n a multiple of the block size:
 * vbp_format_rndaccess.h:71-73, dynamic_vbp.h:106-118, delta.h:91-101,
 * for.h:99-111, rle.h:43-45. */
uint64_t orc_size_max_byte(int fmt, unsigned bw, uint64_t n) {
    switch (fmt) {
    case ORC_FMT_UNCOMPR: return 8 * n;
    case ORC_FMT_STATIC_VBP: return n * bw / 8;
    case ORC_FMT_DYNAMIC_VBP:
    case ORC_FMT_DELTA_DVBP: return 8 * n + (n / VBP_BLOCK) * DVBP_META;
    case ORC_FMT_FOR_DVBP: {
        uint64_t pages = (n + CASC_BLOCK * FOR_PAGE_BLOCKS - 1) / (CASC_BLOCK * FOR_PAGE_BLOCKS);
        uint64_t blocks = n / CASC_BLOCK;
        return pages * 8 * FOR_PAGE_BLOCKS +
               blocks * orc_size_max_byte(ORC_FMT_DYNAMIC_VBP, 0, CASC_BLOCK);
    }
    case ORC_FMT_RLE: return 16 * n;
    default: return 0;
    }
}

/* get_size_max_byte_any_len, format.h:114-153 (64-B alignment padding added
 * by get_size_with_alignment_padding is included as +64). */
uint64_t orc_size_max_byte_any_len(int fmt, unsigned bw, uint64_t n) {
    if (fmt == ORC_FMT_UNCOMPR) return 8 * n;
    if (fmt == ORC_FMT_RLE) return 16 * n + 16;
    uint64_t b = orc_block_size(fmt);
    uint64_t cnt = (n + b - 1) / b * b + b;
    uint64_t compr = orc_size_max_byte(fmt, bw, cnt);
    uint64_t unc = 8 * (n % b + b);
    /* plus the gap of two blocks before the rest, column.h:186-195 */
    return compr + 2 * orc_size_max_byte(fmt, bw, b) + 64 + unc + 64;
}

/* column<F>::create_data_uncompr_start, column.h:182-196, as an offset from a
 * 64-B aligned data start. */
uint64_t orc_rest_offset(int fmt, unsigned bw, uint64_t compr_bytes) {
    if (fmt == ORC_FMT_UNCOMPR) return align64(compr_bytes);
    return align64(compr_bytes + 2 * orc_size_max_byte(fmt, bw, orc_block_size(fmt)));
}

/* column<F>::get_count_values_uncompr, column.h:205-214 */
uint64_t orc_count_rest(int fmt, unsigned bw, const orc_meta *m) {
    if (m->size_compr_byte == m->size_used_byte) return 0;
    return (m->size_used_byte - orc_rest_offset(fmt, bw, m->size_compr_byte)) / 8;
}

/* ------------------------------------------------------------------------- */
/* vbp_l<bw,8> (vbp_format_rndaccess.h:61-87; pack/unpack as generated by
 * vbp_routine_gen.py:61-180).  Value j of a 512-block: lane j%8, slot j/8,
 * bit offset slot*bw in the lane's LSB-first word stream; stream word w of
 * lane l is stored at word index w*8+l.  Inputs are not masked on packing.  */
/* ------------------------------------------------------------------------- */
static void vbp_pack_block(const uint64_t *in, unsigned bw, uint64_t *out) {
    memset(out, 0, (size_t)8 * bw * 8);
    for (unsigned l = 0; l < STEP; l++) {
        for (unsigned v = 0; v < 64; v++) {
            uint64_t x = in[v * STEP + l];
            unsigned bit = v * bw, w = bit >> 6, s = bit & 63u;
            out[w * STEP + l] |= x << s;
            if (s + bw > 64) out[(w + 1) * STEP + l] |= x >> (64 - s);
        }
    }
}

static void vbp_unpack_block(const uint64_t *in, unsigned bw, uint64_t *out) {
    uint64_t mask = bw == 64 ? ~(uint64_t)0 : (((uint64_t)1 << bw) - 1);
    for (unsigned l = 0; l < STEP; l++) {
        for (unsigned v = 0; v < 64; v++) {
            unsigned bit = v * bw, w = bit >> 6, s = bit & 63u;
            uint64_t x = in[w * STEP + l] >> s;
            if (s + bw > 64) x |= in[(w + 1) * STEP + l] << (64 - s);
            out[v * STEP + l] = x & mask;
        }
    }
}

uint64_t orc_vbp_pack(const uint64_t *in, uint64_t n, unsigned bw, uint8_t *out) {
    uint64_t blk_bytes = (uint64_t)64 * bw;
    for (uint64_t b = 0; b < n / VBP_BLOCK; b++)
        vbp_pack_block(in + b * VBP_BLOCK, bw, (uint64_t *)(out + b * blk_bytes));
    return n / VBP_BLOCK * blk_bytes;
}

uint64_t orc_vbp_unpack(const uint8_t *in, uint64_t n, unsigned bw, uint64_t *out) {
    uint64_t blk_bytes = (uint64_t)64 * bw;
    for (uint64_t b = 0; b < n / VBP_BLOCK; b++)
        vbp_unpack_block((const uint64_t *)(in + b * blk_bytes), bw, out + b * VBP_BLOCK);
    return n / VBP_BLOCK * blk_bytes;
}

/* dynamic_vbp_f<512,64,8>: determine_max_bitwidth (dynamic_vbp.h:124-158),
 * compression (:176-258), decompression (:270-308). */
uint64_t orc_dvbp_pack(const uint64_t *in, uint64_t n, uint8_t *out) {
    uint64_t nblocks = n / VBP_BLOCK, o = 0;
    for (uint64_t b0 = 0; b0 < nblocks; b0 += DVBP_PAGE_BLOCKS) {
        uint8_t *meta = out + o;
        o += DVBP_META;
        uint64_t nb = nblocks - b0 < DVBP_PAGE_BLOCKS ? nblocks - b0 : DVBP_PAGE_BLOCKS;
        for (uint64_t j = 0; j < nb; j++) {
            const uint64_t *blk = in + (b0 + j) * VBP_BLOCK;
            uint64_t acc = 1;
            for (unsigned i = 0; i < VBP_BLOCK; i++) acc |= blk[i];
            unsigned bw = orc_effective_bitwidth(acc);
            meta[j] = (uint8_t)bw;
            vbp_pack_block(blk, bw, (uint64_t *)(out + o));
            o += (uint64_t)64 * bw;
        }
        for (uint64_t j = nb; j < DVBP_PAGE_BLOCKS; j++) meta[j] = DVBP_NOBLOCK;
    }
    return o;
}

uint64_t orc_dvbp_unpack(const uint8_t *in, uint64_t n, uint64_t *out) {
    uint64_t i = 0, o = 0;
    while (o < n) {
        const uint8_t *meta = in + i;
        i += DVBP_META;
        for (unsigned j = 0; j < DVBP_PAGE_BLOCKS; j++) {
            unsigned bw = meta[j];
            if (bw == DVBP_NOBLOCK) continue;
            vbp_unpack_block((const uint64_t *)(in + i), bw, out + o);
            i += (uint64_t)64 * bw;
            o += VBP_BLOCK;
        }
    }
    return i;
}

/* delta_f<1024,8,dvbp>::compress_batch (delta.h:107-156): d[i] = x[i]-x[i-8]
 * with the previous vector carried in `last` across blocks; each 1024-block
 * of deltas is a separate morph_batch<dvbp>(1024). */
uint64_t orc_delta_pack(const uint64_t *in, uint64_t n, uint8_t *out, uint64_t last[8]) {
    uint64_t tmp[CASC_BLOCK], o = 0;
    for (uint64_t b = 0; b < n / CASC_BLOCK; b++) {
        const uint64_t *x = in + b * CASC_BLOCK;
        for (unsigned i = 0; i < CASC_BLOCK; i++) {
            tmp[i] = x[i] - last[i & 7u];
            last[i & 7u] = x[i];
        }
        o += orc_dvbp_pack(tmp, CASC_BLOCK, out + o);
    }
    return o;
}

/* delta decompression (delta.h:202-266): lane-wise running sum continuous
 * across blocks. */
uint64_t orc_delta_unpack(const uint8_t *in, uint64_t n, uint64_t *out) {
    uint64_t tmp[CASC_BLOCK], acc[8] = {0}, i = 0;
    for (uint64_t b = 0; b < n / CASC_BLOCK; b++) {
        i += orc_dvbp_unpack(in + i, CASC_BLOCK, tmp);
        for (unsigned k = 0; k < CASC_BLOCK; k++) {
            acc[k & 7u] += tmp[k];
            out[b * CASC_BLOCK + k] = acc[k & 7u];
        }
    }
    return i;
}

/* for_f::determine_reference_value (for.h:121-161) with the AVX-512 TVL min:
 * per lane signed 64-bit min (_mm512_min_epi64, calc_avx512.h:78), then an
 * unsigned minimum over the eight lanes; UINT64_MAX is decremented. */
static uint64_t for_reference(const uint64_t *blk) {
    int64_t lane_min[8];
    for (unsigned l = 0; l < 8; l++) lane_min[l] = (int64_t)blk[l];
    for (unsigned i = 8; i < CASC_BLOCK; i++) {
        int64_t v = (int64_t)blk[i];
        if (v < lane_min[i & 7u]) lane_min[i & 7u] = v;
    }
    uint64_t m = ~(uint64_t)0;
    for (unsigned l = 0; l < 8; l++)
        if ((uint64_t)lane_min[l] < m) m = (uint64_t)lane_min[l];
    if (m == ~(uint64_t)0) m--;
    return m;
}

/* for_f compression (for.h:183-273).  Header words after the end marker are
 * left uninitialised by the reference; they are written as 0 here. */
uint64_t orc_for_pack(const uint64_t *in, uint64_t n, uint8_t *out) {
    uint64_t tmp[CASC_BLOCK], o = 0, nblocks = n / CASC_BLOCK;
    for (uint64_t b0 = 0; b0 < nblocks; b0 += FOR_PAGE_BLOCKS) {
        uint64_t *meta = (uint64_t *)(out + o);
        o += 8 * FOR_PAGE_BLOCKS;
        uint64_t nb = nblocks - b0 < FOR_PAGE_BLOCKS ? nblocks - b0 : FOR_PAGE_BLOCKS;
        if (nb < FOR_PAGE_BLOCKS) {
            for (uint64_t j = nb; j < FOR_PAGE_BLOCKS; j++) meta[j] = 0;
            meta[nb] = ~(uint64_t)0;
        }
        for (uint64_t j = 0; j < nb; j++) {
            const uint64_t *x = in + (b0 + j) * CASC_BLOCK;
            uint64_t ref = for_reference(x);
            meta[j] = ref;
            for (unsigned i = 0; i < CASC_BLOCK; i++) tmp[i] = x[i] - ref;
            o += orc_dvbp_pack(tmp, CASC_BLOCK, out + o);
        }
    }
    return o;
}

/* for_f decompression (for.h:285-365). */
uint64_t orc_for_unpack(const uint8_t *in, uint64_t n, uint64_t *out) {
    uint64_t tmp[CASC_BLOCK], i = 0, o = 0;
    while (o < n) {
        const uint64_t *meta = (const uint64_t *)(in + i);
        i += 8 * FOR_PAGE_BLOCKS;
        for (unsigned j = 0; j < FOR_PAGE_BLOCKS; j++) {
            uint64_t ref = meta[j];
            if (ref == ~(uint64_t)0) break;
            i += orc_dvbp_unpack(in + i, CASC_BLOCK, tmp);
            for (unsigned k = 0; k < CASC_BLOCK; k++) out[o + k] = tmp[k] + ref;
            o += CASC_BLOCK;
        }
    }
    return i;
}

/* rle_f (rle.h:63-150): (value, length) pairs of maximal runs.  For n == 0
 * the reference reads in[0] and emits one pair; here no pair is emitted. */
uint64_t orc_rle_pack(const uint64_t *in, uint64_t n, uint8_t *out) {
    uint64_t *o = (uint64_t *)out, runs = 0;
    if (n == 0) return 0;
    uint64_t cur = in[0], start = 0;
    for (uint64_t i = 1; i < n; i++) {
        if (in[i] != cur) {
            o[2 * runs] = cur;
            o[2 * runs + 1] = i - start;
            runs++;
            cur = in[i];
            start = i;
        }
    }
    o[2 * runs] = cur;
    o[2 * runs + 1] = n - start;
    runs++;
    return runs * 16;
}

/* rle decompression (rle.h:196-259). */
uint64_t orc_rle_unpack(const uint8_t *in, uint64_t n_words, uint64_t *out) {
    const uint64_t *w = (const uint64_t *)in;
    uint64_t o = 0;
    for (uint64_t i = 0; i + 1 < n_words; i += 2)
        for (uint64_t k = 0; k < w[i + 1]; k++) out[o++] = w[i];
    return o;
}

uint64_t orc_batch_pack(int fmt, unsigned bw, const uint64_t *in, uint64_t n, uint8_t *out) {
    uint64_t last[8] = {0};
    switch (fmt) {
    case ORC_FMT_UNCOMPR: memcpy(out, in, 8 * n); return 8 * n;
    case ORC_FMT_STATIC_VBP: return orc_vbp_pack(in, n, bw, out);
    case ORC_FMT_DYNAMIC_VBP: return orc_dvbp_pack(in, n, out);
    case ORC_FMT_DELTA_DVBP: return orc_delta_pack(in, n, out, last);
    case ORC_FMT_FOR_DVBP: return orc_for_pack(in, n, out);
    default: return 0;
    }
}

/* ------------------------------------------------------------------------- */
/* column-level morph: morph.h:157-197 (compress) and :203-241 (decompress);
 * rle is column-level only (rle.h:155-188, 264-297).                        */
/* ------------------------------------------------------------------------- */
int orc_compress(int fmt, unsigned bw, const uint64_t *in, uint64_t n, uint8_t *out,
                 uint64_t out_cap, orc_meta *meta) {
    if (fmt == ORC_FMT_STATIC_VBP && (bw < 1 || bw > 64)) return -1;
    if (fmt == ORC_FMT_RLE) {
        if (out_cap < 16 * n) return -2;
        uint64_t b = orc_rle_pack(in, n, out);
        meta->count_values = n;
        meta->size_used_byte = b;
        meta->size_compr_byte = b;
        return 0;
    }
    if (fmt == ORC_FMT_UNCOMPR) {
        if (out_cap < 8 * n) return -2;
        memcpy(out, in, 8 * n);
        meta->count_values = n;
        meta->size_used_byte = 8 * n;
        meta->size_compr_byte = 0;
        return 0;
    }
    if (out_cap < orc_size_max_byte_any_len(fmt, bw, n)) return -2;
    uint64_t b = orc_block_size(fmt);
    uint64_t ncompr = n / b * b;
    uint64_t compr = ncompr ? orc_batch_pack(fmt, bw, in, ncompr, out) : 0;
    uint64_t used = compr;
    if (n > ncompr) {
        uint64_t r = orc_rest_offset(fmt, bw, compr);
        memcpy(out + r, in + ncompr, 8 * (n - ncompr));
        used = r + 8 * (n - ncompr);
    }
    meta->count_values = n;
    meta->size_used_byte = used;
    meta->size_compr_byte = compr;
    return 0;
}

int orc_decompress(int fmt, unsigned bw, const uint8_t *in, const orc_meta *meta, uint64_t *out) {
    uint64_t n = meta->count_values;
    if (fmt == ORC_FMT_UNCOMPR) {
        memcpy(out, in, 8 * n);
        return 0;
    }
    if (fmt == ORC_FMT_RLE) {
        uint64_t got = orc_rle_unpack(in, meta->size_used_byte / 8, out);
        return got == n ? 0 : -3;
    }
    uint64_t nrest = orc_count_rest(fmt, bw, meta);
    uint64_t ncompr = n - nrest;
    if (ncompr) {
        switch (fmt) {
        case ORC_FMT_STATIC_VBP: orc_vbp_unpack(in, ncompr, bw, out); break;
        case ORC_FMT_DYNAMIC_VBP: orc_dvbp_unpack(in, ncompr, out); break;
        case ORC_FMT_DELTA_DVBP: orc_delta_unpack(in, ncompr, out); break;
        case ORC_FMT_FOR_DVBP: orc_for_unpack(in, ncompr, out); break;
        default: return -1;
        }
    }
    if (nrest)
        memcpy(out + ncompr, in + orc_rest_offset(fmt, bw, meta->size_compr_byte), 8 * nrest);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Write-iterator output model (write_iterator.h:67-306, uncompr.h:126-237,
 * delta.h:375-490).  The first n_vec values are written through the
 * format's write iterator: every full buffer of 2048 values is a separate
 * morph_batch, done() compresses the largest block multiple of what is left
 * and stores the remainder uncompressed at create_data_uncompr_start.  The
 * next n_scalar values come from the operator's scalar remainder loop and
 * are appended uncompressed behind that (select_compr.h:211-250).          */
/* ------------------------------------------------------------------------- */
int orc_wi_write(int fmt, unsigned bw, const uint64_t *vals, uint64_t n_vec, uint64_t n_scalar,
                 uint8_t *out, uint64_t out_cap, orc_meta *meta) {
    uint64_t n = n_vec + n_scalar;
    if (fmt == ORC_FMT_UNCOMPR) {
        if (out_cap < 8 * n) return -2;
        memcpy(out, vals, 8 * n);
        meta->count_values = n;
        meta->size_used_byte = 8 * n;
        meta->size_compr_byte = 0;
        return 0;
    }
    if (fmt == ORC_FMT_RLE) return -1; /* rle_f has no write iterator */
    if (out_cap < orc_size_max_byte_any_len(fmt, bw, n)) return -2;
    uint64_t b = orc_block_size(fmt), o = 0, i = 0, last[8] = {0};
    while (n_vec - i >= WI_BUFFER) {
        if (fmt == ORC_FMT_DELTA_DVBP) o += orc_delta_pack(vals + i, WI_BUFFER, out + o, last);
        else o += orc_batch_pack(fmt, bw, vals + i, WI_BUFFER, out + o);
        i += WI_BUFFER;
    }
    uint64_t rem = n_vec - i, rc = rem / b * b;
    if (rc) {
        if (fmt == ORC_FMT_DELTA_DVBP) o += orc_delta_pack(vals + i, rc, out + o, last);
        else o += orc_batch_pack(fmt, bw, vals + i, rc, out + o);
        i += rc;
    }
    uint64_t compr = o, used = o, nrest = n - i;
    if (nrest) {
        uint64_t r = orc_rest_offset(fmt, bw, compr);
        memcpy(out + r, vals + i, 8 * nrest);
        used = r + 8 * nrest;
    }
    meta->count_values = n;
    meta->size_used_byte = used;
    meta->size_compr_byte = compr;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* operators on decoded values                                               */
/* ------------------------------------------------------------------------- */

/* select (select_compr.h:59-260).  Values at index < scalar_from are compared
 * with the AVX-512 TVL primitives (signed 64-bit, compare_avx512.h:35-111);
 * the scalar remainder uses the scalar primitives (unsigned,
 * compare_scalar.h:17-77).  The two agree for all values below 2^63. */
static int cmp_signed(int cmp, uint64_t a, uint64_t b) {
    int64_t x = (int64_t)a, y = (int64_t)b;
    switch (cmp) {
    case ORC_CMP_EQ: return x == y;
    case ORC_CMP_LT: return x < y;
    case ORC_CMP_LE: return x <= y;
    case ORC_CMP_GT: return x > y;
    default: return x >= y;
    }
}
static int cmp_unsigned(int cmp, uint64_t a, uint64_t b) {
    switch (cmp) {
    case ORC_CMP_EQ: return a == b;
    case ORC_CMP_LT: return a < b;
    case ORC_CMP_LE: return a <= b;
    case ORC_CMP_GT: return a > b;
    default: return a >= b;
    }
}

uint64_t orc_select(int cmp, uint64_t val, const uint64_t *data, uint64_t n, uint64_t scalar_from,
                    uint64_t *out_pos) {
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; i++) {
        int hit = i < scalar_from ? cmp_signed(cmp, data[i], val) : cmp_unsigned(cmp, data[i], val);
        if (hit) out_pos[k++] = i;
    }
    return k;
}

/* agg_sum (agg_sum_compr.h:47-153, scalar/agg_sum_uncompr.h:43-62): sum mod 2^64 */
uint64_t orc_agg_sum(const uint64_t *data, uint64_t n) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) s += data[i];
    return s;
}

/* project (scalar/project_uncompr.h:39-70) */
void orc_project(const uint64_t *data, const uint64_t *pos, uint64_t n, uint64_t *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = data[pos[i]];
}

/* select -> project -> agg_sum, the select_sum_query pipeline
 * (src/examples/select_sum_query.cpp:77-97). */
uint64_t orc_select_project_sum(int cmp, uint64_t c, const uint64_t *x, const uint64_t *y, uint64_t n,
                                uint64_t scalar_from, uint64_t *count) {
    uint64_t s = 0, k = 0;
    for (uint64_t i = 0; i < n; i++) {
        int hit = i < scalar_from ? cmp_signed(cmp, x[i], c) : cmp_unsigned(cmp, x[i], c);
        if (hit) {
            s += y[i];
            k++;
        }
    }
    if (count) *count = k;
    return s;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

static int contains_sorted(const uint64_t *s, uint64_t n, uint64_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (s[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && s[lo] == v;
}

/* semi_join (join_semi_equi_compr.h:106-300): ascending positions of the
 * probe side R whose value occurs in the build side L. */
uint64_t orc_semi_join(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr, uint64_t *out_pos) {
    uint64_t *s = (uint64_t *)malloc(8 * (nl ? nl : 1));
    memcpy(s, l, 8 * nl);
    qsort(s, nl, 8, cmp_u64);
    uint64_t k = 0;
    for (uint64_t i = 0; i < nr; i++)
        if (contains_sorted(s, nl, r[i])) out_pos[k++] = i;
    free(s);
    return k;
}

/* natural equi-join (join_natural_equi_compr.h:116-300 with the hash_map of
 * join.h:158-187): the build side L maps each key to the position of its
 * first occurrence (an insert of a key already present keeps the old value,
 * linear_probing.h:315-366); every probe row of R whose value is a key emits
 * (L position, R position), in R order.  Returns the number of pairs. */
typedef struct {
    uint64_t key, pos;
} orc_kp;

static int cmp_kp(const void *a, const void *b) {
    const orc_kp *x = (const orc_kp *)a, *y = (const orc_kp *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

uint64_t orc_natural_join(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr, uint64_t *out_l,
                          uint64_t *out_r) {
    orc_kp *m = (orc_kp *)malloc(sizeof(orc_kp) * (nl ? nl : 1));
    for (uint64_t i = 0; i < nl; i++) {
        m[i].key = l[i];
        m[i].pos = i;
    }
    qsort(m, nl, sizeof(orc_kp), cmp_kp);
    uint64_t u = 0;  /* keep the first position of every key */
    for (uint64_t i = 0; i < nl; i++)
        if (i == 0 || m[i].key != m[u - 1].key) m[u++] = m[i];
    uint64_t k = 0;
    for (uint64_t j = 0; j < nr; j++) {
        uint64_t lo = 0, hi = u;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (m[mid].key < r[j]) lo = mid + 1;
            else hi = mid;
        }
        if (lo < u && m[lo].key == r[j]) {
            out_l[k] = m[lo].pos;
            out_r[k] = j;
            k++;
        }
    }
    free(m);
    return k;
}

/* intersect_sorted (scalar/intersect_uncompr.h:41-86) */
uint64_t orc_intersect_sorted(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr, uint64_t *out) {
    uint64_t i = 0, j = 0, k = 0;
    while (i < nl && j < nr) {
        if (l[i] < r[j]) i++;
        else if (r[j] < l[i]) j++;
        else {
            out[k++] = l[i];
            i++;
            j++;
        }
    }
    return k;
}

/* group (scalar/group_uncompr.h:48-153): group ids in order of first
 * occurrence, extents = position of each group's first occurrence.  With
 * gr_in != NULL the key is the pair (gr_in[i], data[i]) (binary group). */
typedef struct { uint64_t a, b, id; int used; } gslot;

static uint64_t hash2(uint64_t a, uint64_t b) {
    uint64_t z = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    return z ^ (z >> 31);
}

uint64_t orc_group(const uint64_t *gr_in, const uint64_t *data, uint64_t n, uint64_t *out_gr, uint64_t *out_ext) {
    uint64_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    gslot *t = (gslot *)calloc(cap, sizeof(gslot));
    uint64_t groups = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t a = gr_in ? gr_in[i] : 0, b = data[i];
        uint64_t h = hash2(a, b) & (cap - 1);
        while (t[h].used && !(t[h].a == a && t[h].b == b)) h = (h + 1) & (cap - 1);
        if (!t[h].used) {
            t[h].used = 1;
            t[h].a = a;
            t[h].b = b;
            t[h].id = groups;
            out_ext[groups] = i;
            groups++;
        }
        out_gr[i] = t[h].id;
    }
    free(t);
    return groups;
}

/* grouped agg_sum (scalar/agg_sum_uncompr.h:64-95) */
void orc_agg_sum_grouped(const uint64_t *gr, const uint64_t *data, uint64_t n, uint64_t n_groups, uint64_t *out) {
    for (uint64_t g = 0; g < n_groups; g++) out[g] = 0;
    for (uint64_t i = 0; i < n; i++) out[gr[i]] += data[i];
}

/* ------------------------------------------------------------------------- */
/* seeded generators: counter-based splitmix64 (the i-th output of a
 * splitmix64 stream started at `seed`), identical on host and device.       */
/* ------------------------------------------------------------------------- */
uint64_t orc_mix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void orc_gen_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *out) {
    orc_gen_uniform_bits_at(seed, bits, 0, n, out);
}

/* rows [row0, row0 + n) of the same stream: a shard of a longer column */
void orc_gen_uniform_bits_at(uint64_t seed, unsigned bits, uint64_t row0, uint64_t n, uint64_t *out) {
    for (uint64_t i = 0; i < n; i++) {
        uint64_t z = orc_mix64(seed, row0 + i);
        out[i] = bits >= 64 ? z : (bits == 0 ? 0 : z >> (64 - bits));
    }
}

/* Inverse-CDF threshold tables: table[k] = floor(2^64 * F(k)), last = 2^64-1.
 * A draw u maps to the smallest k with u < table[k]. */
static uint64_t to_threshold(long double f) {
    if (f >= 1.0L) return ~(uint64_t)0;
    long double t = f * 18446744073709551616.0L;
    if (t >= 18446744073709551615.0L) return ~(uint64_t)0;
    return (uint64_t)t;
}

void orc_cdf_table_zipf(double s, uint64_t n_vals, uint64_t *table) {
    long double total = 0, acc = 0;
    for (uint64_t k = 0; k < n_vals; k++) total += powl((long double)(k + 1), -(long double)s);
    for (uint64_t k = 0; k < n_vals; k++) {
        acc += powl((long double)(k + 1), -(long double)s);
        table[k] = to_threshold(acc / total);
    }
    table[n_vals - 1] = ~(uint64_t)0;
}

/* P(G = k) = p (1-p)^k, k >= 0; returns the table length used (<= max_len). */
uint64_t orc_cdf_table_geom(double p, uint64_t max_len, uint64_t *table) {
    long double q = 1.0L - (long double)p, qk = q;
    uint64_t k;
    for (k = 0; k < max_len; k++) {
        table[k] = to_threshold(1.0L - qk);
        qk *= q;
        if (table[k] == ~(uint64_t)0) break;
    }
    if (k == max_len) k = max_len - 1;
    table[k] = ~(uint64_t)0;
    return k + 1;
}

static uint64_t table_lookup(const uint64_t *table, uint64_t n_tab, uint64_t u) {
    uint64_t lo = 0, hi = n_tab - 1;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (u < table[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

void orc_gen_from_table(uint64_t seed, const uint64_t *table, uint64_t n_tab, uint64_t n, uint64_t *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = table_lookup(table, n_tab, orc_mix64(seed, i));
}

/* sorted ascending, gaps 1 + G with G drawn from gap_table; x_0 = gap_0. */
void orc_gen_sorted_gaps(uint64_t seed, const uint64_t *gap_table, uint64_t n_tab, uint64_t n, uint64_t *out) {
    uint64_t acc = 0;
    for (uint64_t i = 0; i < n; i++) {
        acc += 1 + table_lookup(gap_table, n_tab, orc_mix64(seed, i));
        out[i] = acc;
    }
}

/* runs: position i starts a new run with probability 2^-log2_mean_len
 * (geometric run lengths, mean 2^log2_mean_len); run r has the value
 * mix64(seed ^ C, r) >> (64 - value_bits). */
void orc_gen_runs(uint64_t seed, unsigned log2_mean_len, unsigned value_bits, uint64_t n, uint64_t *out) {
    uint64_t run = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (i > 0 && (orc_mix64(seed, i) >> (64 - log2_mean_len)) == 0) run++;
        uint64_t z = orc_mix64(seed ^ 0xD1B54A32D192ED03ull, run);
        out[i] = value_bits >= 64 ? z : z >> (64 - value_bits);
    }
}
