/*
 * ms_oracle.h -- CPU oracle for the compression-aware query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, scalar restatement of the
 * MorphStore reference's codecs and operators, used by the tests, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * Nothing in the product path (engine_b200/) links, loads or calls it.
 *
 * Layouts restated here are the reference's AVX-512 defaults
 * (include/core/morphing/default_formats.h:35-82):
 *   static_vbp_f<vbp_l<bw,8>>          block 512 values
 *   dynamic_vbp_f<512,64,8>            block 512, page 64 blocks, 64-B header
 *   delta_f<1024,8,dynamic_vbp_f<..>>  block 1024
 *   for_f<1024,8,dynamic_vbp_f<..>>    block 1024, page 8 blocks, 64-B header
 *   rle_f                              (value, run length) pairs
 */
#ifndef MS_ORACLE_H
#define MS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_FMT_UNCOMPR = 0,
    ORC_FMT_STATIC_VBP = 1,
    ORC_FMT_DYNAMIC_VBP = 2,
    ORC_FMT_DELTA_DVBP = 3,
    ORC_FMT_FOR_DVBP = 4,
    ORC_FMT_RLE = 5
};

enum { ORC_CMP_EQ = 0, ORC_CMP_LT = 1, ORC_CMP_LE = 2, ORC_CMP_GT = 3, ORC_CMP_GE = 4 };

/* Column metadata, as column<F>::m_MetaData (include/core/storage/column.h:133-144). */
typedef struct orc_meta {
    uint64_t count_values;
    uint64_t size_used_byte;
    uint64_t size_compr_byte;
} orc_meta;

/* ---- generic helpers ---------------------------------------------------- */
unsigned orc_effective_bitwidth(uint64_t v);
uint64_t orc_block_size(int fmt);                 /* m_BlockSize; 0 for rle */
uint64_t orc_size_max_byte(int fmt, unsigned bw, uint64_t n);   /* F::get_size_max_byte */
uint64_t orc_size_max_byte_any_len(int fmt, unsigned bw, uint64_t n);
uint64_t orc_rest_offset(int fmt, unsigned bw, uint64_t compr_bytes);
uint64_t orc_count_rest(int fmt, unsigned bw, const orc_meta *m);

/* ---- batch-level codecs (morph_batch analogues) ------------------------- */
uint64_t orc_vbp_pack(const uint64_t *in, uint64_t n, unsigned bw, uint8_t *out);
uint64_t orc_vbp_unpack(const uint8_t *in, uint64_t n, unsigned bw, uint64_t *out);
uint64_t orc_dvbp_pack(const uint64_t *in, uint64_t n, uint8_t *out);
uint64_t orc_dvbp_unpack(const uint8_t *in, uint64_t n, uint64_t *out);
uint64_t orc_delta_pack(const uint64_t *in, uint64_t n, uint8_t *out, uint64_t last[8]);
uint64_t orc_delta_unpack(const uint8_t *in, uint64_t n, uint64_t *out);
uint64_t orc_for_pack(const uint64_t *in, uint64_t n, uint8_t *out);
uint64_t orc_for_unpack(const uint8_t *in, uint64_t n, uint64_t *out);
uint64_t orc_rle_pack(const uint64_t *in, uint64_t n, uint8_t *out);
uint64_t orc_rle_unpack(const uint8_t *in, uint64_t n_words, uint64_t *out);
uint64_t orc_batch_pack(int fmt, unsigned bw, const uint64_t *in, uint64_t n, uint8_t *out);

/* ---- column-level morph ------------------------------------------------- */
int orc_compress(int fmt, unsigned bw, const uint64_t *in, uint64_t n,
                 uint8_t *out, uint64_t out_cap, orc_meta *meta);
int orc_decompress(int fmt, unsigned bw, const uint8_t *in, const orc_meta *meta,
                   uint64_t *out);

/* ---- write-iterator output model ---------------------------------------- */
int orc_wi_write(int fmt, unsigned bw, const uint64_t *vals, uint64_t n_vec,
                 uint64_t n_scalar, uint8_t *out, uint64_t out_cap, orc_meta *meta);

/* ---- operators on decoded values ---------------------------------------- */
uint64_t orc_select(int cmp, uint64_t val, const uint64_t *data, uint64_t n,
                    uint64_t scalar_from, uint64_t *out_pos);
uint64_t orc_agg_sum(const uint64_t *data, uint64_t n);
void orc_project(const uint64_t *data, const uint64_t *pos, uint64_t n, uint64_t *out);
uint64_t orc_select_project_sum(int cmp, uint64_t c, const uint64_t *x, const uint64_t *y,
                                uint64_t n, uint64_t scalar_from, uint64_t *count);
uint64_t orc_semi_join(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr,
                       uint64_t *out_pos);
uint64_t orc_natural_join(const uint64_t *l, uint64_t nl, const uint64_t *r, uint64_t nr, uint64_t *out_l,
                          uint64_t *out_r);
uint64_t orc_intersect_sorted(const uint64_t *l, uint64_t nl, const uint64_t *r,
                              uint64_t nr, uint64_t *out);
uint64_t orc_group(const uint64_t *gr_in, const uint64_t *data, uint64_t n,
                   uint64_t *out_gr, uint64_t *out_ext);
void orc_agg_sum_grouped(const uint64_t *gr, const uint64_t *data, uint64_t n,
                         uint64_t n_groups, uint64_t *out);

/* ---- seeded generators (counter-based splitmix64) ----------------------- */
uint64_t orc_mix64(uint64_t seed, uint64_t i);
void orc_gen_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *out);
void orc_gen_uniform_bits_at(uint64_t seed, unsigned bits, uint64_t row0, uint64_t n, uint64_t *out);
void orc_cdf_table_zipf(double s, uint64_t n_vals, uint64_t *table);
uint64_t orc_cdf_table_geom(double p, uint64_t max_len, uint64_t *table);
void orc_gen_from_table(uint64_t seed, const uint64_t *table, uint64_t n_tab,
                        uint64_t n, uint64_t *out);
void orc_gen_sorted_gaps(uint64_t seed, const uint64_t *gap_table, uint64_t n_tab,
                         uint64_t n, uint64_t *out);
void orc_gen_runs(uint64_t seed, unsigned log2_mean_len, unsigned value_bits,
                  uint64_t n, uint64_t *out);

#ifdef __cplusplus
}
#endif
#endif
