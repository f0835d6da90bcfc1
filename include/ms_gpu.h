/*
 * ms_gpu.h -- C ABI of the B200 compression-aware query path.
 *
 * Plain pointers and sizes only.  Every entry point is stream-ordered on the
 * `stream` argument (a cudaStream_t passed as void*, NULL = legacy default
 * stream) and returns an ms_status.  No exceptions cross this boundary; the
 * C++ drop-in layer (engine_b200/include/morphstore_b200/) and the Python
 * layer (engine_b200/__init__.py) turn a non-OK status into an exception, as
 * the reference's host code signals errors with std::runtime_error.
 *
 * Columns live in device memory (HBM) and are described by ms_col, the
 * device-resident counterpart of the reference's column<F>
 * (include/core/storage/column.h:45-287).  Byte layouts are the reference's
 * AVX-512 defaults (include/core/morphing/default_formats.h:35-82) and are
 * bit-identical to what the reference writes:
 *   MS_FMT_UNCOMPR      uncompr_f                                  (format.h:90-96)
 *   MS_FMT_STATIC_VBP   static_vbp_f<vbp_l<bw,8>>, bw in 1..64     (static_vbp.h:61-68)
 *   MS_FMT_DYNAMIC_VBP  dynamic_vbp_f<512,64,8>                    (dynamic_vbp.h:84-159)
 *   MS_FMT_DELTA_DVBP   delta_f<1024,8,dynamic_vbp_f<512,64,8>>    (delta.h:79-157)
 *   MS_FMT_FOR_DVBP     for_f<1024,8,dynamic_vbp_f<512,64,8>>      (for.h:85-164)
 *   MS_FMT_RLE          rle_f                                      (rle.h:42-49)
 * A compressed column is its compressed main part followed, at
 * ms_rest_offset(), by an uncompressed rest (column.h:182-214).
 */
#ifndef MS_GPU_H
#define MS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MS_ABI_VERSION 1

typedef enum ms_status {
    MS_OK = 0,
    MS_ERR_INVALID = 1,      /* bad argument (null pointer, unknown format, bw) */
    MS_ERR_UNSUPPORTED = 2,  /* format combination the reference rejects too   */
    MS_ERR_CUDA = 3,         /* a CUDA runtime call failed                      */
    MS_ERR_NOMEM = 4,        /* arena or output capacity exhausted              */
    MS_ERR_CORRUPT = 5,      /* a kernel found an invalid header / bit width    */
    MS_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up              */
    MS_ERR_IO = 7            /* a column file could not be read or written      */
} ms_status;

enum {
    MS_FMT_UNCOMPR = 0,
    MS_FMT_STATIC_VBP = 1,
    MS_FMT_DYNAMIC_VBP = 2,
    MS_FMT_DELTA_DVBP = 3,
    MS_FMT_FOR_DVBP = 4,
    MS_FMT_RLE = 5
};

/* Comparison of select (vectorlib::equal/less/lessequal/greater/greaterequal,
 * include/vector/primitives/compare.h:22-76).  Values before the operator's
 * scalar remainder compare as signed 64-bit integers and the remainder as
 * unsigned, as in the reference's AVX-512 build (compare_avx512.h:35-111,
 * compare_scalar.h:17-77); both agree for values below 2^63. */
enum { MS_CMP_EQ = 0, MS_CMP_LT = 1, MS_CMP_LE = 2, MS_CMP_GT = 3, MS_CMP_GE = 4 };
/* OR-ed into ms_gpu_select's `cmp`: compare every row as unsigned, as the
 * scalar processing style's select_t<std::less, scalar<v64<uint64_t>>, ...>
 * does (scalar/select_uncompr.h:39-77, compare_scalar.h:37). */
enum { MS_CMP_UNSIGNED = 16 };

/* Device-resident column descriptor (column<F> metadata, column.h:133-144).
 * `index` is an optional device array built by ms_gpu_build_index (or by the
 * compressing morph): one uint64 per 512-value block of the compressed part,
 * (byte offset of the packed block) | (bit width << 56); for MS_FMT_FOR_DVBP
 * `index_aux` holds one reference value per 1024-value block. */
typedef struct ms_col {
    uint32_t format;
    uint32_t bw;              /* static_vbp bit width, 0 otherwise */
    uint64_t count_values;    /* m_CountLogicalValues */
    uint64_t size_used_byte;  /* m_SizeUsedByte */
    uint64_t size_compr_byte; /* m_SizeComprByte */
    uint64_t size_alloc_byte; /* capacity of `data` */
    void *data;               /* device pointer, 64-B aligned at least */
    uint64_t *index;          /* optional, device; see above */
    uint64_t *index_aux;      /* optional, device */
    uint64_t n_index;         /* entries in `index` */
} ms_col;

/* Device memory arena: the device-resident replacement of the reference's
 * query_memory_manager (include/core/memory/management/query_mm.h:83-238).
 * One cudaMalloc at creation; ms_gpu_arena_alloc bumps; reset frees all. */
typedef struct ms_arena ms_arena;

/* ---- library / arena ------------------------------------------------------ */
int ms_gpu_abi_version(void);
const char *ms_gpu_status_string(int status);
int ms_gpu_device_info(int *sm_count, int *cc_major, int *cc_minor);
int ms_gpu_arena_create(uint64_t capacity_byte, ms_arena **out);
int ms_gpu_arena_alloc(ms_arena *a, uint64_t size_byte, void **out);
int ms_gpu_arena_reset(ms_arena *a);
int ms_gpu_arena_used(const ms_arena *a, uint64_t *used_byte);
int ms_gpu_arena_destroy(ms_arena *a);
/* Synchronise `stream` and report (then clear) errors that asynchronous
 * kernels recorded in the arena's device error word. */
int ms_gpu_arena_check(ms_arena *a, void *stream);

/* Copies between host and device memory for callers that do not include the
 * CUDA headers (kind: 0 host->device, 1 device->host, 2 device->device);
 * synchronous with respect to `stream` when `sync` is non-zero. */
int ms_gpu_memcpy(void *dst, const void *src, uint64_t bytes, int kind, int sync, void *stream);
int ms_gpu_stream_sync(void *stream);

/* Launch parameters of the fused kernels, chosen per format class by the
 * autotuner (engine_b200/autotune.py) or set by hand.  staged = 1 selects the
 * TMA-staged pipeline (shared-memory ring of `stages` x `stage_bytes` per CTA,
 * `warps` consumer warps, `ctas_per_sm` CTAs per SM); 0 the direct-load
 * kernel (one warp per 512-row block, loads straight from HBM). */
typedef struct ms_tuning {
    int staged;
    unsigned warps;
    unsigned stages;
    unsigned stage_bytes;
    unsigned ctas_per_sm;
    unsigned values_per_thread; /* 16: one warp per 512-row block; 32: two blocks per warp */
} ms_tuning;
int ms_gpu_set_tuning(const ms_tuning *t);
int ms_gpu_get_tuning(ms_tuning *t);

/* ---- layout arithmetic (host only) --------------------------------------- */
/* get_size_max_byte_any_len<F>(n)  (include/core/morphing/format.h:114-153) */
uint64_t ms_size_max_byte_any_len(int format, unsigned bw, uint64_t count_values);
/* column<F>::create_data_uncompr_start as an offset (column.h:182-196) */
uint64_t ms_rest_offset(int format, unsigned bw, uint64_t size_compr_byte);
/* Host-side page walk that fills a host copy of ms_col.index from a host copy
 * of the compressed bytes (no counterpart in the reference; it replaces the
 * sequential header walk of dynamic_vbp.h:283-307 / for.h:297-360).
 * `index` needs count_compr/512 entries, `aux` count_compr/1024 (FOR). */
int ms_host_build_index(int format, const uint8_t *host_data, uint64_t size_compr_byte,
                        uint64_t count_compr, uint64_t *index, uint64_t *aux);

/* ---- morph (include/core/morphing/morph.h:81-241) -------------------------- */
/* Compress an uncompressed device column into `dst_format`, or decompress a
 * compressed one into uncompr_f.  `out` storage comes from the arena; on
 * return *out is complete (the call synchronises `stream` to read back sizes).
 * Compressing to a dynamic_vbp-family format also fills out->index. */
int ms_gpu_morph(const ms_col *src, int dst_format, unsigned dst_bw, ms_col *out,
                 ms_arena *arena, void *stream);
/* Build ms_col.index for a device column (device-side page walk). */
int ms_gpu_build_index(ms_col *col, ms_arena *arena, void *stream);
/* Copy a column (data and block index) into storage of exactly its used
 * size in `arena`: operators allocate the format's worst case
 * (get_size_max_byte_any_len, format.h:114-153), so a column that is kept
 * can be compacted after it is produced.  Asynchronous. */
int ms_gpu_col_compact(const ms_col *in, ms_col *out, ms_arena *arena, void *stream);

/* Views of block ranges, for sharding one column across ranks (no
 * counterpart in the reference, whose columns are never split).  A view of
 * rows [row_begin, row_end) shares the column's storage and block index; no
 * data is copied and nothing is allocated.  row_begin lies on a block
 * boundary of the compressed part (512 rows; 1024 for delta_f and for_f; an
 * even row for uncompr_f) and so does row_end, unless it is the column's
 * count, in which case the view keeps the uncompressed rest.  Every operator
 * treats a view as a column of its own (its scalar remainder included).
 * dynamic_vbp-family columns need their block index.  A delta_f view decodes
 * from d_carry_in, the 8 lane values of the row before row_begin (device
 * array; NULL = zeros, as at the column's start), which the view keeps by
 * reference in out->index_aux; a rank obtains it as the lane-wise sum of the
 * earlier shards' ms_gpu_delta_lane_sums.  Views are not batched
 * (ms_gpu_batch_create rejects a delta_f view with a carry-in) and are not
 * stored: store or compact the column itself. */
int ms_gpu_col_slice(const ms_col *in, uint64_t row_begin, uint64_t row_end, const uint64_t *d_carry_in,
                     ms_col *out);
/* The 8 lane-wise wrapping sums of a delta_f column's (or view's) deltas over
 * its compressed part (delta.h:229-262 decodes value i as the running sum of
 * lane i mod 8), written to device d_sums[0..8): what a shard adds to the
 * carry-in of the shards after it.  Synchronises `stream`. */
int ms_gpu_delta_lane_sums(const ms_col *in, uint64_t *d_sums, ms_arena *arena, void *stream);

/* ---- persistence (binary_io<F>, include/core/persistence/binary_io.h:40-87)
 * File layout as the reference's: [count_values u64][size_used_byte u64]
 * [size_used_byte bytes of the column buffer].  store copies the column to
 * the host and writes it (synchronous); load reads it, recovers the
 * compressed size from the format (page walk for the dynamic_vbp family,
 * which also builds the block index), checks that it agrees with the stored
 * size and uploads the column into the arena.  `format`/`bw` name the
 * column's format, as binary_io<F>'s template argument does. */
int ms_col_store(const ms_col *col, const char *path, void *stream);
int ms_col_load(const char *path, int format, unsigned bw, ms_col *out, ms_arena *arena, void *stream);

/* ---- operators (include/core/operators/interfaces/) ----------------------- */
/* agg_sum<ve,F>(col) (agg_sum.h:56-65; agg_sum_compr.h:78-153): the uint64
 * wrapping sum written to device *d_sum (asynchronous; the arena supplies
 * scratch such as delta carries; ms_gpu_arena_check reports kernel errors). */
int ms_gpu_agg_sum(const ms_col *in, uint64_t *d_sum, ms_arena *arena, void *stream);

/* my_select_wit_t<cmp,ve,out_f,in_f>::apply(in, val) (select_compr.h:100-260):
 * ascending positions where cmp(value, val) holds, written in `out_format`
 * with the reference write iterator's chunking (write_iterator.h:67-306). */
int ms_gpu_select(int cmp, uint64_t val, const ms_col *in, int out_format, unsigned out_bw,
                  ms_col *out, ms_arena *arena, void *stream);

/* my_project_wit_t<ve,out_f,data_f,pos_f>::apply(data, pos)
 * (project_compr.h:75-262).  Unlike the reference, data may also be a
 * dynamic_vbp-family column (random access through ms_col.index). */
int ms_gpu_project(const ms_col *data, const ms_col *pos, int out_format, unsigned out_bw,
                   ms_col *out, ms_arena *arena, void *stream);

/* The fused select -> project -> agg_sum pipeline of
 * src/examples/select_sum_query.cpp:77-97: sum of y[i] over rows with
 * cmp(x[i], c), without materialising positions.  x and y have the same
 * count.  Optional outputs (NULL to skip): d_count, and uncompressed
 * positions / projected values (device arrays of capacity >= count). */
int ms_gpu_select_project_sum(const ms_col *x, int cmp, uint64_t c, const ms_col *y,
                              uint64_t *d_sum, uint64_t *d_count, uint64_t *d_pos,
                              uint64_t *d_vals, ms_arena *arena, void *stream);

/* Launch-only form of the fused pipeline for graph capture and timing: no
 * scratch, no synchronisation; x and y must be uncompr / static_vbp or carry
 * a block index; kernel errors are OR-ed into device *d_err. */
int ms_gpu_select_project_sum_async(const ms_col *x, int cmp, uint64_t c, const ms_col *y,
                                    uint64_t *d_sum, uint64_t *d_count, unsigned *d_err, void *stream);

/* semi_join<ve,out_f,L_f,R_f>(L, R) (join.h:193-218,
 * join_semi_equi_compr.h:106-300): ascending positions of R whose value
 * occurs in L. */
int ms_gpu_semi_join(const ms_col *l, const ms_col *r, int out_format, unsigned out_bw,
                     ms_col *out, ms_arena *arena, void *stream);

/* join<ve, outL_f, outR_f, L_f, R_f>(L, R) (include/core/operators/
 * interfaces/join.h:158-187, general_vectorized/join_natural_equi_compr.h:
 * 116-300): the natural equi-join of build side L and probe side R; out_l
 * receives, for every row of R (in order) whose value occurs in L, the
 * position of that value's first occurrence in L, out_r the row of R.  Both
 * outputs in their formats (write-iterator model). */
int ms_gpu_natural_join(const ms_col *l, const ms_col *r, int out_l_format, unsigned out_l_bw, int out_r_format,
                        unsigned out_r_bw, ms_col *out_l, ms_col *out_r, ms_arena *arena, void *stream);

/* intersect_sorted / my_intersect_wit_t (intersect.h:52-63,
 * intersect_compr.h:190-347): sorted intersection of two position lists. */
int ms_gpu_intersect_sorted(const ms_col *l, const ms_col *r, int out_format, unsigned out_bw,
                            ms_col *out, ms_arena *arena, void *stream);

/* group_vec<ve,gr_f,ext_f,in_f>(in) (group_compr.h:281-300) and the binary
 * group (group.h:97-112, gr_in != NULL): group ids in order of first
 * occurrence and the first position of every group. */
int ms_gpu_group(const ms_col *gr_in, const ms_col *in, int gr_format, ms_col *out_gr,
                 int ext_format, ms_col *out_ext, ms_arena *arena, void *stream);

/* grouped agg_sum<ve>(gr, data, n_groups) (agg_sum.h:95-106,
 * scalar/agg_sum_uncompr.h:64-95): uncompressed sums per group. */
int ms_gpu_agg_sum_grouped(const ms_col *gr, const ms_col *data, uint64_t n_groups,
                           ms_col *out, ms_arena *arena, void *stream);

/* Allocation-free select (no counterpart in the reference).  For callers that
 * cannot allocate device memory -- the device budget was reserved up front by
 * the host application, memory belongs to another allocator (a buffer pool, a
 * plugin host), or cudaMalloc/cudaFree must be avoided because they
 * synchronise the device.  The caller passes the input column and the output
 * buffers: d_out_pos (capacity out_capacity >= count_values; uncompressed
 * ascending positions) and d_out_count (the hit count, device memory);
 * d_err (required, device) is cleared and then receives kernel error bits
 * (1 = corrupt header or bit width), which the caller reads after the stream
 * has run; the call itself only reports argument errors.  Nothing is allocated:
 * scratch lives in a 2 MiB file-scope device array that every GPU loading the
 * library keeps until exit, so inputs are limited to
 * ms_gpu_select_noalloc_max_rows() = 2^26 rows; longer inputs, delta_f/rle_f
 * inputs and dynamic_vbp/for_f inputs without a block index are rejected.
 * The first call on a device looks up the array's device address, so make it
 * before any stream capture; the address is kept for the life of the
 * process, so do not call it on a device after cudaDeviceReset.  All calls
 * share the array and it keeps the last call's contents: calls that overlap
 * on the GPU race.  Asynchronous. */
int ms_gpu_select_noalloc(int cmp, uint64_t val, const ms_col *in, uint64_t *d_out_pos,
                          uint64_t out_capacity, uint64_t *d_out_count, unsigned *d_err, void *stream);
uint64_t ms_gpu_select_noalloc_max_rows(void);

/* The fused compressed multi-operator query: select(filter cmp c) ->
 * semi_join(l, fk) -> intersect -> project(gkey, measure) -> group ->
 * grouped agg_sum, in one pass over the fact table (no counterpart as one
 * call in the reference; it equals the operator pipeline of
 * select_compr.h, join_semi_equi_compr.h, intersect_compr.h, project_compr.h,
 * group_compr.h and scalar/agg_sum_uncompr.h bit for bit).  Outputs, in group
 * id order (first occurrence): keys, extents (first position within the
 * intersected position list, as group_vec returns them) and sums. */
int ms_gpu_query3(const ms_col *filter, int cmp, uint64_t c, const ms_col *fk, const ms_col *l,
                  const ms_col *gkey, const ms_col *measure, uint64_t cap, uint64_t *h_keys,
                  uint64_t *h_ext, uint64_t *h_sums, uint64_t *n_groups, uint64_t *n_rows_p,
                  ms_arena *arena, void *stream);
/* Launch configuration of ms_gpu_query3's staged kernel (no counterpart in
 * the reference): staged (0 = direct kernel only, 1 = staged with the
 * build side's bitmap in shared memory when it fits beside the ring, else in
 * global memory, 2 = staged with the bitmap in global memory, 3 = staged
 * with the bitmap split over a 2-CTA cluster -- half per CTA, read through
 * distributed shared memory -- with the ring's stages shrunk to make room),
 * warps (consumer warps 8, 16 or 24), stages, stage_bytes; other fields
 * ignored.  Rejects a ring that does not fit shared memory with the 48 KiB
 * group table. */
int ms_gpu_set_query_tuning(const ms_tuning *t);
int ms_gpu_get_query_tuning(ms_tuning *t);
/* Device time (CUDA events around the fact-table pass: the staged kernel and
 * the direct kernel for the rest) of the last successful ms_gpu_query3 call
 * in this process, in ms; -1 before the first.  For measurement only (no
 * counterpart in the reference). */
int ms_gpu_query3_last_pass_ms(double *ms);

/* ---- batched persistent execution (no counterpart as one call in the
 * reference: for every column i it runs the chain morph<uncompr_f> ->
 * select<cmp>(c_i) -> agg_sum of the selected values, select_compr.h:100-260
 * with project_compr.h and agg_sum_compr.h, over many columns in one
 * persistent launch off a device work queue) --------------------------------
 * ms_gpu_batch_create builds the plan (work items, per-item seek values for
 * delta_f and rle_f) in the arena; the columns and the arena must outlive it.
 * ms_gpu_batch_run launches it (memsets and one kernel, no host
 * synchronisation): d_counts[i] / d_sums[i] receive column i's hit count and
 * the sum of its selected values (mod 2^64).  ms_gpu_batch_run_graph does
 * the same through a CUDA graph captured on first use for these output
 * buffers.  Kernel errors are reported by ms_gpu_arena_check. */
typedef struct ms_batch ms_batch;
int ms_gpu_batch_create(const ms_col *cols, const uint64_t *consts, uint64_t n_cols, int cmp, ms_arena *arena,
                        ms_batch **out, void *stream);
/* warps per CTA (4, 8, 12, 16), stages and stage_bytes of each warp's ring,
 * ctas_per_sm; other fields ignored */
int ms_gpu_batch_set_config(ms_batch *b, const ms_tuning *t);
int ms_gpu_batch_get_config(const ms_batch *b, ms_tuning *t);
/* The queue is sorted by decoder kind: MS_BATCH_VBP (static_vbp and
 * dynamic_vbp blocks), MS_BATCH_FOR, MS_BATCH_DELTA, MS_BATCH_REST
 * (uncompressed rows), MS_BATCH_RLE.  A kind may get its own configuration
 * (t = NULL: back to the plan's); the run then launches consecutive kinds of
 * one configuration together, each launch on its own forked stream (joined
 * before the run ends; a graph captures the fork and join).  get also reports
 * the kind's number of work items. */
enum { MS_BATCH_VBP = 0, MS_BATCH_FOR = 1, MS_BATCH_DELTA = 2, MS_BATCH_REST = 3, MS_BATCH_RLE = 4 };
int ms_gpu_batch_set_kind_config(ms_batch *b, int kind, const ms_tuning *t);
int ms_gpu_batch_get_kind_config(const ms_batch *b, int kind, ms_tuning *t, uint64_t *n_items);
int ms_gpu_batch_run(ms_batch *b, uint64_t *d_counts, uint64_t *d_sums, void *stream);
int ms_gpu_batch_run_graph(ms_batch *b, uint64_t *d_counts, uint64_t *d_sums, void *stream);
int ms_gpu_batch_info(const ms_batch *b, uint64_t *n_items, uint64_t *plan_bytes);
void ms_gpu_batch_destroy(ms_batch *b);

/* ---- per-block format selection and the learned selector ------------------
 * Blocks of ms_gpu_sel_block_values() = 2048 values; five candidates per block
 * (0 static_vbp<max width>, 1 dynamic_vbp, 2 delta+dvbp, 3 for+dvbp, 4 rle),
 * each sized exactly as the reference's morph_batch of 2048 values writes it.
 * The exhaustive judge restates exhaustive_size_format_selector.h:36-141 over
 * these candidates; the container follows blockwise_individual_f
 * (blockwise_individual.h:89-99): a format-code byte (format_selector_commons.h:
 * 25-103; 71 = rle, which the reference's container lacks), padding to 64 B,
 * the payload.  The learned selector (no counterpart in the reference) is an
 * MLP 32 -> 64 -> 64 -> 5 over sampled block statistics predicting log2 of
 * every candidate's size; BF16 weights, FP32 accumulation. */
uint64_t ms_gpu_sel_block_values(void);
uint64_t ms_gpu_sel_stats_bytes(void);
int ms_gpu_sel_gen(uint64_t seed, uint64_t nblk, unsigned seg_blocks, const uint64_t *d_zipf_table,
                   uint64_t n_zipf, uint64_t *d_out, void *stream);
int ms_gpu_sel_analyze(const uint64_t *d_in, uint64_t nblk, void *d_stats, uint32_t *d_sizes, void *stream);
uint64_t ms_gpu_sel_compress_all_scratch_bytes(void);
int ms_gpu_sel_compress_all(const uint64_t *d_in, uint64_t nblk, void *d_stats, uint32_t *d_sizes,
                            uint8_t *d_scratch, unsigned *d_err, void *stream);
int ms_gpu_sel_features(const uint64_t *d_in, uint64_t nblk, float *d_feats, void *stream);
int ms_gpu_sel_argmin(const uint32_t *d_sizes, uint64_t nblk, uint8_t *d_choice, uint64_t *d_total, void *stream);
int ms_gpu_sel_resolve(const uint64_t *d_in, uint64_t nblk, uint8_t *d_choice, void *stream);
int ms_gpu_sel_footprint(const uint32_t *d_sizes, const uint8_t *d_choice, uint64_t nblk, uint64_t *d_total,
                         void *stream);
int ms_gpu_bwi_compress(const uint64_t *d_in, uint64_t nblk, const void *d_stats, const uint8_t *d_choice,
                        uint8_t **d_out, uint64_t **d_offsets, uint64_t *h_bytes, ms_arena *arena, void *stream);
int ms_gpu_bwi_codes(const void *d_stats, const uint8_t *d_choice, uint64_t nblk, uint8_t *d_codes,
                     uint32_t *d_payload_bytes, void *stream);
int ms_gpu_bwi_select_sum(const uint8_t *d_data, const uint64_t *d_offsets, const uint8_t *d_codes,
                          const uint32_t *d_payload_bytes, uint64_t nblk, int cmp, uint64_t val,
                          uint64_t *d_sum, uint64_t *d_cnt, unsigned *d_err, void *stream);

typedef struct ms_mlp ms_mlp;
uint64_t ms_gpu_mlp_param_count(void);
int ms_gpu_mlp_create(uint64_t seed, unsigned max_batch, ms_mlp **out);
int ms_gpu_mlp_destroy(ms_mlp *m);
int ms_gpu_mlp_train(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n, unsigned steps,
                     unsigned batch, float lr, uint64_t seed, float *d_loss_curve, void *stream);
int ms_gpu_mlp_grads(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n,
                     const uint32_t *d_idx, unsigned batch, float *d_grads, float *d_loss, void *stream);
int ms_gpu_mlp_eval_loss(ms_mlp *m, const float *d_feats, const uint32_t *d_sizes, uint64_t n,
                         const uint32_t *d_idx, unsigned batch, float *d_loss, void *stream);
int ms_gpu_mlp_choose(ms_mlp *m, const float *d_feats, uint64_t n, float margin_log2, float *d_pred,
                      uint8_t *d_choice, uint64_t *d_nfallback, void *stream);
uint64_t ms_gpu_mlp_state_bytes(void);
int ms_gpu_mlp_save(ms_mlp *m, void *h_state);
int ms_gpu_mlp_load(ms_mlp *m, const void *h_state);

/* ---- synthetic data (device-side, counter-based splitmix64) -------------- */
int ms_gpu_gen_uniform_bits(uint64_t seed, unsigned bits, uint64_t n, uint64_t *d_out, void *stream);
/* rows [row0, row0 + n) of the same column: one rank's shard of a table */
int ms_gpu_gen_uniform_bits_at(uint64_t seed, unsigned bits, uint64_t row0, uint64_t n, uint64_t *d_out,
                               void *stream);
int ms_gpu_gen_from_table(uint64_t seed, const uint64_t *d_table, uint64_t n_table, uint64_t n,
                          uint64_t *d_out, void *stream);
/* sorted ascending: prefix sums of 1 + (draw from the gap table) */
int ms_gpu_gen_sorted_gaps(uint64_t seed, const uint64_t *d_gap_table, uint64_t n_table, uint64_t n,
                           uint64_t *d_out, ms_arena *arena, void *stream);
/* runs: a new run at row i > 0 with probability 2^-log2_mean_len, run values
 * over value_bits bits */
int ms_gpu_gen_runs(uint64_t seed, unsigned log2_mean_len, unsigned value_bits, uint64_t n, uint64_t *d_out,
                    ms_arena *arena, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MS_GPU_H */
