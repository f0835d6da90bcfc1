// internal.h -- host-side glue shared by the .cu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "colview.cuh"
#include "ms_common.cuh"

struct ms_arena {
    char *base;
    uint64_t cap;
    uint64_t used;
    int device;
    unsigned *d_err;  // device error word shared by the arena's launches
};

namespace ms {

// Bump allocation with 256-B alignment (stream-ordered reuse is the
// caller's business: reset only after the stream has drained).
void *arena_take(ms_arena *a, uint64_t bytes);

template <class T> T *arena_take_t(ms_arena *a, uint64_t count) {
    return static_cast<T *>(arena_take(a, count * sizeof(T)));
}

int sm_count();
unsigned persistent_grid(unsigned threads_per_cta, unsigned ctas_per_sm_hint);

// Validate a descriptor (format / bw / sizes).
int check_col(const ms_col *c, bool need_index_for_dvbp);

// Builds a kernel view of `c`: block index (built into the arena when the
// descriptor has none), delta carries.  The view stays valid while the arena
// allocations do.
int prepare_view(const ms_col *c, ms_arena *a, cudaStream_t st, ColView *v);

// Device-side index walk for dynamic_vbp-family columns.
int build_index_device(const ms_col *c, uint64_t *index, uint64_t *aux, unsigned *d_err, cudaStream_t st);

// Write `n` values (device) into format `fmt` with the write-iterator
// chunking: the first n_vec values in 2048-value morph batches, done() and
// the n_scalar appended rows (write_iterator.h:67-306).  `out` gets arena
// storage.  `d_count` (optional) is a device pointer holding n_vec; when set
// it overrides n_vec (the count is then only known on the device).
int write_values(const uint64_t *d_vals, uint64_t n_vec, uint64_t n_scalar, int fmt, unsigned bw, ms_col *out,
                 ms_arena *a, cudaStream_t st);

// Compress a device uncompr array of n values into fmt (column-level morph,
// morph.h:157-197).  Fills out (sync).
int compress_values(const uint64_t *d_in, uint64_t n, int fmt, unsigned bw, ms_col *out, ms_arena *a,
                    cudaStream_t st);

// Decompress into a device array of count_values values (async).
int decompress_to(const ms_col *in, uint64_t *d_out, ms_arena *a, cudaStream_t st);

int read_err(ms_arena *a, cudaStream_t st);

// Current launch parameters of the fused kernels (ms_gpu_set_tuning).
ms_tuning tuning();

// Staged (TMA) fused select/sum: see sps_tma.cu.
int sps_tma(const ColView &x, const ColView &y, bool has_y, int cmp, uint64_t val, unsigned warps, unsigned stages,
            unsigned stage_bytes, unsigned ctas_per_sm, unsigned vpt, uint64_t *d_sum, uint64_t *d_cnt,
            unsigned *d_err, cudaStream_t st);

}  // namespace ms
