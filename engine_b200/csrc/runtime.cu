// runtime.cu -- arena, status strings, layout arithmetic, column
// validation, block-index construction and kernel views.
#include <stdio.h>
#include <string.h>

#include <cstdio>
#include <vector>

#include "internal.h"
#include "scan.cuh"

static thread_local char g_last_error[256];

int ms_fail_cuda(cudaError_t e, const char *what) {
    snprintf(g_last_error, sizeof g_last_error, "%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MS_ERR_NOMEM : MS_ERR_CUDA;
}

int ms_fail(int status, const char *what) {
    snprintf(g_last_error, sizeof g_last_error, "%s", what);
    return status;
}

extern "C" int ms_gpu_abi_version(void) { return MS_ABI_VERSION; }

static ms_tuning g_tuning = {1, 16, 3, 65536, 1, 32};  // the tuned headline configuration

ms_tuning ms::tuning() { return g_tuning; }

extern "C" int ms_gpu_set_tuning(const ms_tuning *t) {
    if (!t) return ms_fail(MS_ERR_INVALID, "set_tuning: null");
    if (t->staged) {
        if (t->warps != 4 && t->warps != 8 && t->warps != 12 && t->warps != 16 && t->warps != 20 && t->warps != 24)
            return ms_fail(MS_ERR_INVALID, "set_tuning: warps must be 4, 8, 12, 16, 20 or 24");
        if (t->stages < 2 || t->stages > 32 || t->stage_bytes < 8320 || t->stage_bytes % 128 ||
            uint64_t(t->stages) * t->stage_bytes > 220 * 1024 || t->ctas_per_sm < 1 || t->ctas_per_sm > 4 ||
            (t->values_per_thread != 16 && t->values_per_thread != 32))
            return ms_fail(MS_ERR_INVALID, "set_tuning: stages x stage_bytes must fit shared memory");
    }
    g_tuning = *t;
    return MS_OK;
}

extern "C" int ms_gpu_get_tuning(ms_tuning *t) {
    if (!t) return ms_fail(MS_ERR_INVALID, "get_tuning: null");
    *t = g_tuning;
    return MS_OK;
}

extern "C" const char *ms_gpu_status_string(int status) {
    static const char *names[] = {"MS_OK",        "MS_ERR_INVALID", "MS_ERR_UNSUPPORTED", "MS_ERR_CUDA",
                                  "MS_ERR_NOMEM", "MS_ERR_CORRUPT", "MS_ERR_TIMEOUT",     "MS_ERR_IO"};
    if (status < 0 || status > 7) return "MS_ERR_UNKNOWN";
    return status == MS_OK ? names[0] : (g_last_error[0] ? g_last_error : names[status]);
}

extern "C" int ms_gpu_device_info(int *sm, int *major, int *minor) {
    int dev = 0;
    MS_CUDA_TRY(cudaGetDevice(&dev));
    cudaDeviceProp p;
    MS_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
    if (sm) *sm = p.multiProcessorCount;
    if (major) *major = p.major;
    if (minor) *minor = p.minor;
    return MS_OK;
}

// ---------------------------------------------------------------------------
// arena (device-resident replacement of query_mm.h:83-238)
// ---------------------------------------------------------------------------
extern "C" int ms_gpu_arena_create(uint64_t cap, ms_arena **out) {
    if (!out || cap == 0) return ms_fail(MS_ERR_INVALID, "arena_create: bad argument");
    ms_arena *a = new ms_arena();
    MS_CUDA_TRY(cudaGetDevice(&a->device));
    cudaError_t e = cudaMalloc(&a->base, cap + 256);
    if (e != cudaSuccess) {
        delete a;
        return ms_fail_cuda(e, "arena cudaMalloc");
    }
    a->cap = cap;
    a->used = 0;
    a->d_err = reinterpret_cast<unsigned *>(a->base + cap);  // tail word, outside the bump range
    MS_CUDA_TRY(cudaMemset(a->d_err, 0, 256));
    *out = a;
    return MS_OK;
}

void *ms::arena_take(ms_arena *a, uint64_t bytes) {
    const uint64_t off = align_up(a->used, 256);
    if (off + bytes > a->cap) return nullptr;
    a->used = off + bytes;
    return a->base + off;
}

extern "C" int ms_gpu_arena_alloc(ms_arena *a, uint64_t size, void **out) {
    if (!a || !out) return ms_fail(MS_ERR_INVALID, "arena_alloc: bad argument");
    void *p = ms::arena_take(a, size);
    if (!p) return ms_fail(MS_ERR_NOMEM, "arena_alloc: arena exhausted");
    *out = p;
    return MS_OK;
}

extern "C" int ms_gpu_arena_reset(ms_arena *a) {
    if (!a) return ms_fail(MS_ERR_INVALID, "arena_reset: null");
    a->used = 0;
    return MS_OK;
}

extern "C" int ms_gpu_arena_used(const ms_arena *a, uint64_t *used) {
    if (!a || !used) return ms_fail(MS_ERR_INVALID, "arena_used: null");
    *used = a->used;
    return MS_OK;
}

extern "C" int ms_gpu_arena_destroy(ms_arena *a) {
    if (!a) return MS_OK;
    cudaError_t e = cudaFree(a->base);
    delete a;
    if (e != cudaSuccess) return ms_fail_cuda(e, "arena cudaFree");
    return MS_OK;
}

extern "C" int ms_gpu_memcpy(void *dst, const void *src, uint64_t bytes, int kind, int sync, void *stream) {
    if (!bytes) return MS_OK;
    if (!dst || !src) return ms_fail(MS_ERR_INVALID, "memcpy: null pointer");
    const cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice : kind == 1 ? cudaMemcpyDeviceToHost
                                                                            : cudaMemcpyDeviceToDevice;
    if (kind < 0 || kind > 2) return ms_fail(MS_ERR_INVALID, "memcpy: unknown kind");
    MS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream));
    if (sync) MS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return MS_OK;
}

extern "C" int ms_gpu_stream_sync(void *stream) {
    MS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return MS_OK;
}

int ms::read_err(ms_arena *a, cudaStream_t st) {
    unsigned h = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&h, a->d_err, sizeof h, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    if (h) {
        MS_CUDA_TRY(cudaMemsetAsync(a->d_err, 0, sizeof h, st));
        if (h & kErrCorrupt) return ms_fail(MS_ERR_CORRUPT, "kernel found a corrupt header or bit width");
        if (h & kErrTimeout) return ms_fail(MS_ERR_TIMEOUT, "bounded device wait gave up");
        if (h & kErrCapacity) return ms_fail(MS_ERR_NOMEM, "output capacity exceeded on the device");
    }
    return MS_OK;
}

extern "C" int ms_gpu_arena_check(ms_arena *a, void *stream) {
    if (!a) return ms_fail(MS_ERR_INVALID, "arena_check: null");
    return ms::read_err(a, (cudaStream_t)stream);
}

int ms::sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

unsigned ms::persistent_grid(unsigned, unsigned ctas_per_sm) { return unsigned(sm_count()) * ctas_per_sm; }

// ---------------------------------------------------------------------------
// layout arithmetic
// ---------------------------------------------------------------------------
extern "C" uint64_t ms_size_max_byte_any_len(int fmt, unsigned bw, uint64_t n) {
    using namespace ms;
    if (fmt == MS_FMT_UNCOMPR) return 8 * n;
    if (fmt == MS_FMT_RLE) return 16 * n + 16;
    const uint64_t b = block_size(fmt);
    if (!b) return 0;
    const uint64_t cnt = (n + b - 1) / b * b + b;
    uint64_t compr;
    switch (fmt) {
    case MS_FMT_STATIC_VBP: compr = cnt * bw / 8; break;
    case MS_FMT_DYNAMIC_VBP:
    case MS_FMT_DELTA_DVBP: compr = 8 * cnt + cnt / 512 * 64; break;
    default: compr = (cnt + 8191) / 8192 * 64 + cnt / 1024 * (8 * 1024 + 128); break;
    }
    return compr + 2 * max_block_bytes(fmt, bw) + 64 + 8 * (n % b + b) + 64;
}

extern "C" uint64_t ms_rest_offset(int fmt, unsigned bw, uint64_t compr) { return ms::rest_offset(fmt, bw, compr); }

// Host page walk (dynamic_vbp.h:283-307, delta.h:229-262, for.h:297-360).
extern "C" int ms_host_build_index(int fmt, const uint8_t *d, uint64_t compr, uint64_t count_compr, uint64_t *index,
                                   uint64_t *aux) {
    using namespace ms;
    if (!d && compr) return ms_fail(MS_ERR_INVALID, "host_build_index: null data");
    const uint64_t nb = count_compr / kBlock;
    uint64_t cur = 0, b = 0;
    if (fmt == MS_FMT_DYNAMIC_VBP || fmt == MS_FMT_DELTA_DVBP) {
        while (b < nb) {
            if (cur + kMeta > compr) return ms_fail(MS_ERR_CORRUPT, "dvbp page header beyond the compressed part");
            const uint8_t *h = d + cur;
            uint64_t off = cur + kMeta;
            for (unsigned j = 0; j < kPageBlocks && b < nb; j++) {
                const unsigned bw = h[j];
                if (bw == kNoBlock) continue;
                if (bw < 1 || bw > 64) return ms_fail(MS_ERR_CORRUPT, "dvbp header bit width out of range");
                index[b++] = idx_pack(off, bw);
                off += 64ull * bw;
            }
            cur = off;
        }
        return MS_OK;
    }
    if (fmt == MS_FMT_FOR_DVBP) {
        while (b < nb) {
            const uint64_t *refs = reinterpret_cast<const uint64_t *>(d + cur);
            cur += 64;
            for (unsigned j = 0; j < kForPageBlocks && b < nb; j++) {
                if (refs[j] == ~uint64_t(0)) break;
                aux[b / 2] = refs[j];
                const uint8_t *h = d + cur;
                uint64_t off = cur + kMeta;
                for (unsigned k = 0; k < 2; k++) {
                    const unsigned bw = h[k];
                    if (bw < 1 || bw > 64) return ms_fail(MS_ERR_CORRUPT, "for inner header bit width out of range");
                    index[b++] = idx_pack(off, bw);
                    off += 64ull * bw;
                }
                cur = off;
            }
        }
        return MS_OK;
    }
    return ms_fail(MS_ERR_INVALID, "host_build_index: format has no block index");
}

// ---------------------------------------------------------------------------
// device-side index walk: one warp, page by page (latency bound; only used
// for columns that arrive without an index)
// ---------------------------------------------------------------------------
namespace {

__global__ void k_walk_dvbp(const uint8_t *__restrict__ d, uint64_t compr, uint64_t nb, int per_page_limit,
                            uint64_t *__restrict__ index, unsigned *err) {
    const unsigned lane = threadIdx.x;
    uint64_t cur = 0, b = 0;
    while (b < nb) {
        if (cur + 64 > compr) {
            if (lane == 0) atomicOr(err, ms::kErrCorrupt);
            return;
        }
        // lane handles header bytes 2*lane, 2*lane+1
        const unsigned b0 = d[cur + 2 * lane], b1 = d[cur + 2 * lane + 1];
        const bool bad = (b0 != ms::kNoBlock && (b0 < 1 || b0 > 64)) || (b1 != ms::kNoBlock && (b1 < 1 || b1 > 64));
        if (__any_sync(0xFFFFFFFFu, bad)) {
            if (lane == 0) atomicOr(err, ms::kErrCorrupt);
            return;
        }
        const unsigned c0 = b0 == ms::kNoBlock ? 0 : 1, c1 = b1 == ms::kNoBlock ? 0 : 1;
        const unsigned w0 = c0 ? b0 : 0, w1 = c1 ? b1 : 0;
        // inclusive scans of (count, bytes/64) across lanes
        unsigned cnt = c0 + c1, wsum = w0 + w1;
        for (int s = 1; s < 32; s <<= 1) {
            unsigned a = __shfl_up_sync(0xFFFFFFFFu, cnt, s), w = __shfl_up_sync(0xFFFFFFFFu, wsum, s);
            if (lane >= unsigned(s)) {
                cnt += a;
                wsum += w;
            }
        }
        const unsigned cex = cnt - c0 - c1, wex = wsum - w0 - w1;
        const unsigned tot_c = __shfl_sync(0xFFFFFFFFu, cnt, 31), tot_w = __shfl_sync(0xFFFFFFFFu, wsum, 31);
        const uint64_t base = cur + 64;
        if (c0 && b + cex < nb) index[b + cex] = ms::idx_pack(base + 64ull * wex, b0);
        if (c1 && b + cex + c0 < nb) index[b + cex + c0] = ms::idx_pack(base + 64ull * (wex + w0), b1);
        if (tot_c == 0 || (per_page_limit && tot_c > unsigned(per_page_limit))) {
            if (lane == 0) atomicOr(err, ms::kErrCorrupt);
            return;
        }
        b += tot_c;
        cur = base + 64ull * tot_w;
    }
}

__global__ void k_walk_for(const uint8_t *__restrict__ d, uint64_t compr, uint64_t nb, uint64_t *__restrict__ index,
                           uint64_t *__restrict__ aux, unsigned *err) {
    if (threadIdx.x != 0) return;
    uint64_t cur = 0, b = 0;
    while (b < nb) {
        if (cur + 64 > compr) {
            atomicOr(err, ms::kErrCorrupt);
            return;
        }
        const uint64_t *refs = reinterpret_cast<const uint64_t *>(d + cur);
        cur += 64;
        for (unsigned j = 0; j < ms::kForPageBlocks && b < nb; j++) {
            const uint64_t ref = refs[j];
            if (ref == ~uint64_t(0)) break;
            aux[b / 2] = ref;
            const unsigned bw0 = d[cur], bw1 = d[cur + 1];
            if (bw0 < 1 || bw0 > 64 || bw1 < 1 || bw1 > 64) {
                atomicOr(err, ms::kErrCorrupt);
                return;
            }
            index[b] = ms::idx_pack(cur + 64, bw0);
            index[b + 1] = ms::idx_pack(cur + 64 + 64ull * bw0, bw1);
            b += 2;
            cur += 64 + 64ull * (bw0 + bw1);
        }
    }
}

// delta carries: per 512-block, lane-wise sums of the decoded deltas.
__global__ void __launch_bounds__(256, 3) k_delta_block_sums(ms::ColView c, uint64_t *__restrict__ sums, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    const uint64_t nb = c.nb();
    ms::ColView raw = c;
    raw.fmt = MS_FMT_DYNAMIC_VBP;  // decode the deltas themselves
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nb;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        if (!ms::decode_block(raw, b, l, q, v, valid)) {
            if (lane == 0) atomicOr(err, ms::kErrCorrupt);
        }
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) s += v[k];
        s += __shfl_xor_sync(0xFFFFFFFFu, s, 8);
        s += __shfl_xor_sync(0xFFFFFFFFu, s, 16);
        if (q == 0) sums[b * 8 + l] = s;
    }
}

}  // namespace

// A delta_f view's carry-in (the 8 lane values before its first row) added
// to every block's lane carry.
__global__ void k_add_carry_in(uint64_t *__restrict__ carry, uint64_t nb, const uint64_t *__restrict__ carry_in) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nb * 8; i += uint64_t(gridDim.x) * blockDim.x)
        carry[i] += carry_in[i & 7];
}

int ms::build_index_device(const ms_col *c, uint64_t *index, uint64_t *aux, unsigned *d_err, cudaStream_t st) {
    const uint64_t ncompr = c->count_values - count_rest(*c);
    const uint64_t nb = ncompr / kBlock;
    if (nb == 0) return MS_OK;
    if (c->format == MS_FMT_DYNAMIC_VBP || c->format == MS_FMT_DELTA_DVBP) {
        k_walk_dvbp<<<1, 32, 0, st>>>((const uint8_t *)c->data, c->size_compr_byte, nb,
                                      c->format == MS_FMT_DELTA_DVBP ? 2 : 0, index, d_err);
    } else if (c->format == MS_FMT_FOR_DVBP) {
        k_walk_for<<<1, 32, 0, st>>>((const uint8_t *)c->data, c->size_compr_byte, nb, index, aux, d_err);
    } else {
        return ms_fail(MS_ERR_INVALID, "build_index: format has no block index");
    }
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// Copy a column into storage of exactly its used size (the producing
// operators allocate the format's worst case, get_size_max_byte_any_len),
// block index included.
extern "C" int ms_gpu_col_compact(const ms_col *in, ms_col *out, ms_arena *a, void *stream) {
    using namespace ms;
    if (!in || !out || !a) return ms_fail(MS_ERR_INVALID, "col_compact: null");
    int rc = check_col(in, false);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t bytes = in->size_used_byte;
    const bool has_index = in->index && in->n_index, has_aux = in->index_aux && in->n_index;
    // index_aux: FOR references (one per 1024 rows) or a delta_f view's 8 carry-in lanes
    const uint64_t aux_words = in->format == MS_FMT_DELTA_DVBP ? 8 : in->n_index / 2;
    uint8_t *data = arena_take_t<uint8_t>(a, bytes + 64);
    uint64_t *index = has_index ? arena_take_t<uint64_t>(a, in->n_index + 1) : nullptr;
    uint64_t *aux = has_aux ? arena_take_t<uint64_t>(a, aux_words + 1) : nullptr;
    if (!data || (has_index && !index) || (has_aux && !aux)) return ms_fail(MS_ERR_NOMEM, "arena exhausted (col_compact)");
    if (bytes) MS_CUDA_TRY(cudaMemcpyAsync(data, in->data, bytes, cudaMemcpyDeviceToDevice, st));
    if (index) MS_CUDA_TRY(cudaMemcpyAsync(index, in->index, 8 * in->n_index, cudaMemcpyDeviceToDevice, st));
    if (aux && aux_words)
        MS_CUDA_TRY(cudaMemcpyAsync(aux, in->index_aux, 8 * aux_words, cudaMemcpyDeviceToDevice, st));
    ms_col c = *in;
    c.data = data;
    c.size_alloc_byte = bytes + 64;
    c.index = index;
    c.index_aux = aux;
    if (!index) c.n_index = 0;
    *out = c;
    return MS_OK;
}

// ---------------------------------------------------------------------------
// persistence: binary_io<F> (binary_io.h:40-87)
// ---------------------------------------------------------------------------
extern "C" int ms_col_store(const ms_col *c, const char *path, void *stream) {
    using namespace ms;
    if (!c || !path) return ms_fail(MS_ERR_INVALID, "col_store: null argument");
    int rc = check_col(c, false);
    if (rc) return rc;
    std::vector<uint8_t> h(c->size_used_byte);
    if (!h.empty()) {
        MS_CUDA_TRY(cudaMemcpyAsync(h.data(), c->data, h.size(), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
        MS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return ms_fail(MS_ERR_IO, "col_store: could not open the file for writing");
    const uint64_t meta[2] = {c->count_values, c->size_used_byte};
    bool ok = std::fwrite(meta, 8, 2, f) == 2 && (h.empty() || std::fwrite(h.data(), 1, h.size(), f) == h.size());
    ok = (std::fclose(f) == 0) && ok;
    return ok ? MS_OK : ms_fail(MS_ERR_IO, "col_store: could not write the column meta data and data");
}

extern "C" int ms_col_load(const char *path, int fmt, unsigned bw, ms_col *out, ms_arena *a, void *stream) {
    using namespace ms;
    if (!path || !out || !a) return ms_fail(MS_ERR_INVALID, "col_load: null argument");
    if (fmt < MS_FMT_UNCOMPR || fmt > MS_FMT_RLE || (fmt == MS_FMT_STATIC_VBP && (bw < 1 || bw > 64)))
        return ms_fail(MS_ERR_INVALID, "col_load: format");
    FILE *f = std::fopen(path, "rb");
    if (!f) return ms_fail(MS_ERR_IO, "col_load: could not open the file for reading");
    uint64_t meta[2] = {0, 0};
    if (std::fread(meta, 8, 2, f) != 2) {
        std::fclose(f);
        return ms_fail(MS_ERR_IO, "col_load: could not read the column meta data");
    }
    const uint64_t count = meta[0], used = meta[1];
    if (used > (uint64_t(1) << 40)) {
        std::fclose(f);
        return ms_fail(MS_ERR_CORRUPT, "col_load: implausible column size");
    }
    std::vector<uint8_t> h(used + 64, 0);
    const bool ok = used == 0 || std::fread(h.data(), 1, used, f) == used;
    std::fclose(f);
    if (!ok) return ms_fail(MS_ERR_IO, "col_load: could not read the column data");
    // the compressed size, recovered from the format
    uint64_t compr = 0, ncompr = 0;
    std::vector<uint64_t> idx, aux;
    if (fmt == MS_FMT_RLE) {
        compr = used;
        if (used % 16) return ms_fail(MS_ERR_CORRUPT, "col_load: rle_f size is not a multiple of 16");
    } else if (fmt == MS_FMT_STATIC_VBP) {
        ncompr = count - count % kBlock;
        compr = ncompr / 8 * bw;
    } else if (fmt != MS_FMT_UNCOMPR) {
        const uint64_t blk = fmt == MS_FMT_DYNAMIC_VBP ? kBlock : 2 * kBlock;
        ncompr = count - count % blk;
        const uint64_t nb = ncompr / kBlock;
        if (nb) {
            idx.resize(nb + 1);
            aux.resize(nb / 2 + 1);
            int rc = ms_host_build_index(fmt, h.data(), used, ncompr, idx.data(),
                                         fmt == MS_FMT_FOR_DVBP ? aux.data() : nullptr);
            if (rc) return rc;
            compr = idx_off(idx[nb - 1]) + 64ull * idx_bw(idx[nb - 1]);
        }
    }
    const uint64_t nrest = count - ncompr;
    const uint64_t expect = fmt == MS_FMT_UNCOMPR ? 8 * count
                            : fmt == MS_FMT_RLE ? used
                            : (nrest ? rest_offset(fmt, bw, compr) + 8 * nrest : compr);
    if (expect != used) return ms_fail(MS_ERR_CORRUPT, "col_load: stored size disagrees with the format");
    ms_col c{};
    c.format = uint32_t(fmt);
    c.bw = fmt == MS_FMT_STATIC_VBP ? bw : 0;
    c.count_values = count;
    c.size_used_byte = used;
    c.size_compr_byte = fmt == MS_FMT_UNCOMPR ? 0 : compr;
    c.size_alloc_byte = used + 64;
    c.data = arena_take_t<uint8_t>(a, used + 64);
    if (!c.data) return ms_fail(MS_ERR_NOMEM, "arena exhausted (col_load)");
    cudaStream_t st = (cudaStream_t)stream;
    MS_CUDA_TRY(cudaMemcpyAsync(c.data, h.data(), used + 64, cudaMemcpyHostToDevice, st));
    if (!idx.empty()) {
        const uint64_t nb = idx.size() - 1;
        uint64_t *di = arena_take_t<uint64_t>(a, nb + 1);
        uint64_t *da = fmt == MS_FMT_FOR_DVBP ? arena_take_t<uint64_t>(a, nb / 2 + 1) : nullptr;
        if (!di || (fmt == MS_FMT_FOR_DVBP && !da)) return ms_fail(MS_ERR_NOMEM, "arena exhausted (col_load index)");
        MS_CUDA_TRY(cudaMemcpyAsync(di, idx.data(), 8 * nb, cudaMemcpyHostToDevice, st));
        if (da) MS_CUDA_TRY(cudaMemcpyAsync(da, aux.data(), 8 * (nb / 2 + 1), cudaMemcpyHostToDevice, st));
        c.index = di;
        c.index_aux = da;
        c.n_index = nb;
    }
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    *out = c;
    return MS_OK;
}

extern "C" int ms_gpu_build_index(ms_col *c, ms_arena *a, void *stream) {
    using namespace ms;
    if (!c || !a) return ms_fail(MS_ERR_INVALID, "build_index: null");
    int rc = check_col(c, false);
    if (rc) return rc;
    if (c->format != MS_FMT_DYNAMIC_VBP && c->format != MS_FMT_DELTA_DVBP && c->format != MS_FMT_FOR_DVBP)
        return MS_OK;
    const uint64_t nb = (c->count_values - count_rest(*c)) / kBlock;
    uint64_t *idx = arena_take_t<uint64_t>(a, nb + 1);
    uint64_t *aux = c->format == MS_FMT_FOR_DVBP ? arena_take_t<uint64_t>(a, nb / 2 + 1) : nullptr;
    if (!idx || (c->format == MS_FMT_FOR_DVBP && !aux)) return ms_fail(MS_ERR_NOMEM, "build_index: arena exhausted");
    cudaStream_t st = (cudaStream_t)stream;
    rc = build_index_device(c, idx, aux, a->d_err, st);
    if (rc) return rc;
    rc = read_err(a, st);
    if (rc) return rc;
    c->index = idx;
    c->index_aux = aux;
    c->n_index = nb;
    return MS_OK;
}

int ms::check_col(const ms_col *c, bool) {
    if (!c) return ms_fail(MS_ERR_INVALID, "null column");
    if (c->format > MS_FMT_RLE) return ms_fail(MS_ERR_INVALID, "unknown format");
    if (c->format == MS_FMT_STATIC_VBP && (c->bw < 1 || c->bw > 64))
        return ms_fail(MS_ERR_INVALID, "static_vbp bit width must be in 1..64");
    if (c->count_values && !c->data) return ms_fail(MS_ERR_INVALID, "column without data");
    if (c->size_compr_byte > c->size_used_byte) return ms_fail(MS_ERR_INVALID, "size_compr_byte > size_used_byte");
    if (c->format == MS_FMT_UNCOMPR && c->size_used_byte != 8 * c->count_values)
        return ms_fail(MS_ERR_INVALID, "uncompr column with size_used != 8 * count");
    if (c->format != MS_FMT_UNCOMPR && c->format != MS_FMT_RLE && c->size_compr_byte < c->size_used_byte) {
        const uint64_t ro = rest_offset(c->format, c->bw, c->size_compr_byte);
        if (c->size_used_byte < ro || (c->size_used_byte - ro) % 8)
            return ms_fail(MS_ERR_CORRUPT, "rest part does not fit the column");
        const uint64_t nrest = (c->size_used_byte - ro) / 8;
        if (nrest > c->count_values) return ms_fail(MS_ERR_CORRUPT, "rest longer than the column");
        if ((c->count_values - nrest) % block_size(c->format))
            return ms_fail(MS_ERR_CORRUPT, "compressed part is not a multiple of the block size");
    } else if (c->format != MS_FMT_UNCOMPR && c->format != MS_FMT_RLE) {
        if (c->count_values % block_size(c->format))
            return ms_fail(MS_ERR_CORRUPT, "compressed part is not a multiple of the block size");
    }
    if (c->format == MS_FMT_STATIC_VBP) {
        const uint64_t nc = c->count_values - count_rest(*c);
        if (c->size_compr_byte != nc * c->bw / 8) return ms_fail(MS_ERR_CORRUPT, "static_vbp size mismatch");
    }
    if ((reinterpret_cast<uintptr_t>(c->data) & 15u) != 0)
        return ms_fail(MS_ERR_INVALID, "column data must be 16-B aligned");
    return MS_OK;
}

int ms::prepare_view(const ms_col *c, ms_arena *a, cudaStream_t st, ColView *v) {
    int rc = check_col(c, false);
    if (rc) return rc;
    if (c->format == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "rle_f has no block view");
    ColView w{};
    w.fmt = int(c->format);
    w.bw = c->bw;
    w.data = (const uint8_t *)c->data;
    w.n = c->count_values;
    if (c->format == MS_FMT_UNCOMPR) {
        w.n_compr = 0;
        w.rest = (const uint64_t *)c->data;
        w.sfrom = c->count_values - c->count_values % kStep;
        *v = w;
        return MS_OK;
    }
    const uint64_t nrest = count_rest(*c);
    w.n_compr = c->count_values - nrest;
    w.rest = (const uint64_t *)((const uint8_t *)c->data + rest_offset(c->format, c->bw, c->size_compr_byte));
    w.sfrom = c->count_values - nrest % kStep;
    const uint64_t nb = w.n_compr / kBlock;
    if (c->format != MS_FMT_STATIC_VBP && nb) {
        if (c->index && c->n_index >= nb && (c->format != MS_FMT_FOR_DVBP || c->index_aux)) {
            w.index = c->index;
            w.aux = c->index_aux;
        } else {
            uint64_t *idx = arena_take_t<uint64_t>(a, nb + 1);
            uint64_t *aux = c->format == MS_FMT_FOR_DVBP ? arena_take_t<uint64_t>(a, nb / 2 + 1) : nullptr;
            if (!idx || (c->format == MS_FMT_FOR_DVBP && !aux)) return ms_fail(MS_ERR_NOMEM, "arena exhausted (index)");
            rc = build_index_device(c, idx, aux, a->d_err, st);
            if (rc) return rc;
            w.index = idx;
            w.aux = aux;
        }
    }
    if (c->format == MS_FMT_DELTA_DVBP && nb) {
        uint64_t *sums = arena_take_t<uint64_t>(a, nb * 8);
        uint64_t *carry = arena_take_t<uint64_t>(a, nb * 8);
        uint64_t *tot = arena_take_t<uint64_t>(a, 8);
        uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nb, 8));
        if (!sums || !carry || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (delta carry)");
        k_delta_block_sums<<<persistent_grid(256, 8), 256, 0, st>>>(w, sums, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint64_t, 8>(sums, nb, carry, tot, scr, st)));
        if (c->index_aux) {  // a view's carry-in
            k_add_carry_in<<<unsigned(minu((nb * 8 + 255) / 256, uint64_t(persistent_grid(256, 4)))), 256, 0, st>>>(
                carry, nb, c->index_aux);
            MS_CUDA_TRY(cudaGetLastError());
        }
        w.carry = carry;
    }
    *v = w;
    return MS_OK;
}

// ---------------------------------------------------------------------------
// Views of block ranges (one rank's shard of a column) and the delta_f
// lane sums a shard hands to the next one
// ---------------------------------------------------------------------------
extern "C" int ms_gpu_col_slice(const ms_col *in, uint64_t row_begin, uint64_t row_end, const uint64_t *d_carry_in,
                                ms_col *out) {
    using namespace ms;
    if (!in || !out) return ms_fail(MS_ERR_INVALID, "col_slice: null argument");
    int rc = check_col(in, false);
    if (rc) return rc;
    const int fmt = int(in->format);
    const uint64_t n = in->count_values;
    if (row_begin > row_end || row_end > n) return ms_fail(MS_ERR_INVALID, "col_slice: rows outside the column");
    if (fmt == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "col_slice: rle_f has no block structure");
    if (d_carry_in && fmt != MS_FMT_DELTA_DVBP) return ms_fail(MS_ERR_INVALID, "col_slice: a carry-in is for delta_f");
    if (fmt == MS_FMT_DELTA_DVBP && in->index_aux)
        return ms_fail(MS_ERR_UNSUPPORTED, "col_slice: a delta_f view with a carry-in cannot be sliced again");
    ms_col v = *in;
    v.count_values = row_end - row_begin;
    if (fmt == MS_FMT_UNCOMPR) {
        if (row_begin % 2) return ms_fail(MS_ERR_INVALID, "col_slice: uncompr_f views start at an even row");
        v.data = static_cast<uint8_t *>(in->data) + 8 * row_begin;
        v.size_used_byte = v.size_alloc_byte = 8 * v.count_values;
        v.size_compr_byte = 0;
        *out = v;
        return MS_OK;
    }
    const uint64_t nrest = count_rest(*in), ncompr = n - nrest, unit = block_size(fmt);
    const bool last = row_end == n;
    if (row_begin % unit || row_begin > ncompr)
        return ms_fail(MS_ERR_INVALID, "col_slice: a view starts on a block boundary of the compressed part");
    if (!last && (row_end % unit || row_end > ncompr))
        return ms_fail(MS_ERR_INVALID, "col_slice: a view ends on a block boundary or at the column's end");
    const uint64_t b0 = row_begin / kBlock, b1 = (last ? ncompr : row_end) / kBlock;
    if (fmt == MS_FMT_STATIC_VBP) {
        const uint64_t boff = b0 * 64 * in->bw;
        v.data = static_cast<uint8_t *>(in->data) + boff;
        v.size_compr_byte = (b1 - b0) * 64 * in->bw;
        v.size_used_byte = last && nrest ? rest_offset(fmt, in->bw, v.size_compr_byte) + 8 * nrest : v.size_compr_byte;
        v.size_alloc_byte = in->size_alloc_byte - boff;
        v.index = v.index_aux = nullptr;
        v.n_index = 0;
    } else {
        if (b1 > b0 && (!in->index || in->n_index < b1 || (fmt == MS_FMT_FOR_DVBP && !in->index_aux)))
            return ms_fail(MS_ERR_INVALID, "col_slice: the column needs its block index (ms_gpu_build_index)");
        // blocks are found through the index (offsets from the column's start);
        // the sizes only place the uncompressed rest, which the last view keeps
        v.index = in->index ? in->index + b0 : nullptr;
        v.n_index = b1 - b0;
        v.index_aux = fmt == MS_FMT_FOR_DVBP ? (in->index_aux ? in->index_aux + b0 / 2 : nullptr)
                      : fmt == MS_FMT_DELTA_DVBP ? const_cast<uint64_t *>(d_carry_in)
                                                 : nullptr;
        if (!last) v.size_used_byte = v.size_compr_byte;
    }
    *out = v;
    return MS_OK;
}

extern "C" int ms_gpu_delta_lane_sums(const ms_col *in, uint64_t *d_sums, ms_arena *a, void *stream) {
    using namespace ms;
    if (!in || !d_sums || !a) return ms_fail(MS_ERR_INVALID, "delta_lane_sums: null argument");
    if (in->format != MS_FMT_DELTA_DVBP) return ms_fail(MS_ERR_INVALID, "delta_lane_sums: not a delta_f column");
    cudaStream_t st = (cudaStream_t)stream;
    ColView w;
    ms_col c = *in;
    c.index_aux = nullptr;  // the sums do not depend on the carry-in
    int rc = prepare_view(&c, a, st, &w);
    if (rc) return rc;
    const uint64_t nb = w.nb();
    if (!nb) {
        MS_CUDA_TRY(cudaMemsetAsync(d_sums, 0, 8 * sizeof(uint64_t), st));
        return MS_OK;
    }
    uint64_t *sums = arena_take_t<uint64_t>(a, nb * 8);
    uint64_t *excl = arena_take_t<uint64_t>(a, nb * 8);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nb, 8));
    if (!sums || !excl || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (delta lane sums)");
    k_delta_block_sums<<<persistent_grid(256, 8), 256, 0, st>>>(w, sums, a->d_err);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint64_t, 8>(sums, nb, excl, d_sums, scr, st)));
    return read_err(a, st);
}
