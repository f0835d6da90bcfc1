// ops.cu -- fused decompress-and-process operators: agg_sum, select,
// project and the select -> project -> agg_sum pipeline.
//
// Every kernel maps one warp to one 512-row block (colview.cuh) and keeps
// decoded values in registers, so uncompressed data never round-trips
// through HBM (the reference's decompress_and_process_batch, format.h:164-195,
// weaves decoding into the operator the same way on the CPU).
#include <mutex>

#include "internal.h"
#include "scan.cuh"

namespace ms {
namespace {

__device__ __forceinline__ uint64_t warp_sum(uint64_t x) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, s);
    return x;
}

// sum / count of y over the rows where cmp(x, val) holds.
//   kPred = false: every valid row of x counts (agg_sum, y unused)
//   kHasY = false: the sum is taken over x itself
//   blk_counts != nullptr: per-block hit counts (pass 1 of select)
template <bool kPred, bool kHasY>
__global__ void __launch_bounds__(256) k_sps(ColView x, ColView y, int cmp, uint64_t val,
                                            unsigned long long *__restrict__ d_sum,
                                            unsigned long long *__restrict__ d_cnt, uint32_t *__restrict__ blk_counts,
                                            unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    const uint64_t nbt = x.nblocks_total();
    uint64_t s = 0, cnt = 0;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nbt;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(x, b, l, q, v, valid);
        const unsigned m = kPred ? select_mask(x, b, l, q, v, valid, cmp, val) : valid;
        const unsigned c = __popc(m);
        cnt += c;
        if (blk_counts) {
            const unsigned tot = __reduce_add_sync(0xFFFFFFFFu, c);
            if (lane == 0) blk_counts[b] = tot;
        }
        if (kHasY) {
            if (__any_sync(0xFFFFFFFFu, m != 0)) {
                uint64_t w[16];
                unsigned vy;
                ok &= decode_block(y, b, l, q, w, vy);
#pragma unroll
                for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? w[k] : 0;
            }
        } else if (d_sum) {
#pragma unroll
            for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? v[k] : 0;
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
    s = warp_sum(s);
    cnt = warp_sum(cnt);
    if (lane == 0) {
        if (d_sum) atomicAdd(d_sum, (unsigned long long)s);
        if (d_cnt) atomicAdd(d_cnt, (unsigned long long)cnt);
    }
}

// Pass 2 of select: positions (and projected values of y) in row order.
template <bool kHasY>
__global__ void __launch_bounds__(256) k_select_write(ColView x, ColView y, int cmp, uint64_t val,
                                                     const uint64_t *__restrict__ blk_off,
                                                     uint64_t *__restrict__ out_pos, uint64_t *__restrict__ out_vals,
                                                     unsigned long long *__restrict__ d_scalar_hits, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    const uint64_t nbt = x.nblocks_total();
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nbt;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(x, b, l, q, v, valid);
        const unsigned m = select_mask(x, b, l, q, v, valid, cmp, val);
        if (!__any_sync(0xFFFFFFFFu, m != 0)) continue;
        unsigned rank[16];
        block_ranks(m, l, q, rank);
        const uint64_t base = blk_off[b], row0 = b * kBlock;
        uint64_t w[16];
        if (kHasY) {
            unsigned vy;
            ok &= decode_block(y, b, l, q, w, vy);
        }
        unsigned scal = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if ((m >> k) & 1u) {
                const uint64_t row = row0 + (16u * q + k) * 8u + l;
                if (out_pos) out_pos[base + rank[k]] = row;
                if (kHasY && out_vals) out_vals[base + rank[k]] = w[k];
                scal += row >= x.sfrom;
            }
        }
        if (scal) atomicAdd(d_scalar_hits, (unsigned long long)scal);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// rle input: per run (value, length).
__global__ void k_rle_sps(const uint64_t *__restrict__ pairs, uint64_t runs, bool pred, int cmp, uint64_t val,
                          unsigned long long *__restrict__ d_sum, unsigned long long *__restrict__ d_cnt) {
    uint64_t s = 0, c = 0;
    for (uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < runs; k += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t v = pairs[2 * k], len = pairs[2 * k + 1];
        // rle_f has no scalar-remainder split: compare as the AVX-512 path does
        if (!pred || cmp_eval(cmp, v, val, true)) {
            s += v * len;
            c += len;
        }
    }
    s = warp_sum(s);
    c = warp_sum(c);
    if ((threadIdx.x & 31u) == 0) {
        if (d_sum) atomicAdd(d_sum, (unsigned long long)s);
        if (d_cnt) atomicAdd(d_cnt, (unsigned long long)c);
    }
}

// Random access into a compressed column (project on compressed data): one
// thread per position.  static_vbp / dynamic_vbp / for_f read one or two
// lane-stream words (vbp_format_rndaccess.h:462-537 reads words w*8+lane
// and (w+1)*8+lane); other formats are decompressed first.
__global__ void k_gather(ColView d, const uint64_t *__restrict__ pos, uint64_t npos, uint64_t *__restrict__ out,
                         unsigned *err) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < npos; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t p = pos[i];
        if (p >= d.n) {
            atomicOr(err, kErrCorrupt);
            out[i] = 0;
            continue;
        }
        if (p >= d.n_compr) {
            out[i] = d.rest[p - d.n_compr];
            continue;
        }
        const uint64_t b = p / kBlock;
        const unsigned j = unsigned(p % kBlock), lane = j & 7u, slot = j >> 3;
        unsigned bw;
        uint64_t off;
        if (d.fmt == MS_FMT_STATIC_VBP) {
            bw = d.bw;
            off = b * 64ull * bw;
        } else {
            const uint64_t e = d.index[b];
            bw = idx_bw(e);
            off = idx_off(e);
        }
        const uint64_t *blk = reinterpret_cast<const uint64_t *>(d.data + off);
        const unsigned bit = slot * bw, w = bit >> 6, sh = bit & 63u;
        uint64_t x = blk[w * 8 + lane] >> sh;
        if (sh + bw > 64) x |= blk[(w + 1) * 8 + lane] << (64 - sh);
        if (bw < 64) x &= (uint64_t(1) << bw) - 1;
        if (d.fmt == MS_FMT_FOR_DVBP) x += d.aux[b >> 1];
        out[i] = x;
    }
}

}  // namespace

static unsigned grid_for_blocks(uint64_t nbt) {
    return (unsigned)maxu(1, minu((nbt + 7) / 8, persistent_grid(256, 8)));
}

// Pass 1 + scan + pass 2: uncompressed positions (and values of y) into
// arena arrays; returns counts.
static int select_positions(const ColView &x, const ColView *y, int cmp, uint64_t val, ms_arena *a, cudaStream_t st,
                            uint64_t **d_pos, uint64_t **d_vals, uint64_t *count, uint64_t *n_scalar) {
    const uint64_t nbt = x.nblocks_total();
    uint32_t *bc = arena_take_t<uint32_t>(a, nbt + 1);
    uint64_t *bo = arena_take_t<uint64_t>(a, nbt + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 2);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nbt, 1));
    if (!bc || !bo || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (select)");
    MS_CUDA_TRY(cudaMemsetAsync(tot, 0, 16, st));
    const unsigned grid = grid_for_blocks(nbt);
    if (nbt) {
        k_sps<true, false><<<grid, 256, 0, st>>>(x, x, cmp, val, nullptr, nullptr, bc, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(bc, nbt, bo, tot, scr, st)));
    }
    uint64_t total = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t *pos = arena_take_t<uint64_t>(a, total + 1);
    uint64_t *vals = y ? arena_take_t<uint64_t>(a, total + 1) : nullptr;
    if (!pos || (y && !vals)) return ms_fail(MS_ERR_NOMEM, "arena exhausted (select output)");
    MS_CUDA_TRY(cudaMemsetAsync(tot + 1, 0, 8, st));
    if (total) {
        if (y)
            k_select_write<true><<<grid, 256, 0, st>>>(x, *y, cmp, val, bo, pos, vals,
                                                      (unsigned long long *)(tot + 1), a->d_err);
        else
            k_select_write<false><<<grid, 256, 0, st>>>(x, x, cmp, val, bo, pos, nullptr,
                                                       (unsigned long long *)(tot + 1), a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    uint64_t scal = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&scal, tot + 1, 8, cudaMemcpyDeviceToHost, st));
    int rc = read_err(a, st);
    if (rc) return rc;
    *d_pos = pos;
    if (d_vals) *d_vals = vals;
    *count = total;
    *n_scalar = scal;
    return MS_OK;
}

int gather_values(const ms_col *data, const uint64_t *d_pos, uint64_t npos, uint64_t *d_out, ms_arena *a,
                  cudaStream_t st) {
    ColView dv;
    if (data->format == MS_FMT_DELTA_DVBP || data->format == MS_FMT_RLE) {
        // no random access into these formats: decompress, then gather
        uint64_t *tmp = arena_take_t<uint64_t>(a, data->count_values + 1);
        if (!tmp) return ms_fail(MS_ERR_NOMEM, "arena exhausted (project)");
        int rc = decompress_to(data, tmp, a, st);
        if (rc) return rc;
        dv = ColView{};
        dv.fmt = MS_FMT_UNCOMPR;
        dv.n = data->count_values;
        dv.rest = tmp;
    } else {
        int rc = prepare_view(data, a, st, &dv);
        if (rc) return rc;
    }
    if (npos) {
        k_gather<<<(unsigned)minu((npos + 255) / 256, persistent_grid(256, 8)), 256, 0, st>>>(dv, d_pos, npos,
                                                                                                  d_out, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    return MS_OK;
}

}  // namespace ms

using namespace ms;

// The fused select/sum launch: staged (TMA) pipeline or direct loads, as
// the current tuning says.
static int launch_sps(const ColView &x, const ColView &y, int cmp, uint64_t c, uint64_t *d_sum, uint64_t *d_count,
                      unsigned *d_err, cudaStream_t st) {
    MS_CUDA_TRY(cudaMemsetAsync(d_sum, 0, 8, st));
    if (d_count) MS_CUDA_TRY(cudaMemsetAsync(d_count, 0, 8, st));
    const uint64_t nbt = x.nblocks_total();
    if (!nbt) return MS_OK;
    const ms_tuning t = tuning();
    if (t.staged)
        return sps_tma(x, y, true, cmp, c, t.warps, t.stages, t.stage_bytes, t.ctas_per_sm, t.values_per_thread, d_sum,
                       d_count, d_err, st);
    k_sps<true, true><<<grid_for_blocks(nbt), 256, 0, st>>>(x, y, cmp, c, (unsigned long long *)d_sum,
                                                            (unsigned long long *)d_count, nullptr, d_err);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_agg_sum(const ms_col *in, uint64_t *d_sum, ms_arena *a, void *stream) {
    if (!in || !d_sum || !a) return ms_fail(MS_ERR_INVALID, "agg_sum: null argument");
    int rc = check_col(in, false);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    MS_CUDA_TRY(cudaMemsetAsync(d_sum, 0, 8, st));
    if (in->format == MS_FMT_RLE) {
        // sum over runs: value * length (rle.h:42-49 pairs)
        const uint64_t runs = in->size_used_byte / 16;
        if (runs) {
            k_rle_sps<<<(unsigned)minu((runs + 255) / 256, persistent_grid(256, 8)), 256, 0, st>>>(
                (const uint64_t *)in->data, runs, false, 0, 0, (unsigned long long *)d_sum, nullptr);
            MS_CUDA_TRY(cudaGetLastError());
        }
        return MS_OK;
    }
    ColView v;
    rc = prepare_view(in, a, st, &v);
    if (rc) return rc;
    const uint64_t nbt = v.nblocks_total();
    if (nbt) {
        k_sps<false, false><<<grid_for_blocks(nbt), 256, 0, st>>>(v, v, 0, 0, (unsigned long long *)d_sum, nullptr,
                                                                  nullptr, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    return MS_OK;
}

extern "C" int ms_gpu_select(int cmp, uint64_t val, const ms_col *in, int out_format, unsigned out_bw, ms_col *out,
                             ms_arena *a, void *stream) {
    if (!in || !out || !a) return ms_fail(MS_ERR_INVALID, "select: null argument");
    const bool all_unsigned = (cmp & MS_CMP_UNSIGNED) != 0;
    cmp &= ~MS_CMP_UNSIGNED;
    if (cmp < MS_CMP_EQ || cmp > MS_CMP_GE) return ms_fail(MS_ERR_INVALID, "select: unknown comparison");
    if (in->format == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "select: rle_f input has no sequential reader");
    cudaStream_t st = (cudaStream_t)stream;
    ColView x;
    int rc = prepare_view(in, a, st, &x);
    if (rc) return rc;
    // the scalar style compares every row unsigned: its "remainder" is the
    // whole column, and all hits are written as remainder rows
    if (all_unsigned) x.sfrom = 0;
    uint64_t *pos, cnt, nscal;
    rc = select_positions(x, nullptr, cmp, val, a, st, &pos, nullptr, &cnt, &nscal);
    if (rc) return rc;
    return write_values(pos, cnt - nscal, nscal, out_format, out_bw, out, a, st);
}

extern "C" int ms_gpu_project(const ms_col *data, const ms_col *pos, int out_format, unsigned out_bw, ms_col *out,
                              ms_arena *a, void *stream) {
    if (!data || !pos || !out || !a) return ms_fail(MS_ERR_INVALID, "project: null argument");
    int rc = check_col(data, false);
    if (rc) return rc;
    rc = check_col(pos, false);
    if (rc) return rc;
    if (pos->format == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "project: rle_f positions");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t npos = pos->count_values;
    const uint64_t *d_pos = (const uint64_t *)pos->data;
    if (pos->format != MS_FMT_UNCOMPR) {
        uint64_t *tmp = arena_take_t<uint64_t>(a, npos + 1);
        if (!tmp) return ms_fail(MS_ERR_NOMEM, "arena exhausted (project)");
        rc = decompress_to(pos, tmp, a, st);
        if (rc) return rc;
        d_pos = tmp;
    }
    uint64_t *vals = arena_take_t<uint64_t>(a, npos + 1);
    if (!vals) return ms_fail(MS_ERR_NOMEM, "arena exhausted (project output)");
    rc = gather_values(data, d_pos, npos, vals, a, st);
    if (rc) return rc;
    rc = read_err(a, st);
    if (rc) return rc;
    // outputs from the position column's scalar remainder are appended
    // uncompressed (project_compr.h:187-252)
    const uint64_t nscal = npos - scalar_from(*pos);
    return write_values(vals, npos - nscal, nscal, out_format, out_bw, out, a, st);
}

extern "C" int ms_gpu_select_project_sum(const ms_col *xc, int cmp, uint64_t c, const ms_col *yc, uint64_t *d_sum,
                                         uint64_t *d_count, uint64_t *d_pos, uint64_t *d_vals, ms_arena *a,
                                         void *stream) {
    if (!xc || !yc || !d_sum || !a) return ms_fail(MS_ERR_INVALID, "select_project_sum: null argument");
    if (cmp < MS_CMP_EQ || cmp > MS_CMP_GE) return ms_fail(MS_ERR_INVALID, "select_project_sum: unknown comparison");
    if (xc->count_values != yc->count_values)
        return ms_fail(MS_ERR_INVALID, "select_project_sum: x and y differ in length");
    if (xc->format == MS_FMT_RLE || yc->format == MS_FMT_RLE)
        return ms_fail(MS_ERR_UNSUPPORTED, "select_project_sum: rle_f input");
    cudaStream_t st = (cudaStream_t)stream;
    ColView x, y;
    int rc = prepare_view(xc, a, st, &x);
    if (rc) return rc;
    rc = prepare_view(yc, a, st, &y);
    if (rc) return rc;
    rc = launch_sps(x, y, cmp, c, d_sum, d_count, a->d_err, st);
    if (rc) return rc;
    if (d_pos || d_vals) {
        uint64_t *pos, *vals, cnt, nscal;
        rc = select_positions(x, &y, cmp, c, a, st, &pos, &vals, &cnt, &nscal);
        if (rc) return rc;
        if (d_pos && cnt) MS_CUDA_TRY(cudaMemcpyAsync(d_pos, pos, 8 * cnt, cudaMemcpyDeviceToDevice, st));
        if (d_vals && cnt) MS_CUDA_TRY(cudaMemcpyAsync(d_vals, vals, 8 * cnt, cudaMemcpyDeviceToDevice, st));
    }
    return MS_OK;
}

// Fused pipeline launch only (no scratch, no synchronisation): x and y must
// be static_vbp / uncompr, or carry a block index.  Used by benchmarks and
// graph capture.
extern "C" int ms_gpu_select_project_sum_async(const ms_col *xc, int cmp, uint64_t c, const ms_col *yc,
                                               uint64_t *d_sum, uint64_t *d_count, unsigned *d_err, void *stream) {
    if (!xc || !yc || !d_sum || !d_err) return ms_fail(MS_ERR_INVALID, "select_project_sum_async: null argument");
    if (xc->count_values != yc->count_values) return ms_fail(MS_ERR_INVALID, "x and y differ in length");
    for (const ms_col *col : {xc, yc}) {
        if (col->format == MS_FMT_RLE || col->format == MS_FMT_DELTA_DVBP)
            return ms_fail(MS_ERR_UNSUPPORTED, "select_project_sum_async: needs scratch for this format");
        if ((col->format == MS_FMT_DYNAMIC_VBP || col->format == MS_FMT_FOR_DVBP) && !col->index &&
            col->count_values >= kBlock)
            return ms_fail(MS_ERR_INVALID, "select_project_sum_async: dynamic_vbp column without index");
    }
    cudaStream_t st = (cudaStream_t)stream;
    ColView x, y;
    int rc = prepare_view(xc, nullptr, st, &x);
    if (rc) return rc;
    rc = prepare_view(yc, nullptr, st, &y);
    if (rc) return rc;
    return launch_sps(x, y, cmp, c, d_sum, d_count, d_err, st);
}

// ---------------------------------------------------------------------------
// Allocation-free select.
//
// Some callers cannot allocate device memory at all: code that runs after a
// host application has reserved the whole device budget up front, engines
// whose memory is owned by another allocator (a database buffer pool, a
// plugin host), and paths where cudaMalloc / cudaFree are forbidden because
// they synchronise the device.  For them this entry point takes the caller's
// input and output buffers and keeps its own scratch (per-block hit counts,
// block offsets, scan partials, the scalar-remainder hit counter) in one file-scope device
// array, kNoAllocScratchBytes large, which every GPU that loads the library
// holds until the process exits.  Inputs are limited to kNoAllocMaxRows rows
// so that the scratch fits.
//
// The array's host-side name is not a device address: its device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on the device.  That first call should
// therefore happen before any stream capture.  Every call shares the one
// array and it keeps the last call's contents, so calls that overlap on the
// GPU (concurrent streams, other threads) race; the counters that must start
// at zero are cleared at the start of every call.  The looked-up address is
// kept for the life of the process, so the entry point must not be used on a
// device after cudaDeviceReset (or after the primary context was otherwise
// destroyed and re-created).  Kernel errors (a corrupt header or bit width)
// go to the caller's d_err word, which is therefore required.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t round256(uint64_t x) { return (x + 255) / 256 * 256; }
constexpr uint64_t kNoAllocMaxRows = uint64_t(1) << 26;
constexpr uint64_t kNoAllocMaxBlocks = kNoAllocMaxRows / kBlock;
constexpr uint64_t kNoAllocCountsBytes = round256(4 * kNoAllocMaxBlocks);
constexpr uint64_t kNoAllocOffsetsBytes = round256(8 * kNoAllocMaxBlocks);
constexpr uint64_t kNoAllocScanWords = 2 * ((kNoAllocMaxBlocks + kScanTile - 1) / kScanTile) + 2 * 1 + 1;
constexpr uint64_t kNoAllocScanBytes = round256(8 * kNoAllocScanWords);
constexpr uint64_t kNoAllocWordsBytes = 256;  // scalar-hit counter
constexpr uint64_t kNoAllocScratchBytes =
    kNoAllocCountsBytes + kNoAllocOffsetsBytes + kNoAllocScanBytes + kNoAllocWordsBytes;

static_assert(kNoAllocScratchBytes <= (uint64_t(2) << 20), "no-alloc scratch is stated as at most 2 MiB");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

}  // namespace

static int noalloc_scratch_address(unsigned char **out) {
    constexpr int kMaxDevices = 64;
    static unsigned char *addr[kMaxDevices] = {};
    static std::mutex mu;
    int dev = 0;
    MS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return ms_fail(MS_ERR_INVALID, "select_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        MS_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = addr[dev];
    return MS_OK;
}

extern "C" uint64_t ms_gpu_select_noalloc_max_rows(void) { return kNoAllocMaxRows; }

extern "C" int ms_gpu_select_noalloc(int cmp, uint64_t val, const ms_col *in, uint64_t *d_out_pos,
                                     uint64_t out_capacity, uint64_t *d_out_count, unsigned *d_err, void *stream) {
    if (!in || !d_out_count || !d_err || (!d_out_pos && in->count_values))
        return ms_fail(MS_ERR_INVALID, "select_noalloc: null argument (d_out_count and d_err are required)");
    if (cmp < MS_CMP_EQ || cmp > MS_CMP_GE) return ms_fail(MS_ERR_INVALID, "select_noalloc: unknown comparison");
    int rc = check_col(in, false);
    if (rc) return rc;
    if (in->count_values > kNoAllocMaxRows)
        return ms_fail(MS_ERR_INVALID, "select_noalloc: column longer than 2^26 rows (the scratch limit)");
    if (out_capacity < in->count_values)
        return ms_fail(MS_ERR_INVALID, "select_noalloc: output capacity below the column length");
    if (in->format == MS_FMT_RLE || in->format == MS_FMT_DELTA_DVBP)
        return ms_fail(MS_ERR_UNSUPPORTED, "select_noalloc: rle_f / delta_f inputs need more scratch");
    const uint64_t nb_compr = (in->count_values - count_rest(*in)) / kBlock;
    if ((in->format == MS_FMT_DYNAMIC_VBP || in->format == MS_FMT_FOR_DVBP) && nb_compr &&
        (!in->index || in->n_index < nb_compr || (in->format == MS_FMT_FOR_DVBP && !in->index_aux)))
        return ms_fail(MS_ERR_INVALID, "select_noalloc: dynamic_vbp / for_f input needs its block index");
    unsigned char *scr = nullptr;
    rc = noalloc_scratch_address(&scr);
    if (rc) return rc;
    uint32_t *counts = reinterpret_cast<uint32_t *>(scr);
    uint64_t *offsets = reinterpret_cast<uint64_t *>(scr + kNoAllocCountsBytes);
    uint64_t *scan_scr = reinterpret_cast<uint64_t *>(scr + kNoAllocCountsBytes + kNoAllocOffsetsBytes);
    unsigned long long *scalar_hits =
        reinterpret_cast<unsigned long long *>(scr + kNoAllocCountsBytes + kNoAllocOffsetsBytes + kNoAllocScanBytes);
    unsigned *err = d_err;
    cudaStream_t st = (cudaStream_t)stream;
    ColView x;
    rc = prepare_view(in, nullptr, st, &x);
    if (rc) return rc;
    MS_CUDA_TRY(cudaMemsetAsync(scalar_hits, 0, kNoAllocWordsBytes, st));
    MS_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(unsigned), st));
    const uint64_t nbt = x.nblocks_total();
    if (nbt == 0) {
        MS_CUDA_TRY(cudaMemsetAsync(d_out_count, 0, 8, st));
        return MS_OK;
    }
    if (scan_scratch_words(nbt, 1) > kNoAllocScanWords)
        return ms_fail(MS_ERR_INVALID, "select_noalloc: scan scratch too small");
    const unsigned grid = grid_for_blocks(nbt);
    k_sps<true, false><<<grid, 256, 0, st>>>(x, x, cmp, val, nullptr, nullptr, counts, err);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(counts, nbt, offsets, d_out_count, scan_scr, st)));
    k_select_write<false><<<grid, 256, 0, st>>>(x, x, cmp, val, offsets, d_out_pos, nullptr, scalar_hits, err);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}
