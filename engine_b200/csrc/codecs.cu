// codecs.cu -- compression and decompression kernels for every format and
// the column-level morph (morph.h:81-241).
//
// Encoding a dynamic_vbp-family column is size-then-scatter:
//   1. k_analyze: one warp per 512-value block computes the block's bit width
//      (OR-reduce, dynamic_vbp.h:124-158) after the cascade transform
//      (delta: x[i]-x[i-8], delta.h:107-156; for: minus the block minimum,
//      for.h:121-161);
//   2. an exclusive scan of the bit widths gives every block's byte offset:
//      64 * (headers before the block) + 64 * (sum of earlier widths);
//   3. k_pack: one thread per lane stream (8 per block) packs the block at
//      its offset and records the block index entry; k_headers writes the
//      page headers (bit-width bytes / 0xFF, FOR reference words).
// The same encoder writes operator outputs with the write iterator's
// 2048-value chunking (write_iterator.h:67-306): only the number of blocks
// per page changes (64 -> 4 for dynamic_vbp, 8 -> 2 for for_f).
#include <string.h>

#include "internal.h"
#include "scan.cuh"
#include "tma.cuh"

namespace ms {
namespace {

struct Layout {
    int fmt;
    unsigned bw;           // static_vbp
    unsigned dvbp_page;    // blocks per dynamic_vbp page (64 morph, 4 write iterator)
    unsigned for_page;     // cascade blocks per for_f page (8 morph, 2 write iterator)
};

// 64-B headers preceding block b's packed data.
__host__ __device__ inline uint64_t headers_before(const Layout &L, uint64_t b) {
    switch (L.fmt) {
    case MS_FMT_DYNAMIC_VBP: return b / L.dvbp_page + 1;
    case MS_FMT_DELTA_DVBP: return b / 2 + 1;
    case MS_FMT_FOR_DVBP: return b / (2 * L.for_page) + 1 + b / 2 + 1;
    default: return 0;
    }
}

__device__ __forceinline__ uint64_t warp_or(uint64_t x) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) x |= __shfl_xor_sync(0xFFFFFFFFu, x, s);
    return x;
}

// --- 1. analysis -----------------------------------------------------------
// dynamic_vbp / delta: one warp per 512-block.
template <int FMT>
__global__ void __launch_bounds__(256) k_analyze_blocks(const uint64_t *__restrict__ in, uint64_t nb,
                                                       uint32_t *__restrict__ bw_out) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nb;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const uint64_t *blk = in + b * kBlock;
        uint64_t acc = 1;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const unsigned r = k * 32 + lane;  // coalesced rows
            uint64_t x = __ldg(blk + r);
            if (FMT == MS_FMT_DELTA_DVBP) {
                const uint64_t row = b * kBlock + r;
                x -= row >= 8 ? __ldg(in + row - 8) : 0;
            }
            acc |= x;
        }
        acc = warp_or(acc);
        if (lane == 0) bw_out[b] = effective_bitwidth(acc);
    }
}

// for_f: one warp per 1024-block; reference = AVX-512 TVL minimum (signed
// per lane, _mm512_min_epi64, then unsigned across lanes; for.h:121-161).
__global__ void __launch_bounds__(256) k_analyze_for(const uint64_t *__restrict__ in, uint64_t ncb,
                                                    uint32_t *__restrict__ bw_out, uint64_t *__restrict__ refs) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t c = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; c < ncb;
         c += uint64_t(gridDim.x) * blockDim.x / 32) {
        const uint64_t *blk = in + c * kCascBlock;
        // lane & 7 is the TVL lane of every row this thread reads
        int64_t mn = INT64_MAX;
        uint64_t x[32];
#pragma unroll
        for (int k = 0; k < 32; k++) {
            x[k] = __ldg(blk + k * 32 + lane);
            mn = min(mn, (int64_t)x[k]);
        }
        mn = min(mn, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (uint64_t)mn, 8));
        mn = min(mn, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (uint64_t)mn, 16));
        uint64_t um = (uint64_t)mn;
        um = min(um, __shfl_xor_sync(0xFFFFFFFFu, um, 1));
        um = min(um, __shfl_xor_sync(0xFFFFFFFFu, um, 2));
        um = min(um, __shfl_xor_sync(0xFFFFFFFFu, um, 4));
        if (um == ~uint64_t(0)) um--;
        uint64_t o0 = 1, o1 = 1;
#pragma unroll
        for (int k = 0; k < 16; k++) o0 |= x[k] - um;
#pragma unroll
        for (int k = 16; k < 32; k++) o1 |= x[k] - um;
        o0 = warp_or(o0);
        o1 = warp_or(o1);
        if (lane == 0) {
            refs[c] = um;
            bw_out[2 * c] = effective_bitwidth(o0);
            bw_out[2 * c + 1] = effective_bitwidth(o1);
        }
    }
}

// --- 3. packing -------------------------------------------------------------
// Eight threads per block, one per lane stream; a warp packs four blocks.
template <int FMT>
__global__ void __launch_bounds__(256) k_pack(const uint64_t *__restrict__ in, uint64_t nb, Layout L,
                                             const uint32_t *__restrict__ bws, const uint64_t *__restrict__ prefix,
                                             const uint64_t *__restrict__ refs, uint8_t *__restrict__ out,
                                             uint64_t *__restrict__ index, unsigned *err) {
    const unsigned l = threadIdx.x & 7u;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 8; b < nb;
         b += uint64_t(gridDim.x) * blockDim.x / 8) {
        unsigned bw;
        uint64_t off;
        if (FMT == MS_FMT_STATIC_VBP) {
            bw = L.bw;
            off = b * 64ull * bw;
        } else {
            bw = bws[b];
            off = 64ull * headers_before(L, b) + 64ull * prefix[b];
            if (l == 0 && index) index[b] = idx_pack(off, bw);
        }
        const uint64_t *blk = in + b * kBlock;
        const uint64_t ref = FMT == MS_FMT_FOR_DVBP ? refs[b >> 1] : 0;
        auto get = [&](unsigned v) -> uint64_t {
            const unsigned r = v * 8 + l;
            uint64_t x = __ldg(blk + r);
            if (FMT == MS_FMT_DELTA_DVBP) {
                const uint64_t row = b * kBlock + r;
                x -= row >= 8 ? __ldg(in + row - 8) : 0;
            } else if (FMT == MS_FMT_FOR_DVBP) {
                x -= ref;
            }
            return x;
        };
        if (!vbp_pack_lane_rt(bw, get, reinterpret_cast<uint64_t *>(out + off), l)) atomicOr(err, kErrCorrupt);
    }
}

// Page headers.  dynamic_vbp: one thread per header byte.
__global__ void k_headers_dvbp(uint64_t nb, Layout L, const uint32_t *__restrict__ bws,
                               const uint64_t *__restrict__ prefix, uint8_t *__restrict__ out) {
    const uint64_t pages = (nb + L.dvbp_page - 1) / L.dvbp_page;
    for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < pages * kPageBlocks;
         t += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t p = t / kPageBlocks, j = t % kPageBlocks, b0 = p * L.dvbp_page;
        const uint64_t start = 64ull * headers_before(L, b0) + 64ull * prefix[b0] - 64;
        const uint64_t b = b0 + j;
        out[start + j] = (j < L.dvbp_page && b < nb) ? uint8_t(bws[b]) : uint8_t(kNoBlock);
    }
}

// delta / for: inner dynamic_vbp header of each 1024-block (2 widths + 62 x
// 0xFF) and, for for_f, the page header of reference words.
template <int FMT>
__global__ void k_headers_casc(uint64_t nb, Layout L, const uint32_t *__restrict__ bws,
                               const uint64_t *__restrict__ prefix, const uint64_t *__restrict__ refs,
                               uint8_t *__restrict__ out) {
    const uint64_t ncb = nb / 2;
    for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < ncb * 8;
         t += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t c = t / 8, w = t % 8;
        const uint64_t start = 64ull * headers_before(L, 2 * c) + 64ull * prefix[2 * c] - 64;
        uint64_t word = ~uint64_t(0);
        if (w == 0) word = (~uint64_t(0) << 16) | uint64_t(bws[2 * c] & 0xFF) | (uint64_t(bws[2 * c + 1] & 0xFF) << 8);
        reinterpret_cast<uint64_t *>(out + start)[w] = word;
        if (FMT == MS_FMT_FOR_DVBP && c % L.for_page == 0) {
            const uint64_t fstart = start - 64;
            const uint64_t nbp = minu(L.for_page, ncb - c);
            uint64_t fw;
            if (w < nbp) fw = refs[c + w];
            else if (w == nbp) fw = ~uint64_t(0);
            else fw = 0;
            reinterpret_cast<uint64_t *>(out + fstart)[w] = fw;
        }
    }
}

// Uncompressed rest: copied behind the gap (morph.h:186-189,
// write_iterator.h:157-170).  The compressed size is read on the device.
__global__ void k_copy_rest(const uint64_t *__restrict__ in, uint64_t nrest, int fmt, unsigned bw,
                            const uint64_t *__restrict__ d_compr, uint8_t *__restrict__ out) {
    const uint64_t ro = rest_offset(fmt, bw, *d_compr);
    uint64_t *dst = reinterpret_cast<uint64_t *>(out + ro);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nrest; i += uint64_t(gridDim.x) * blockDim.x)
        dst[i] = in[i];
}

__global__ void k_finish_sizes(uint64_t nb, Layout L, const uint32_t *__restrict__ bws,
                               const uint64_t *__restrict__ prefix, uint64_t *__restrict__ d_compr) {
    if (threadIdx.x || blockIdx.x) return;
    if (nb == 0) {
        *d_compr = 0;
        return;
    }
    if (L.fmt == MS_FMT_STATIC_VBP) {
        *d_compr = nb * 64ull * L.bw;
        return;
    }
    *d_compr = 64ull * headers_before(L, nb - 1) + 64ull * prefix[nb - 1] + 64ull * bws[nb - 1];
}

// --- decompression ------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) k_decode_all(ColView c, uint64_t *__restrict__ out, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    const uint64_t nbt = c.nblocks_total();
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nbt;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        if (!decode_block(c, b, l, q, v, valid) && lane == 0) atomicOr(err, kErrCorrupt);
        const uint64_t row0 = b * kBlock;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((valid >> k) & 1u) out[row0 + (16u * q + k) * 8u + l] = v[k];
    }
}

// --- rle ----------------------------------------------------------------------
// Encoder: one pass over the input in tiles of kRleTile rows, tiles taken in
// order from a ticket counter.  A row starts a run (a "head") when it differs
// from the row before (rle.h:63-150: maximal runs).  Each tile needs the
// number of runs before it (its first head's run index) and the row of the
// last head before it (where the run its first head ends began): both come
// from a decoupled look-back over the tiles before it (every tile publishes
// its own run count and last head, then -- once known -- the inclusive
// values).  Every head writes its run's value and the length of the run
// before it; the last tile writes the length of the final run.  So the input
// is read once and each pair written once (8 B/row + 16 B/run).
constexpr unsigned kRleEncThreads = 1024;
constexpr unsigned kRleRowsPerThread = 16;
constexpr unsigned kRleEncTile = kRleEncThreads * kRleRowsPerThread;  // rows per encoder tile
constexpr uint64_t kRleNone = ~uint64_t(0);
enum : unsigned { kRleFlagAgg = 1, kRleFlagInc = 2 };

// A tile's published values in two 64-bit words, each carrying the flag in
// its low two bits (0: nothing yet, kRleFlagAgg: the tile's own values,
// kRleFlagInc: the values over tiles [0, this tile]): r = runs << 2 | flag,
// l = (last head + 1, 0 for none) << 2 | flag.  Each word is written and
// read whole, so a value is never seen without its flag and no fence is
// needed; a reader that sees the two words with different flags (one
// already updated) reads again.
struct RleTileState {
    unsigned long long r, l;
};

__device__ __forceinline__ void rle_publish(RleTileState *s, unsigned flag, uint64_t runs, uint64_t last) {
    const unsigned long long r = (runs << 2) | flag;
    const unsigned long long l = ((last == kRleNone ? 0 : last + 1) << 2) | flag;
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(s), "l"(r), "l"(l) : "memory");
}

// Warp-wide look-back (warp 0 of the tile): lane i inspects tile j - i, 32
// predecessors per step, with one 16-byte load per lane and step; the
// nearest one with an inclusive prefix ends the walk.  Returns false if a
// predecessor never published (bounded spin).
__device__ bool rle_lookback(const RleTileState *state, uint64_t tile, uint64_t &excl_runs, uint64_t &excl_last) {
    const unsigned lane = threadIdx.x & 31u;
    excl_runs = 0;
    excl_last = kRleNone;
    for (int64_t j = int64_t(tile) - 1; j >= 0; j -= 32) {
        const int64_t me = j - int64_t(lane);
        unsigned f = kRleFlagInc;  // lanes before tile 0 act as an empty inclusive prefix
        uint64_t cr = 0, cl = kRleNone;
        if (me >= 0) {
            const RleTileState *o = state + me;
            unsigned long long r = 0, l = 0;
            for (unsigned spins = 0; spins < kSpinLimit; spins++) {
                asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(r), "=l"(l) : "l"(o) : "memory");
                if ((r & 3u) != 0 && (r & 3u) == (l & 3u)) break;
            }
            f = (r & 3u) == (l & 3u) ? unsigned(r & 3u) : 0u;
            cr = r >> 2;
            cl = (l >> 2) ? (l >> 2) - 1 : kRleNone;
        }
        if (__any_sync(0xFFFFFFFFu, f == 0)) return false;
        const unsigned inc = __ballot_sync(0xFFFFFFFFu, f == kRleFlagInc);
        const unsigned stop = inc ? unsigned(__ffs(inc) - 1) : 32u;  // lanes 0..stop count
        const bool take = lane <= stop;
        uint64_t r = take ? cr : 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) r += __shfl_xor_sync(0xFFFFFFFFu, r, d);
        excl_runs += r;
        if (excl_last == kRleNone) {
            // the nearest taken predecessor with a head
            const unsigned has = __ballot_sync(0xFFFFFFFFu, take && cl != kRleNone);
            if (has) excl_last = __shfl_sync(0xFFFFFFFFu, cl, __ffs(has) - 1);
        }
        if (inc) break;
    }
    return true;
}

__global__ void __launch_bounds__(kRleEncThreads) k_rle_encode(const uint64_t *__restrict__ in, uint64_t n,
                                                              RleTileState *state, unsigned *ticket,
                                                              uint64_t *__restrict__ out,
                                                              uint64_t *__restrict__ d_runs, unsigned *err) {
    constexpr unsigned NW = kRleEncThreads / 32, WR = 32 * kRleRowsPerThread;  // warps, rows per warp
    __shared__ uint64_t s_tile;
    __shared__ unsigned s_wcnt[NW];
    __shared__ uint64_t s_wlast[NW];
    __shared__ uint64_t s_excl_runs, s_excl_last;
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t ntiles = (n + kRleEncTile - 1) / kRleEncTile;
    if (tile >= ntiles) return;
    // warp w covers WR consecutive rows; in step k lane l reads row base + 32 k + l
    // (one coalesced 256-byte load per step); heads as one ballot per step
    const uint64_t base = tile * kRleEncTile + uint64_t(wid) * WR;
    uint64_t carry = base > 0 && base <= n ? __ldg(in + base - 1) : 0;  // the row before the step's first
    unsigned ball[kRleRowsPerThread];
    unsigned c = 0;
#pragma unroll
    for (unsigned k = 0; k < kRleRowsPerThread; k++) {
        const uint64_t r = base + 32 * k + lane;
        const uint64_t v = r < n ? __ldg(in + r) : 0;
        const uint64_t up = __shfl_up_sync(0xFFFFFFFFu, v, 1);
        const uint64_t prev = lane ? up : carry;
        carry = __shfl_sync(0xFFFFFFFFu, v, 31);
        ball[k] = __ballot_sync(0xFFFFFFFFu, r < n && (r == 0 || v != prev));
        c += __popc(ball[k]);
    }
    // last head of this warp as row + 1 (0: none)
    uint64_t my_last = 0;
#pragma unroll
    for (unsigned k = 0; k < kRleRowsPerThread; k++)
        if (ball[k]) my_last = base + 32 * k + (31 - __clz(ball[k])) + 1;
    if (lane == 0) {
        s_wcnt[wid] = c;
        s_wlast[wid] = my_last;
    }
    __syncthreads();
    unsigned wpre = 0;
    uint64_t wlast = 0;
    for (unsigned w = 0; w < wid; w++) {
        wpre += s_wcnt[w];
        wlast = maxu(wlast, s_wlast[w]);
    }
    if (wid == 0) {
        // the whole tile: runs and last head; publish, then look back
        uint64_t agg_runs = 0, agg_last = 0;
        for (unsigned w = 0; w < NW; w++) {
            agg_runs += s_wcnt[w];
            agg_last = maxu(agg_last, s_wlast[w]);
        }
        RleTileState *me = state + tile;
        const uint64_t own_last = agg_last ? agg_last - 1 : kRleNone;
        uint64_t excl_runs = 0, excl_last = kRleNone;
        if (tile == 0) {
            if (lane == 0) rle_publish(me, kRleFlagInc, agg_runs, own_last);
        } else {
            if (lane == 0) rle_publish(me, kRleFlagAgg, agg_runs, own_last);
            __syncwarp();
            if (!rle_lookback(state, tile, excl_runs, excl_last) && lane == 0) atomicOr(err, kErrTimeout);
            if (lane == 0)
                rle_publish(me, kRleFlagInc, excl_runs + agg_runs, own_last != kRleNone ? own_last : excl_last);
        }
        if (lane == 0) {
            s_excl_runs = excl_runs;
            s_excl_last = excl_last;
            if (tile == ntiles - 1) {
                // the final run ends at row n
                const uint64_t total = excl_runs + agg_runs;
                const uint64_t last = own_last != kRleNone ? own_last : excl_last;
                *d_runs = total;
                if (total) out[2 * (total - 1) + 1] = n - last;
            }
        }
    }
    __syncthreads();
    // pairs: every head writes its run's value and the length of the run
    // before it; consecutive lanes write consecutive pairs
    uint64_t k_run = s_excl_runs + wpre;                       // run index of the warp's next head
    uint64_t prev_head = wlast ? wlast - 1 : s_excl_last;      // row of the head before it
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (unsigned k = 0; k < kRleRowsPerThread; k++) {
        const unsigned bk = ball[k];
        if (!bk) continue;
        const uint64_t r = base + 32 * k + lane;
        if ((bk >> lane) & 1u) {
            const uint64_t idx = k_run + __popc(bk & below);
            const unsigned lower = bk & below;
            const uint64_t ph = lower ? base + 32 * k + (31 - __clz(lower)) : prev_head;
            out[2 * idx] = __ldg(in + r);
            if (idx) out[2 * (idx - 1) + 1] = r - ph;
        }
        k_run += __popc(bk);
        prev_head = base + 32 * k + (31 - __clz(bk));
    }
}

// Staged encoder: the same algorithm, one tile of kRleStThreads *
// kRleRowsPerThread rows per CTA, with the tile's rows brought into shared
// memory by asynchronous 16-byte copies (cp.async) that are all in flight at
// once instead of one register load per step; each lane compares its row
// with the one before it in shared memory.  Three CTAs per SM, so one CTA's
// look-back overlaps the others' reads.  Needs a 16-byte aligned input.
constexpr unsigned kRleStThreads = 512;
constexpr unsigned kRleStTile = kRleStThreads * kRleRowsPerThread;

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__global__ void __launch_bounds__(kRleStThreads) k_rle_encode_staged(const uint64_t *__restrict__ in, uint64_t n,
                                                                    RleTileState *state, unsigned *ticket,
                                                                    uint64_t *__restrict__ out,
                                                                    uint64_t *__restrict__ d_runs, unsigned *err) {
    constexpr unsigned NW = kRleStThreads / 32, WR = 32 * kRleRowsPerThread;
    extern __shared__ __align__(128) uint8_t rle_smem[];
    uint64_t *const v = reinterpret_cast<uint64_t *>(rle_smem);  // the tile's rows
    __shared__ uint64_t s_tile;
    __shared__ unsigned s_ball[NW][kRleRowsPerThread];
    __shared__ unsigned s_wcnt[NW];
    __shared__ uint64_t s_wlast[NW];
    __shared__ uint64_t s_excl_runs, s_excl_last;
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t ntiles = (n + kRleStTile - 1) / kRleStTile;
    if (tile >= ntiles) return;
    const uint64_t r0 = tile * kRleStTile;
    const unsigned rows = unsigned(minu(kRleStTile, n - r0));
    {
        // every 16-byte pair of rows of the tile, consecutive threads on
        // consecutive pairs; an odd last row of the column is read directly
        const unsigned pairs = rows / 2;
        for (unsigned q = threadIdx.x; q < pairs; q += kRleStThreads) cp_async16(v + 2 * q, in + r0 + 2 * q);
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        if ((rows & 1u) && threadIdx.x == 0) v[rows - 1] = __ldg(in + r0 + rows - 1);
    }
    __syncthreads();
    // heads: warp w covers tile rows [w WR, (w + 1) WR), lane-strided; the
    // tile's first row is compared with the previous tile's last
    const unsigned wbase = wid * WR;
    const uint64_t before = r0 ? __ldg(in + r0 - 1) : 0;
    unsigned c = 0;
    uint64_t my_last = 0;  // last head of this warp as row + 1 (0: none)
#pragma unroll
    for (unsigned k = 0; k < kRleRowsPerThread; k++) {
        const unsigned lr = wbase + 32 * k + lane;
        const bool valid = lr < rows;
        const uint64_t x = valid ? v[lr] : 0;
        const uint64_t prev = lr ? v[lr - 1] : before;
        const unsigned bk = __ballot_sync(0xFFFFFFFFu, valid && (r0 + lr == 0 || x != prev));
        if (lane == 0) s_ball[wid][k] = bk;
        c += __popc(bk);
        if (bk) my_last = r0 + wbase + 32 * k + (31 - __clz(bk)) + 1;
    }
    if (lane == 0) {
        s_wcnt[wid] = c;
        s_wlast[wid] = my_last;
    }
    __syncthreads();
    if (wid == 0) {
        // the whole tile: runs and last head; publish, then look back
        uint64_t agg_runs = lane < NW ? s_wcnt[lane] : 0, agg_last = lane < NW ? s_wlast[lane] : 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            agg_runs += __shfl_xor_sync(0xFFFFFFFFu, agg_runs, d);
            agg_last = maxu(agg_last, __shfl_xor_sync(0xFFFFFFFFu, agg_last, d));
        }
        RleTileState *me = state + tile;
        const uint64_t own_last = agg_last ? agg_last - 1 : kRleNone;
        uint64_t excl_runs = 0, excl_last = kRleNone;
        if (tile > 0) {
            if (lane == 0) rle_publish(me, kRleFlagAgg, agg_runs, own_last);
            __syncwarp();
            if (!rle_lookback(state, tile, excl_runs, excl_last) && lane == 0) atomicOr(err, kErrTimeout);
        }
        if (lane == 0) {
            rle_publish(me, kRleFlagInc, excl_runs + agg_runs, own_last != kRleNone ? own_last : excl_last);
            s_excl_runs = excl_runs;
            s_excl_last = excl_last;
            if (tile == ntiles - 1) {
                // the final run ends at row n
                const uint64_t total = excl_runs + agg_runs;
                const uint64_t last = own_last != kRleNone ? own_last : excl_last;
                *d_runs = total;
                if (total) out[2 * (total - 1) + 1] = n - last;
            }
        }
    }
    __syncthreads();
    // pairs: every head writes its run's value and the length of the run
    // before it; consecutive lanes write consecutive pairs
    unsigned wpre = 0;
    uint64_t wlast = 0;
    for (unsigned w = 0; w < wid; w++) {
        wpre += s_wcnt[w];
        wlast = maxu(wlast, s_wlast[w]);
    }
    uint64_t k_run = s_excl_runs + wpre;                   // run index of the warp's next head
    uint64_t prev_head = wlast ? wlast - 1 : s_excl_last;  // row of the head before it
    const unsigned below = (1u << lane) - 1u;
#pragma unroll 4
    for (unsigned k = 0; k < kRleRowsPerThread; k++) {
        const unsigned bk = s_ball[wid][k];
        if (!bk) continue;
        const unsigned lr = wbase + 32 * k + lane;
        if ((bk >> lane) & 1u) {
            const uint64_t idx = k_run + __popc(bk & below);
            const unsigned lower = bk & below;
            const uint64_t ph = lower ? r0 + wbase + 32 * k + (31 - __clz(lower)) : prev_head;
            out[2 * idx] = v[lr];
            if (idx) out[2 * (idx - 1) + 1] = r0 + lr - ph;
        }
        k_run += __popc(bk);
        prev_head = r0 + wbase + 32 * k + (31 - __clz(bk));
    }
}

constexpr unsigned kRleThreads = 256;
constexpr unsigned kRleRunsPerThread = 8;
constexpr unsigned kRleTile = kRleThreads * kRleRunsPerThread;  // most runs per decoder tile
constexpr unsigned kRleRows = 8192;  // output rows per decoder CTA
// Runs per decoder tile: about as many as one output chunk of kRleRows rows
// holds at the column's mean run length, a power of two in [kRleThreads,
// kRleTile].  Long runs thus mean small tiles, so a chunk loads and scans
// few runs it does not write.
inline unsigned rle_tile_runs(uint64_t n, uint64_t runs) {
    unsigned tr = kRleTile;
    while (tr > kRleThreads && uint64_t(tr) * n > uint64_t(kRleRows) * runs) tr >>= 1;
    return tr;
}

// Decoder, pass 1: run lengths summed per tile of kRleTile runs.
__global__ void __launch_bounds__(kRleThreads) k_rle_tile_rows(const uint64_t *__restrict__ pairs, uint64_t runs,
                                                              unsigned tr, uint64_t *__restrict__ tile_rows) {
    __shared__ uint64_t s_w[kRleThreads / 32];
    const uint64_t t = blockIdx.x, base = t * tr;
    uint64_t s = 0;
    for (unsigned i = threadIdx.x; i < tr; i += kRleThreads) {
        const uint64_t r = base + i;
        if (r < runs) s += __ldg(pairs + 2 * r + 1);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, d);
    if ((threadIdx.x & 31u) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t tot = 0;
        for (unsigned w = 0; w < kRleThreads / 32; w++) tot += s_w[w];
        tile_rows[t] = tot;
    }
}

// Decoder, pass 2: the run tile holding the first row of every chunk of
// kRleRows output rows (one thread per chunk, binary search over the tiles'
// first rows).

__global__ void k_rle_chunk_tiles(const uint64_t *__restrict__ tile_first, uint64_t ntiles, uint64_t chunks,
                                  uint32_t *__restrict__ chunk_tile) {
    for (uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < chunks; c += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t row0 = c * kRleRows;
        uint64_t lo = 0, hi = ntiles;  // last tile whose first row <= row0
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) / 2;
            if (tile_first[mid] <= row0) lo = mid;
            else hi = mid;
        }
        chunk_tile[c] = uint32_t(lo);
    }
}

// Decoder, pass 3: each CTA writes kRleRows output rows.  Starting at the
// run tile that holds its first row, it stages that tile's pairs in shared
// memory and turns them into (value, start) lists -- zero-length runs
// dropped, as they write nothing (rle.h:238-249) -- while marking each run
// start inside its rows in a bitmap (one 32-bit word per 32 rows).  Each
// warp then writes a contiguous range of words: row 32 u + l belongs to the
// run counted by the starts before word u plus the bits of word u at or
// below l.  It moves on to the next tile until its rows are done.  RPT runs
// per thread: the tile holds RPT * kRleThreads runs.
template <unsigned RPT>
__global__ void __launch_bounds__(kRleThreads) k_rle_expand(const uint64_t *__restrict__ pairs, uint64_t runs,
                                                           const uint64_t *__restrict__ tile_first, uint64_t ntiles,
                                                           const uint32_t *__restrict__ chunk_tile,
                                                           const uint64_t *__restrict__ total_rows, uint64_t n,
                                                           uint64_t *__restrict__ out, unsigned *err) {
    constexpr unsigned NWP = kRleThreads / 32, TR = RPT * kRleThreads, NWD = kRleRows / 32;
    __shared__ uint64_t s_val[TR];
    __shared__ uint64_t s_len[TR];  // lengths, then (as 32-bit words) the kept runs' entries
    __shared__ unsigned s_bits[NWD];  // run starts per 32-row word of the CTA's rows
    __shared__ uint64_t s_wsum[NWP];
    __shared__ unsigned s_wcnt[NWP];
    // a kept run's entry is 1 + its start's offset from row0 (0: it starts
    // before row0): row row0 + r lies in the last run whose entry is <= r + 1
    uint32_t *const s_st = reinterpret_cast<uint32_t *>(s_len);
    const uint64_t row0 = uint64_t(blockIdx.x) * kRleRows;
    if (row0 >= n) return;
    const uint64_t row1 = minu(n, row0 + kRleRows);
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const unsigned incl = (2u << lane) - 1u;  // lanes 0..lane
    for (uint64_t t = chunk_tile[blockIdx.x]; t < ntiles && tile_first[t] < row1; t++) {
        const uint64_t rbase = t * TR;
        const unsigned nr = unsigned(minu(TR, runs - rbase));
        // the tile's pairs into shared memory, one 16-byte pair per thread and step
#pragma unroll
        for (unsigned k = 0; k < RPT; k++) {
            const unsigned j = threadIdx.x + k * kRleThreads;
            const ulonglong2 pr = j < nr ? __ldg(reinterpret_cast<const ulonglong2 *>(pairs) + rbase + j)
                                         : make_ulonglong2(0, 0);
            s_val[j] = pr.x;
            s_len[j] = pr.y;
        }
        for (unsigned w = threadIdx.x; w < NWD; w += kRleThreads) s_bits[w] = 0;
        __syncthreads();
        // this thread's RPT consecutive runs: exclusive scans of the lengths
        // and of the number of non-empty runs
        const unsigned j0 = threadIdx.x * RPT;
        uint64_t len[RPT], val[RPT], sum = 0;
        unsigned cnt = 0;
#pragma unroll
        for (unsigned k = 0; k < RPT; k++) {
            len[k] = s_len[j0 + k];
            val[k] = s_val[j0 + k];
            sum += len[k];
            cnt += len[k] != 0;
        }
        uint64_t isum = sum;
        unsigned icnt = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, isum, d);
            const unsigned co = __shfl_up_sync(0xFFFFFFFFu, icnt, d);
            if (int(lane) >= d) {
                isum += o;
                icnt += co;
            }
        }
        if (lane == 31) {
            s_wsum[wid] = isum;
            s_wcnt[wid] = icnt;
        }
        __syncthreads();
        // the warps before this one: lanes 0..NWP-1 scan the warp totals
        uint64_t ws = lane < NWP ? s_wsum[lane] : 0;
        unsigned wc = lane < NWP ? s_wcnt[lane] : 0;
#pragma unroll
        for (int d = 1; d < int(NWP); d <<= 1) {
            const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, ws, d);
            const unsigned co = __shfl_up_sync(0xFFFFFFFFu, wc, d);
            if (int(lane) >= d) {
                ws += o;
                wc += co;
            }
        }
        const unsigned kept = __shfl_sync(0xFFFFFFFFu, wc, NWP - 1);
        const uint64_t wpre = wid ? __shfl_sync(0xFFFFFFFFu, ws, wid - 1) : 0;
        const unsigned cpre = wid ? __shfl_sync(0xFFFFFFFFu, wc, wid - 1) : 0;
        uint64_t run = tile_first[t] + wpre + isum - sum;
        unsigned pos = cpre + icnt - cnt;
#pragma unroll
        for (unsigned k = 0; k < RPT; k++) {
            if (len[k]) {
                const uint32_t e = run < row0 ? 0u : uint32_t(minu(run - row0 + 1, 0xFFFFFFFFull));
                s_st[pos] = e;
                s_val[pos] = val[k];
                if (e - 1u < kRleRows) atomicOr(&s_bits[(e - 1u) >> 5], 1u << ((e - 1u) & 31u));
                pos++;
            }
            run += len[k];
        }
        __syncthreads();
        const uint64_t tile_end = t + 1 < ntiles ? tile_first[t + 1] : n;
        const uint64_t a = maxu(row0, tile_first[t]), b = minu(row1, tile_end);
        if (a < b) {
            const uint32_t ra = uint32_t(a - row0), rb = uint32_t(b - row0);
            const uint32_t tw0 = ra >> 5, tw1 = (rb + 31) >> 5;
            // the words split evenly over the warps
            const uint32_t per = (tw1 - tw0 + NWP - 1) / NWP;
            const uint32_t u0 = tw0 + wid * per, u1 = min(tw1, u0 + per);
            if (u0 < u1) {
                unsigned lo = 0, hi = kept;  // runs with entry <= 32 u0
                while (lo < hi) {
                    const unsigned mid = (lo + hi) >> 1;
                    if (s_st[mid] > 32 * u0) hi = mid;
                    else lo = mid + 1;
                }
                unsigned before = lo - 1u;  // index of the run holding row 32 u0 - 1 (wraps for none)
                uint64_t *const o = out + row0 + lane;
                for (uint32_t u = u0; u < u1; u++) {
                    const unsigned bits = s_bits[u];
                    const uint32_t r = 32 * u + lane;
                    if (r >= ra && r < rb) o[32 * u] = s_val[min(before + __popc(bits & incl), kept - 1)];
                    before += __popc(bits);
                }
            }
        }
        __syncthreads();
    }
    // the run lengths must add up to the column's length
    if (blockIdx.x == 0 && threadIdx.x == 0 && *total_rows != n) atomicOr(err, kErrCorrupt);
}

// One-pass decoder for short runs (mean length <= kRleLbMaxMean): a CTA takes
// the next tile of kRleLbTile runs from a ticket counter, stages its pairs in
// shared memory (cp.async), scans the lengths, compacts the non-empty runs to
// (value, start within the tile), publishes the tile's row count and finds the
// rows before it by the same decoupled look-back as the encoder (warp 0),
// then writes the tile's rows in windows of kRleLbWin rows through per-32-row
// bitmaps of run starts.  Each pair is read once (the two-pass decoder reads
// every pair twice, which for runs of one row is 32 B read per 8 B written).
// Shared-memory pairs sit at slot i + i / 8, so that the threads' runs
// (eight consecutive per thread) fall in different banks.  Writes stop at row
// n whatever the lengths say; lengths that do not add up to n are reported by
// the last tile (kErrCorrupt).  Needs 16-byte aligned pairs.
constexpr unsigned kRleLbThreads = 512, kRleLbRpt = 8;
constexpr unsigned kRleLbTile = kRleLbThreads * kRleLbRpt;  // runs per tile
constexpr unsigned kRleLbWin = 8192;                        // rows per write window
constexpr uint64_t kRleLbMaxMean = 4;
__host__ __device__ constexpr unsigned rle_lb_slot(unsigned i) { return i + (i >> 3); }

__global__ void __launch_bounds__(kRleLbThreads, 2) k_rle_expand_lb(const uint64_t *__restrict__ pairs,
                                                                   uint64_t runs, uint64_t n, RleTileState *state,
                                                                   unsigned *ticket, uint64_t *__restrict__ out,
                                                                   unsigned *err) {
    constexpr unsigned NW = kRleLbThreads / 32, NWD = kRleLbWin / 32;
    extern __shared__ __align__(128) uint8_t rle_smem[];
    // the tile's pairs, then (value, start within the tile) of its non-empty runs
    ulonglong2 *const s_p = reinterpret_cast<ulonglong2 *>(rle_smem);
    __shared__ unsigned s_bits[NWD];
    __shared__ uint64_t s_wsum[NW];
    __shared__ unsigned s_wcnt[NW];
    __shared__ uint64_t s_tile, s_base;
    const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const unsigned incl = (2u << lane) - 1u;  // lanes 0..lane
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t ntiles = (runs + kRleLbTile - 1) / kRleLbTile;
    if (tile >= ntiles) return;
    const uint64_t rb = tile * kRleLbTile;
    const unsigned nr = unsigned(minu(kRleLbTile, runs - rb));
    for (unsigned q = threadIdx.x; q < nr; q += kRleLbThreads) cp_async16(s_p + rle_lb_slot(q), pairs + 2 * (rb + q));
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    // this thread's kRleLbRpt consecutive runs: scans of lengths and of non-empty runs
    const unsigned j0 = threadIdx.x * kRleLbRpt;
    uint64_t len[kRleLbRpt], val[kRleLbRpt], sum = 0;
    unsigned cnt = 0;
#pragma unroll
    for (unsigned k = 0; k < kRleLbRpt; k++) {
        const ulonglong2 pr = j0 + k < nr ? s_p[rle_lb_slot(j0 + k)] : make_ulonglong2(0, 0);
        val[k] = pr.x;
        len[k] = pr.y;
        sum += len[k];
        cnt += len[k] != 0;
    }
    uint64_t isum = sum;
    unsigned icnt = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, isum, d);
        const unsigned co = __shfl_up_sync(0xFFFFFFFFu, icnt, d);
        if (int(lane) >= d) {
            isum += o;
            icnt += co;
        }
    }
    if (lane == 31) {
        s_wsum[wid] = isum;
        s_wcnt[wid] = icnt;
    }
    __syncthreads();  // every thread has its pairs in registers: s_p may be overwritten
    uint64_t ws = lane < NW ? s_wsum[lane] : 0;
    unsigned wc = lane < NW ? s_wcnt[lane] : 0;
#pragma unroll
    for (int d = 1; d < int(NW); d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, ws, d);
        const unsigned co = __shfl_up_sync(0xFFFFFFFFu, wc, d);
        if (int(lane) >= d) {
            ws += o;
            wc += co;
        }
    }
    const uint64_t agg = __shfl_sync(0xFFFFFFFFu, ws, NW - 1);  // the tile's rows
    const unsigned kept = __shfl_sync(0xFFFFFFFFu, wc, NW - 1);
    const uint64_t st0 = (wid ? __shfl_sync(0xFFFFFFFFu, ws, wid - 1) : 0) + isum - sum;  // my first run's start
    {
        unsigned pos = (wid ? __shfl_sync(0xFFFFFFFFu, wc, wid - 1) : 0) + icnt - cnt;
        uint64_t run = st0;
#pragma unroll
        for (unsigned k = 0; k < kRleLbRpt; k++) {
            if (len[k]) s_p[rle_lb_slot(pos++)] = make_ulonglong2(val[k], run);
            run += len[k];
        }
    }
    // publish the tile's rows, then the rows before it
    RleTileState *me = state + tile;
    if (threadIdx.x == 0 && tile > 0) rle_publish(me, kRleFlagAgg, agg, kRleNone);
    if (wid == 0) {
        uint64_t excl = 0, unused = kRleNone;
        if (tile > 0 && !rle_lookback(state, tile, excl, unused) && lane == 0) atomicOr(err, kErrTimeout);
        if (lane == 0) {
            rle_publish(me, kRleFlagInc, excl + agg, kRleNone);
            s_base = excl;
            if (tile == ntiles - 1 && excl + agg != n) atomicOr(err, kErrCorrupt);
        }
    }
    __syncthreads();
    const uint64_t base = s_base;
    if (base >= n) return;
    const uint64_t rows = minu(agg, n - base);  // never past row n
    for (uint64_t w0 = 0; w0 < rows; w0 += kRleLbWin) {
        for (unsigned w = threadIdx.x; w < NWD; w += kRleLbThreads) s_bits[w] = 0;
        __syncthreads();
        {
            // this thread's run starts in the window, one OR per bitmap word
            uint64_t s = st0;
            unsigned cw = ~0u, acc = 0;
#pragma unroll
            for (unsigned k = 0; k < kRleLbRpt; k++) {
                const uint64_t o = s - w0;  // start within the window (wraps when before it)
                if (len[k] && o < kRleLbWin) {
                    const unsigned wi = unsigned(o >> 5);
                    if (wi != cw) {
                        if (acc) atomicOr(&s_bits[cw], acc);
                        cw = wi;
                        acc = 0;
                    }
                    acc |= 1u << (o & 31u);
                }
                s += len[k];
            }
            if (acc) atomicOr(&s_bits[cw], acc);
        }
        __syncthreads();
        const unsigned wr = unsigned(minu(kRleLbWin, rows - w0));
        const unsigned nwd = (wr + 31) / 32, per = (nwd + NW - 1) / NW;
        const unsigned u0 = wid * per, u1 = min(nwd, u0 + per);
        if (u0 < u1) {
            unsigned lo = 0, hi = kept;  // runs starting before the warp's first row
            const uint64_t r0 = w0 + 32ull * u0;
            while (lo < hi) {
                const unsigned mid = (lo + hi) >> 1;
                if (s_p[rle_lb_slot(mid)].y < r0) lo = mid + 1;
                else hi = mid;
            }
            unsigned before = lo - 1u;  // index of the run holding the row before (wraps for none)
            uint64_t *const o = out + base + w0 + lane;
            for (unsigned u = u0; u < u1; u++) {
                const unsigned bits = s_bits[u];
                if (32 * u + lane < wr) o[32 * u] = s_p[rle_lb_slot(min(before + __popc(bits & incl), kept - 1))].x;
                before += __popc(bits);
            }
        }
        __syncthreads();
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
static int encode_rle(const uint64_t *d_in, uint64_t n, ms_col *out, ms_arena *a, cudaStream_t st) {
    // tile states for the smaller of the two encoders' tiles
    const uint64_t tiles = (n + minu(kRleEncTile, kRleStTile) - 1) / minu(kRleEncTile, kRleStTile);
    uint8_t *data = arena_take_t<uint8_t>(a, 16 * n + 64);
    RleTileState *state = arena_take_t<RleTileState>(a, tiles + 1);
    unsigned *ticket = arena_take_t<unsigned>(a, 2);
    uint64_t *d_runs = arena_take_t<uint64_t>(a, 1);
    if (!data || !state || !ticket || !d_runs) return ms_fail(MS_ERR_NOMEM, "arena exhausted (rle)");
    uint64_t runs = 0;
    if (n) {
        MS_CUDA_TRY(cudaMemsetAsync(state, 0, sizeof(RleTileState) * tiles, st));
        MS_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
        if ((reinterpret_cast<uintptr_t>(d_in) & 15u) == 0) {
            // rows staged in shared memory (16-byte aligned input)
            constexpr size_t smem = size_t(kRleStTile) * 8;
            MS_CUDA_TRY(cudaFuncSetAttribute(k_rle_encode_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(smem)));
            k_rle_encode_staged<<<unsigned((n + kRleStTile - 1) / kRleStTile), kRleStThreads, smem, st>>>(
                d_in, n, state, ticket, (uint64_t *)data, d_runs, a->d_err);
        } else {
            k_rle_encode<<<unsigned((n + kRleEncTile - 1) / kRleEncTile), kRleEncThreads, 0, st>>>(
                d_in, n, state, ticket, (uint64_t *)data, d_runs, a->d_err);
        }
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY(cudaMemcpyAsync(&runs, d_runs, 8, cudaMemcpyDeviceToHost, st));
        int rc = read_err(a, st);  // synchronises the stream
        if (rc) return rc;
    }
    *out = ms_col{};
    out->format = MS_FMT_RLE;
    out->count_values = n;
    out->size_used_byte = 16 * runs;
    out->size_compr_byte = 16 * runs;
    out->size_alloc_byte = 16 * n + 64;
    out->data = data;
    return MS_OK;
}

static int decode_rle(const ms_col *in, uint64_t *d_out, ms_arena *a, cudaStream_t st) {
    const uint64_t runs = in->size_used_byte / 16, n = in->count_values;
    if (!n) return MS_OK;
    if (!runs) return ms_fail(MS_ERR_CORRUPT, "rle column with values but no runs");
    if (n <= kRleLbMaxMean * runs && (reinterpret_cast<uintptr_t>(in->data) & 15u) == 0) {
        // short runs: one pass with a look-back
        const uint64_t tiles = (runs + kRleLbTile - 1) / kRleLbTile;
        RleTileState *state = arena_take_t<RleTileState>(a, tiles + 1);
        unsigned *ticket = arena_take_t<unsigned>(a, 2);
        if (!state || !ticket) return ms_fail(MS_ERR_NOMEM, "arena exhausted (rle decode)");
        MS_CUDA_TRY(cudaMemsetAsync(state, 0, sizeof(RleTileState) * tiles, st));
        MS_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
        constexpr size_t smem = size_t(rle_lb_slot(kRleLbTile)) * 16;
        MS_CUDA_TRY(cudaFuncSetAttribute(k_rle_expand_lb, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        k_rle_expand_lb<<<unsigned(tiles), kRleLbThreads, smem, st>>>((const uint64_t *)in->data, runs, n, state,
                                                                      ticket, d_out, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        return MS_OK;
    }
    const unsigned tr = rle_tile_runs(n, runs);
    const uint64_t tiles = (runs + tr - 1) / tr;
    uint64_t *trows = arena_take_t<uint64_t>(a, tiles + 1);
    uint64_t *tfirst = arena_take_t<uint64_t>(a, tiles + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 1);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(tiles, 1));
    if (!trows || !tfirst || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (rle decode)");
    const uint64_t *pairs = (const uint64_t *)in->data;
    k_rle_tile_rows<<<unsigned(tiles), kRleThreads, 0, st>>>(pairs, runs, tr, trows);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint64_t, 1>(trows, tiles, tfirst, tot, scr, st)));
    const uint64_t chunks = (n + kRleRows - 1) / kRleRows;
    uint32_t *ctile = arena_take_t<uint32_t>(a, chunks + 1);
    if (!ctile) return ms_fail(MS_ERR_NOMEM, "arena exhausted (rle decode)");
    k_rle_chunk_tiles<<<unsigned(minu((chunks + 255) / 256, uint64_t(persistent_grid(256, 4)))), 256, 0, st>>>(
        tfirst, tiles, chunks, ctile);
    MS_CUDA_TRY(cudaGetLastError());
    switch (tr / kRleThreads) {
    case 1: k_rle_expand<1><<<unsigned(chunks), kRleThreads, 0, st>>>(pairs, runs, tfirst, tiles, ctile, tot, n, d_out, a->d_err); break;
    case 2: k_rle_expand<2><<<unsigned(chunks), kRleThreads, 0, st>>>(pairs, runs, tfirst, tiles, ctile, tot, n, d_out, a->d_err); break;
    case 4: k_rle_expand<4><<<unsigned(chunks), kRleThreads, 0, st>>>(pairs, runs, tfirst, tiles, ctile, tot, n, d_out, a->d_err); break;
    default: k_rle_expand<8><<<unsigned(chunks), kRleThreads, 0, st>>>(pairs, runs, tfirst, tiles, ctile, tot, n, d_out, a->d_err); break;
    }
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// Shared encoder: `ncompr` rows (a block multiple) go to the compressed part
// with page layout L, rows [ncompr, n) to the uncompressed rest.
static int encode(const uint64_t *d_in, uint64_t n, uint64_t ncompr, Layout L, ms_col *out, ms_arena *a,
                  cudaStream_t st) {
    const int fmt = L.fmt;
    const uint64_t nb = ncompr / kBlock;
    const uint64_t cap = ms_size_max_byte_any_len(fmt, L.bw, n);
    uint8_t *data = arena_take_t<uint8_t>(a, cap);
    uint64_t *d_compr = arena_take_t<uint64_t>(a, 1);
    uint64_t *index = nullptr, *aux = nullptr;
    uint32_t *bws = nullptr;
    uint64_t *prefix = nullptr, *tot = nullptr, *scr = nullptr, *refs = nullptr;
    if (!data || !d_compr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (encode)");
    const unsigned grid = persistent_grid(256, 8);
    if (fmt != MS_FMT_STATIC_VBP && nb) {
        index = arena_take_t<uint64_t>(a, nb + 1);
        bws = arena_take_t<uint32_t>(a, nb + 1);
        prefix = arena_take_t<uint64_t>(a, nb + 1);
        tot = arena_take_t<uint64_t>(a, 1);
        scr = arena_take_t<uint64_t>(a, scan_scratch_words(nb, 1));
        if (fmt == MS_FMT_FOR_DVBP) aux = refs = arena_take_t<uint64_t>(a, nb / 2 + 1);
        if (!index || !bws || !prefix || !tot || !scr || (fmt == MS_FMT_FOR_DVBP && !refs))
            return ms_fail(MS_ERR_NOMEM, "arena exhausted (encode scratch)");
        if (fmt == MS_FMT_DYNAMIC_VBP) k_analyze_blocks<MS_FMT_DYNAMIC_VBP><<<grid, 256, 0, st>>>(d_in, nb, bws);
        else if (fmt == MS_FMT_DELTA_DVBP) k_analyze_blocks<MS_FMT_DELTA_DVBP><<<grid, 256, 0, st>>>(d_in, nb, bws);
        else k_analyze_for<<<grid, 256, 0, st>>>(d_in, nb / 2, bws, refs);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(bws, nb, prefix, tot, scr, st)));
    }
    if (nb) {
        switch (fmt) {
        case MS_FMT_STATIC_VBP:
            k_pack<MS_FMT_STATIC_VBP><<<grid, 256, 0, st>>>(d_in, nb, L, bws, prefix, refs, data, index, a->d_err);
            break;
        case MS_FMT_DYNAMIC_VBP:
            k_pack<MS_FMT_DYNAMIC_VBP><<<grid, 256, 0, st>>>(d_in, nb, L, bws, prefix, refs, data, index, a->d_err);
            k_headers_dvbp<<<grid, 256, 0, st>>>(nb, L, bws, prefix, data);
            break;
        case MS_FMT_DELTA_DVBP:
            k_pack<MS_FMT_DELTA_DVBP><<<grid, 256, 0, st>>>(d_in, nb, L, bws, prefix, refs, data, index, a->d_err);
            k_headers_casc<MS_FMT_DELTA_DVBP><<<grid, 256, 0, st>>>(nb, L, bws, prefix, refs, data);
            break;
        case MS_FMT_FOR_DVBP:
            k_pack<MS_FMT_FOR_DVBP><<<grid, 256, 0, st>>>(d_in, nb, L, bws, prefix, refs, data, index, a->d_err);
            k_headers_casc<MS_FMT_FOR_DVBP><<<grid, 256, 0, st>>>(nb, L, bws, prefix, refs, data);
            break;
        }
        MS_CUDA_TRY(cudaGetLastError());
    }
    k_finish_sizes<<<1, 32, 0, st>>>(nb, L, bws, prefix, d_compr);
    MS_CUDA_TRY(cudaGetLastError());
    const uint64_t nrest = n - ncompr;
    if (nrest) {
        k_copy_rest<<<(unsigned)minu((nrest + 255) / 256, 1024), 256, 0, st>>>(d_in + ncompr, nrest, fmt, L.bw,
                                                                                     d_compr, data);
        MS_CUDA_TRY(cudaGetLastError());
    }
    uint64_t compr = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&compr, d_compr, 8, cudaMemcpyDeviceToHost, st));
    int rc = read_err(a, st);  // synchronises
    if (rc) return rc;
    *out = ms_col{};
    out->format = uint32_t(fmt);
    out->bw = fmt == MS_FMT_STATIC_VBP ? L.bw : 0;
    out->count_values = n;
    out->size_compr_byte = compr;
    out->size_used_byte = nrest ? rest_offset(fmt, L.bw, compr) + 8 * nrest : compr;
    out->size_alloc_byte = cap;
    out->data = data;
    out->index = index;
    out->index_aux = aux;
    out->n_index = index ? nb : 0;
    return MS_OK;
}

int compress_values(const uint64_t *d_in, uint64_t n, int fmt, unsigned bw, ms_col *out, ms_arena *a,
                    cudaStream_t st) {
    if (fmt == MS_FMT_RLE) return encode_rle(d_in, n, out, a, st);
    if (fmt == MS_FMT_UNCOMPR) {
        uint64_t *data = arena_take_t<uint64_t>(a, n + 1);
        if (!data) return ms_fail(MS_ERR_NOMEM, "arena exhausted (copy)");
        if (n) MS_CUDA_TRY(cudaMemcpyAsync(data, d_in, 8 * n, cudaMemcpyDeviceToDevice, st));
        *out = ms_col{};
        out->format = MS_FMT_UNCOMPR;
        out->count_values = n;
        out->size_used_byte = 8 * n;
        out->size_alloc_byte = 8 * n;
        out->data = data;
        return MS_OK;
    }
    if (fmt == MS_FMT_STATIC_VBP && (bw < 1 || bw > 64)) return ms_fail(MS_ERR_INVALID, "static_vbp bw must be 1..64");
    if (fmt < 0 || fmt > MS_FMT_RLE) return ms_fail(MS_ERR_INVALID, "unknown format");
    const uint64_t b = block_size(fmt);
    Layout L{fmt, bw, kPageBlocks, kForPageBlocks};
    return encode(d_in, n, n / b * b, L, out, a, st);
}

int write_values(const uint64_t *d_vals, uint64_t n_vec, uint64_t n_scalar, int fmt, unsigned bw, ms_col *out,
                 ms_arena *a, cudaStream_t st) {
    const uint64_t n = n_vec + n_scalar;
    if (fmt == MS_FMT_UNCOMPR) {
        // uncompr write iterator: the values as they are (uncompr.h:126-237)
        *out = ms_col{};
        out->format = MS_FMT_UNCOMPR;
        out->count_values = n;
        out->size_used_byte = 8 * n;
        out->size_alloc_byte = 8 * n;
        out->data = const_cast<uint64_t *>(d_vals);
        return MS_OK;
    }
    if (fmt == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "rle_f has no write iterator");
    if (fmt == MS_FMT_STATIC_VBP && (bw < 1 || bw > 64)) return ms_fail(MS_ERR_INVALID, "static_vbp bw must be 1..64");
    if (fmt < 0 || fmt > MS_FMT_RLE) return ms_fail(MS_ERR_INVALID, "unknown format");
    const uint64_t b = block_size(fmt);
    const uint64_t full = n_vec / kWiBuffer * kWiBuffer;
    const uint64_t ncompr = full + (n_vec - full) / b * b;
    Layout L{fmt, bw, kWiBuffer / kBlock, kWiBuffer / kCascBlock};
    return encode(d_vals, n, ncompr, L, out, a, st);
}

int decompress_to(const ms_col *in, uint64_t *d_out, ms_arena *a, cudaStream_t st) {
    if (in->format == MS_FMT_RLE) return decode_rle(in, d_out, a, st);
    ColView v;
    int rc = prepare_view(in, a, st, &v);
    if (rc) return rc;
    if (!v.n) return MS_OK;
    const uint64_t nbt = v.nblocks_total();
    const unsigned grid = (unsigned)minu((nbt + 7) / 8, persistent_grid(256, 8));
    k_decode_all<<<grid, 256, 0, st>>>(v, d_out, a->d_err);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

}  // namespace ms

extern "C" int ms_gpu_morph(const ms_col *src, int dst_format, unsigned dst_bw, ms_col *out, ms_arena *a,
                            void *stream) {
    using namespace ms;
    if (!src || !out || !a) return ms_fail(MS_ERR_INVALID, "morph: null argument");
    int rc = check_col(src, false);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // morph from a format to itself returns the input (morph.h:133-160)
    if (int(src->format) == dst_format && (dst_format != MS_FMT_STATIC_VBP || src->bw == dst_bw)) {
        *out = *src;
        return MS_OK;
    }
    if (src->format == MS_FMT_UNCOMPR)
        return compress_values((const uint64_t *)src->data, src->count_values, dst_format, dst_bw, out, a, st);
    // decompress (possibly followed by a compress into another format)
    uint64_t *tmp = arena_take_t<uint64_t>(a, src->count_values + 1);
    if (!tmp) return ms_fail(MS_ERR_NOMEM, "arena exhausted (morph)");
    rc = decompress_to(src, tmp, a, st);
    if (rc) return rc;
    if (dst_format == MS_FMT_UNCOMPR) {
        rc = read_err(a, st);
        if (rc) return rc;
        *out = ms_col{};
        out->format = MS_FMT_UNCOMPR;
        out->count_values = src->count_values;
        out->size_used_byte = 8 * src->count_values;
        out->size_alloc_byte = 8 * src->count_values;
        out->data = tmp;
        return MS_OK;
    }
    return compress_values(tmp, src->count_values, dst_format, dst_bw, out, a, st);
}
