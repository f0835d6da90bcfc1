// sps_tma.cuh -- the fused select -> project -> agg_sum pipeline with the
// compressed blocks staged through shared memory by bulk copies (TMA).
//
// One persistent CTA per SM: warp 0 is the producer, warps 1..W consume.
// Each CTA owns a contiguous range of 512-row blocks.  The producer groups
// consecutive blocks into tiles whose x and y byte ranges (the packed blocks
// plus any page headers between them, contiguous in memory) fit one stage
// buffer, records every block's shared-memory offset and bit width in the
// stage descriptor and issues one 1-D cp.async.bulk per column, completing on
// the stage's `full` mbarrier.  Consumer warps decode their blocks of the
// tile from shared memory (one warp per block, 16 values per thread, as in
// colview.cuh), evaluate the predicate on x, add up y where it holds, and
// arrive on the stage's `empty` mbarrier.  S stages keep S tiles in flight
// per SM, which is what hides HBM latency: the direct-load kernel keeps only
// the few KB its resident warps have requested.
//
// Rows in the uncompressed rests (and blocks past either column's
// compressed part) are handled after the pipeline with the direct decoder.
// All waits are bounded; a timeout records kErrTimeout and the kernel
// leaves after the producer has waited for its own copies.
#pragma once

#include "fastpath.cuh"
#include "internal.h"
#include "stream.cuh"
#include "tma.cuh"

namespace ms {

constexpr unsigned kMaxTile = 32;  // blocks per tile (one producer lane each)

struct TmaCfg {
    unsigned stages;
    unsigned stage_bytes;
    unsigned max_tile;
};

// One launcher per consumer-warp count, each in its own translation unit
// (sps_tma_w<W>.cu) so that the instantiations compile in parallel.
#define MS_SPS_TMA_LAUNCHER(Wn)                                                                                 \
    int sps_tma_launch_w##Wn(const ColView &x, const ColView &y, bool has_y, int cmp, uint64_t val,            \
                             const TmaCfg &cfg, unsigned vpt, uint64_t *d_sum, uint64_t *d_cnt, unsigned *d_err, \
                             unsigned grid, cudaStream_t st)
MS_SPS_TMA_LAUNCHER(4);
MS_SPS_TMA_LAUNCHER(8);
MS_SPS_TMA_LAUNCHER(12);
MS_SPS_TMA_LAUNCHER(16);
MS_SPS_TMA_LAUNCHER(20);
MS_SPS_TMA_LAUNCHER(24);

namespace {

struct StageDesc {
    uint64_t b0;
    unsigned nblk;
    unsigned pad;
};

template <int W, bool kHasY, bool kFast, int VPT>
__global__ void __launch_bounds__(32 * (W + 1), 1)
    k_sps_tma(ColView x, ColView y, StreamCol xs, StreamCol ys, int cmp, uint64_t val, Pred pred, TmaCfg cfg,
              unsigned long long *__restrict__ d_sum, unsigned long long *__restrict__ d_cnt, unsigned *err) {
    extern __shared__ __align__(128) uint8_t smem[];
    const unsigned S = cfg.stages, SB = cfg.stage_bytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + S;
    StageDesc *desc = reinterpret_cast<StageDesc *>(empty + S);
    uint32_t *xoff = reinterpret_cast<uint32_t *>(desc + S);  // [S][kMaxTile]
    uint32_t *yoff = xoff + S * kMaxTile;
    uint8_t *xbw = reinterpret_cast<uint8_t *>(yoff + S * kMaxTile);
    uint8_t *ybw = xbw + S * kMaxTile;
    uint8_t *ring = smem + align_up(uint64_t(16) * S + sizeof(StageDesc) * S + 10 * S * kMaxTile, 128);

    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) {
        for (unsigned s = 0; s < S; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, W);
        }
        mbar_fence_init();
    }
    __syncthreads();

    const uint64_t nbs = minu(xs.nb, kHasY ? ys.nb : xs.nb);
    const uint64_t b_lo = nbs * blockIdx.x / gridDim.x, b_hi = nbs * (blockIdx.x + 1) / gridDim.x;
    bool ok = true;
    uint64_t s_sum = 0, s_cnt = 0;

    if (warp == 0) {
        // ---------------- producer ----------------
        uint64_t b = b_lo;
        unsigned t = 0;  // tiles issued
        for (;; t++) {
            const unsigned st = t % S, use = t / S;
            // the next tile's block locations are requested before waiting
            // for its stage, so the index loads overlap the wait
            const uint64_t blk = b + lane;
            const bool valid = blk < b_hi && lane < cfg.max_tile;
            uint64_t xo = 0, yo = 0;
            unsigned xw = 0, yw = 0;
            if (valid) {
                blk_loc(xs, blk, xo, xw);
                if (kHasY) blk_loc(ys, blk, yo, yw);
            }
            if (use > 0 && !mbar_wait(empty + st, (use - 1) & 1u)) {
                ok = false;
                break;
            }
            if (b >= b_hi) {  // sentinel: no more tiles
                if (lane == 0) {
                    desc[st].nblk = 0;
                    mbar_arrive(full + st);
                }
                t++;
                break;
            }
            const uint64_t x0 = __shfl_sync(0xFFFFFFFFu, xo, 0), y0 = __shfl_sync(0xFFFFFFFFu, yo, 0);
            const uint64_t xlen = valid ? xo + 64ull * xw - x0 : 0;
            const uint64_t ylen = valid ? yo + 64ull * yw - y0 : 0;
            const bool fits = valid && align_up(xlen, 128) + ylen <= SB;
            const unsigned T = __popc(__ballot_sync(0xFFFFFFFFu, fits));
            if (T == 0) {  // a single block larger than a stage: configuration error
                if (lane == 0) atomicOr(err, kErrCapacity);
                ok = false;
                if (lane == 0) {
                    desc[st].nblk = 0;
                    mbar_arrive(full + st);
                }
                t++;
                break;
            }
            const uint64_t xl = __shfl_sync(0xFFFFFFFFu, xlen, T - 1);
            const uint64_t yl = __shfl_sync(0xFFFFFFFFu, ylen, T - 1);
            const uint32_t ybase = uint32_t(align_up(xl, 128));
            if (lane < T) {
                xoff[st * kMaxTile + lane] = st * SB + uint32_t(xo - x0);
                xbw[st * kMaxTile + lane] = uint8_t(xw);
                if (kHasY) {
                    yoff[st * kMaxTile + lane] = st * SB + ybase + uint32_t(yo - y0);
                    ybw[st * kMaxTile + lane] = uint8_t(yw);
                }
            }
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                desc[st].b0 = b;
                desc[st].nblk = T;
                __threadfence_block();
                mbar_arrive_expect_tx(full + st, unsigned(xl + (kHasY ? yl : 0)));
                bulk_g2s(ring + st * SB, xs.base + x0, unsigned(xl), full + st);
                if (kHasY) bulk_g2s(ring + st * SB + ybase, ys.base + y0, unsigned(yl), full + st);
            }
            __syncwarp();
            b += T;
        }
        // wait for every copy this warp issued (bounded) before leaving
        const unsigned issued = t;
        for (unsigned s = 0; s < S && s < issued; s++) {
            const unsigned last_use = (issued - 1 - s) / S;  // uses of stage s = ceil((issued - s) / S)
            (void)last_use;
            const unsigned uses = (issued - s + S - 1) / S;
            if (!mbar_wait(full + s, (uses - 1) & 1u)) ok = false;
        }
    } else {
        // ---------------- consumers ----------------
        const unsigned cw = warp - 1, l = lane & 7u, q = lane >> 3;
        for (unsigned t = 0;; t++) {
            const unsigned st = t % S, use = t / S;
            if (!mbar_wait(full + st, use & 1u)) {
                ok = false;
                break;
            }
            const unsigned T = desc[st].nblk;
            if (T == 0) break;
            const uint64_t b0 = desc[st].b0;
            // blocks are dealt to warps round-robin across tiles, so a tile size
            // that is not a multiple of W does not load one warp systematically
            const unsigned j0 = unsigned((cw + W - (b0 - b_lo) % W) % W);
            if (kFast && VPT == 32) {
                // two blocks per warp, one per half-warp, 32 values per thread;
                // pairs of blocks are dealt to warps round-robin
                bool bad = false;
                const uint64_t base = b0 - b_lo;
                const unsigned hb = lane >> 4, h = (lane >> 3) & 1u;
                const uint64_t p_lo = base >> 1, p_hi = (base + T - 1) >> 1;
                for (uint64_t P = p_lo + (cw + W - p_lo % W) % W; P <= p_hi; P += W) {
                    const int64_t jj = int64_t(2 * P + hb) - int64_t(base);
                    const bool act = jj >= 0 && jj < int64_t(T);
                    const unsigned j = act ? unsigned(jj) : 0;
                    if (act) {
                        // selection flags of x, then the flagged values of y
                        uint32_t sel[32];
                        const uint64_t *xb = reinterpret_cast<const uint64_t *>(ring + xoff[st * kMaxTile + j]);
                        s_cnt += sel32_block_rt(xbw[st * kMaxTile + j], xb, l, h, pred, sel, bad);
                        if (kHasY)
                            s_sum += sum32_sel_rt(ybw[st * kMaxTile + j],
                                                  reinterpret_cast<const uint64_t *>(ring + yoff[st * kMaxTile + j]),
                                                  l, h, sel, bad);
                        else
                            s_sum += sum32_sel_rt(xbw[st * kMaxTile + j], xb, l, h, sel, bad);
                    }
                }
                ok &= !bad;
                __syncwarp();
                if (lane == 0) mbar_arrive(empty + st);
                continue;
            }
            if (kFast) {
                // plain vbp blocks: predicate and sum inside the bit-width switch
                bool bad = false;
                for (unsigned j = j0; j < T; j += W) {
                    const unsigned m = mask_block_rt(
                        xbw[st * kMaxTile + j], reinterpret_cast<const uint64_t *>(ring + xoff[st * kMaxTile + j]), l,
                        q, pred, bad);
                    s_cnt += __popc(m);
                    if (kHasY) {
                        if (__any_sync(0xFFFFFFFFu, m != 0))
                            s_sum += sum_block_rt(ybw[st * kMaxTile + j],
                                                  reinterpret_cast<const uint64_t *>(ring + yoff[st * kMaxTile + j]), l,
                                                  q, m, bad);
                    } else {
                        s_sum += sum_block_rt(xbw[st * kMaxTile + j],
                                              reinterpret_cast<const uint64_t *>(ring + xoff[st * kMaxTile + j]), l, q,
                                              m, bad);
                    }
                }
                ok &= !bad;
                __syncwarp();
                if (lane == 0) mbar_arrive(empty + st);
                continue;
            }
            for (unsigned j = j0; j < T; j += W) {
                const uint64_t blk = b0 + j;
                uint64_t v[16];
                const uint64_t xside = cascade_side(x, blk, l);
                ok &= vbp_decode16_rt<true>(xbw[st * kMaxTile + j],
                                            reinterpret_cast<const uint64_t *>(ring + xoff[st * kMaxTile + j]), l,
                                            q, v);
                apply_cascade(x, blk, l, q, v, xside);
                const unsigned m = select_mask(x, blk, l, q, v, 0xFFFFu, cmp, val);
                s_cnt += __popc(m);
                if (kHasY) {
                    if (__any_sync(0xFFFFFFFFu, m != 0)) {
                        uint64_t w[16];
                        const uint64_t yside = cascade_side(y, blk, l);
                        ok &= vbp_decode16_rt<true>(ybw[st * kMaxTile + j],
                                                    reinterpret_cast<const uint64_t *>(ring + yoff[st * kMaxTile + j]),
                                                    l, q, w);
                        apply_cascade(y, blk, l, q, w, yside);
#pragma unroll
                        for (int k = 0; k < 16; k++) s_sum += ((m >> k) & 1u) ? w[k] : 0;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 16; k++) s_sum += ((m >> k) & 1u) ? v[k] : 0;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + st);
        }
    }
    if (!ok) atomicOr(err, kErrTimeout);
#pragma unroll
    for (int sft = 16; sft > 0; sft >>= 1) {
        s_sum += __shfl_xor_sync(0xFFFFFFFFu, s_sum, sft);
        s_cnt += __shfl_xor_sync(0xFFFFFFFFu, s_cnt, sft);
    }
    if (lane == 0 && warp > 0) {
        if (d_sum) atomicAdd(d_sum, (unsigned long long)s_sum);
        if (d_cnt) atomicAdd(d_cnt, (unsigned long long)s_cnt);
    }
}

// Blocks outside the pipelined range (uncompressed rests, blocks past either
// column's compressed part): the direct decoder, one warp per block.
template <bool kHasY>
__global__ void __launch_bounds__(256) k_sps_tail(ColView x, ColView y, int cmp, uint64_t val, uint64_t b_begin,
                                                 unsigned long long *__restrict__ d_sum,
                                                 unsigned long long *__restrict__ d_cnt, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    const uint64_t nbt = x.nblocks_total();
    uint64_t s_sum = 0, s_cnt = 0;
    bool ok = true;
    for (uint64_t blk = b_begin + (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; blk < nbt;
         blk += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(x, blk, l, q, v, valid);
        const unsigned m = select_mask(x, blk, l, q, v, valid, cmp, val);
        s_cnt += __popc(m);
        if (kHasY) {
            if (__any_sync(0xFFFFFFFFu, m != 0)) {
                uint64_t w[16];
                unsigned vy;
                ok &= decode_block(y, blk, l, q, w, vy);
#pragma unroll
                for (int k = 0; k < 16; k++) s_sum += ((m >> k) & 1u) ? w[k] : 0;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 16; k++) s_sum += ((m >> k) & 1u) ? v[k] : 0;
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
#pragma unroll
    for (int sft = 16; sft > 0; sft >>= 1) {
        s_sum += __shfl_xor_sync(0xFFFFFFFFu, s_sum, sft);
        s_cnt += __shfl_xor_sync(0xFFFFFFFFu, s_cnt, sft);
    }
    if (lane == 0) {
        if (d_sum) atomicAdd(d_sum, (unsigned long long)s_sum);
        if (d_cnt) atomicAdd(d_cnt, (unsigned long long)s_cnt);
    }
}

template <int W, bool kHasY, bool kFast, int VPT>
int launch_tma3(const ColView &x, const ColView &y, int cmp, uint64_t val, const TmaCfg &cfg, uint64_t *d_sum,
                uint64_t *d_cnt, unsigned *d_err, unsigned grid, cudaStream_t st) {
    const size_t meta = align_up(16ull * cfg.stages + sizeof(StageDesc) * cfg.stages + 10ull * cfg.stages * kMaxTile, 128);
    const size_t shm = meta + size_t(cfg.stages) * cfg.stage_bytes;
    auto kern = k_sps_tma<W, kHasY, kFast, VPT>;
    MS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
    kern<<<grid, 32 * (W + 1), shm, st>>>(x, y, stream_of(x), stream_of(y), cmp, val, make_pred(cmp, val), cfg,
                                          (unsigned long long *)d_sum, (unsigned long long *)d_cnt, d_err);
    MS_CUDA_TRY(cudaGetLastError());
    const uint64_t nbs = minu(stream_of(x).nb, kHasY ? stream_of(y).nb : stream_of(x).nb);
    const uint64_t nbt = x.nblocks_total();
    if (nbt > nbs) {
        const unsigned tg = unsigned(minu((nbt - nbs + 7) / 8, uint64_t(sm_count()) * 4));
        k_sps_tail<kHasY><<<tg, 256, 0, st>>>(x, y, cmp, val, nbs, (unsigned long long *)d_sum,
                                              (unsigned long long *)d_cnt, d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    return MS_OK;
}

template <int W, bool kHasY>
int launch_tma(const ColView &x, const ColView &y, int cmp, uint64_t val, const TmaCfg &cfg, unsigned vpt,
               uint64_t *d_sum, uint64_t *d_cnt, unsigned *d_err, unsigned grid, cudaStream_t st) {
    if (plain(x) && (!kHasY || plain(y))) {
        if (vpt == 32) return launch_tma3<W, kHasY, true, 32>(x, y, cmp, val, cfg, d_sum, d_cnt, d_err, grid, st);
        return launch_tma3<W, kHasY, true, 16>(x, y, cmp, val, cfg, d_sum, d_cnt, d_err, grid, st);
    }
    return launch_tma3<W, kHasY, false, 16>(x, y, cmp, val, cfg, d_sum, d_cnt, d_err, grid, st);
}

}  // namespace
}  // namespace ms
