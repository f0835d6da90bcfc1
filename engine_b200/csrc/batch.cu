// batch.cu -- many columns, one persistent launch.
//
// A batch plan turns a set of columns (any format, any length) into a device
// work queue of items: up to 32 consecutive 512-row blocks of one column
// (static_vbp / dynamic_vbp, for_f, delta_f), up to 4096 rows of a column's
// uncompressed rest, or up to 1024 runs of an rle_f column.  Every column
// runs decompress -> select(value cmp c_i) -> agg_sum of the selected values
// (count and sum per column), the per-column chain of the reference's
// morph / select / agg_sum operators.
//
// The kernel is persistent (one or more CTAs per SM) and every warp works
// alone: it takes the next item off the queue with one atomic, and runs its
// own S-stage shared-memory ring -- lane 0 issues a 1-D bulk copy (TMA) of the
// next tile (the consecutive blocks of the item that fit a stage, page headers
// included) while the warp decodes the previous one.  Items of very different
// sizes and formats therefore need no cross-warp synchronisation, and a warp
// keeps S tiles in flight, which is what hides HBM latency.  Blocks are
// decoded as in the single-column kernels: plain vbp blocks compare and sum
// inside the bit-width switch, for_f adds the 1024-block reference, delta_f
// runs the lane-wise prefix with a carry kept in registers across the item's
// blocks; the carry into an item's first block is a per-item seek value the
// plan computes once (the values before the item, lane by lane), so items of
// one column are independent.  The queue is ordered by decoder (kind, bit
// width), so the warps of an SM mostly run the same instructions.
//
// All waits are bounded; errors go to the arena's error word.  The run is a
// fixed sequence of stream operations (three memsets and one launch) with no
// host synchronisation, so it can be captured into a CUDA graph; the plan
// keeps one graph per pair of output buffers.
#include <algorithm>
#include <vector>

#include "fastpath.cuh"
#include "internal.h"
#include "tma.cuh"

namespace ms {
namespace {

constexpr unsigned kBItemBlocks = 32;  // blocks per item (one lane each)
constexpr unsigned kBItemRest = 4096;  // rows of an uncompressed rest per item
constexpr unsigned kBItemRuns = 1024;  // runs of an rle_f column per item

enum : uint32_t { kItVbp = 0, kItFor = 1, kItDelta = 2, kItRest = 3, kItRle = 4 };

struct BCol {
    const uint8_t *data;    // compressed blocks (vbp family) or (value, length) pairs (rle_f)
    const uint64_t *index;  // block index (nullptr: static_vbp, fixed bw)
    const uint64_t *aux;    // for_f references per 1024-block
    const uint64_t *rest;   // uncompressed rest rows [n_compr, n)
    uint64_t n, n_compr, sfrom;
    uint64_t c;             // comparison constant
    Pred pred;              // c reduced to a threshold for plain vbp blocks
    unsigned bw;            // static_vbp width
    unsigned cf;            // comparison as bits: 1 = less passes, 2 = equal passes, 4 = negate
};

struct BItem {
    uint32_t col, kind;
    uint64_t start;       // first block / first rest row / first run
    uint32_t count, pad;  // blocks / rows / runs
    uint64_t seek;        // delta_f: carry slot; rle_f: first row of the item
};

struct BStage {  // one stage of a warp's ring
    uint32_t item, nblk;
    uint64_t b0;
    uint32_t off[kBItemBlocks];
    uint8_t bw[kBItemBlocks];
};

// The comparison without a branch on its kind: (lt & less-passes) |
// (eq & equal-passes), negated for greater / greaterequal.
inline unsigned cmp_flags(int cmp) {
    switch (cmp) {
    case MS_CMP_EQ: return 2u;
    case MS_CMP_LT: return 1u;
    case MS_CMP_LE: return 3u;
    case MS_CMP_GT: return 7u;
    default: return 5u;
    }
}

__device__ __forceinline__ bool cmp_bits(uint64_t v, uint64_t c, unsigned cf, bool sgn) {
    const bool lt = sgn ? (int64_t)v < (int64_t)c : v < c;
    const unsigned hit = ((lt ? 1u : 0u) | (v == c ? 2u : 0u)) & cf & 3u;
    return (hit ? 1u : 0u) ^ (cf >> 2);
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Threshold form of `base + d  cmp  c` (signed 64-bit, as the compressed
// part compares) for d in [0, range), range <= 2^32: a Pred on d.  False when
// base + [0, range) wraps or crosses the signed boundary -- then the order of
// d is not the order of the values and the caller compares 64-bit values.
__device__ __forceinline__ bool rel_pred(uint64_t base, uint64_t range, uint64_t c, int cmp, Pred &p) {
    const uint64_t hi = base + (range - 1);
    if (hi < base || ((int64_t)base < 0) != ((int64_t)hi < 0)) return false;
    const int64_t cs = (int64_t)c, bs = (int64_t)base;
    const uint64_t diff = uint64_t(cs) - uint64_t(bs);  // the true difference when cs >= bs
    const uint64_t nlt = cs <= bs ? 0 : minu(diff, range);
    const uint64_t nle = cs < bs ? 0 : (diff >= range ? range : diff + 1);
    p.cmp = cmp;
    p.val = c - base;
    p.is_eq = cmp == MS_CMP_EQ;
    p.T = (cmp == MS_CMP_LT || cmp == MS_CMP_GE) ? nlt : nle;
    p.flip = cmp == MS_CMP_GT || cmp == MS_CMP_GE;
    return true;
}

// A delta_f block of width BW <= 27 in 32-bit arithmetic: thread (l, q)
// decodes its 16 deltas, forms their running sums P_k (< 2^31), and the
// lane's values are base + P_k with base = carry + the sums of the lane's
// earlier quarters.  The comparison becomes a threshold on P_k (rel_pred)
// unless the thread's values cross the signed boundary; sums are cnt * base
// + the sum of the selected P_k.  Returns the lane's last value (the carry of
// the next block).
template <unsigned BW>
__device__ __forceinline__ uint64_t delta_block(const uint64_t *blk, unsigned l, unsigned q, uint64_t carry,
                                                uint64_t c, int cmp, unsigned cf, uint64_t &cnt, uint64_t &sum) {
    uint32_t P[16];
    vbp_decode16_u32<BW>(blk, l, q, P);
#pragma unroll
    for (int k = 1; k < 16; k++) P[k] += P[k - 1];
    const uint64_t tot = P[15];
    const uint64_t up = __shfl_up_sync(0xFFFFFFFFu, tot, 8);
    uint64_t pre = q >= 1 ? up : 0;
    const uint64_t up2 = __shfl_up_sync(0xFFFFFFFFu, tot + pre, 16);
    pre += q >= 2 ? up2 : 0;
    const uint64_t base = carry + pre;
    Pred pd;
    unsigned m = 0;
    if (rel_pred(base, uint64_t(P[15]) + 1, c, cmp, pd)) {
        if (pd.is_eq) {
            const bool in = pd.val < (uint64_t(1) << 32);
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(in && P[k] == uint32_t(pd.val)) << k;
        } else {
            const bool big = pd.T > 0xFFFFFFFFull;
#pragma unroll
            for (int k = 0; k < 16; k++) m |= unsigned(big || P[k] < uint32_t(pd.T)) << k;
            if (pd.flip) m ^= 0xFFFFu;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) m |= unsigned(cmp_bits(base + P[k], c, cf, true)) << k;
    }
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) s += ((m >> k) & 1u) ? P[k] : 0u;
    const unsigned n = __popc(m);
    cnt += n;
    sum += s + n * base;
    return __shfl_sync(0xFFFFFFFFu, base + P[15], int(24 + l));
}

// Generic delta_f block (any width): 64-bit decode and running sums.
__device__ __forceinline__ uint64_t delta_block_any(unsigned bw, const uint64_t *blk, unsigned l, unsigned q,
                                                    uint64_t carry, uint64_t c, unsigned cf, uint64_t &cnt,
                                                    uint64_t &sum, bool &bad) {
    uint64_t v[16];
    bad |= !vbp_decode16_rt<true>(bw, blk, l, q, v);
#pragma unroll
    for (int k = 1; k < 16; k++) v[k] += v[k - 1];
    const uint64_t tot = v[15];
    const uint64_t up = __shfl_up_sync(0xFFFFFFFFu, tot, 8);
    uint64_t pre = q >= 1 ? up : 0;
    const uint64_t up2 = __shfl_up_sync(0xFFFFFFFFu, tot + pre, 16);
    pre += (q >= 2 ? up2 : 0) + carry;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        v[k] += pre;
        const bool hit = cmp_bits(v[k], c, cf, true);
        cnt += hit;
        sum += hit ? v[k] : 0;
    }
    return __shfl_sync(0xFFFFFFFFu, v[15], int(24 + l));
}

#define MS_BW27(X)                                                                                      \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) \
    X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27)

__device__ __forceinline__ uint64_t delta_block_rt(unsigned bw, const uint64_t *blk, unsigned l, unsigned q,
                                                   uint64_t carry, uint64_t c, int cmp, unsigned cf, uint64_t &cnt,
                                                   uint64_t &sum, bool &bad) {
    switch (bw) {
#define MS_X(B) \
    case B: return delta_block<B>(blk, l, q, carry, c, cmp, cf, cnt, sum);
        MS_BW27(MS_X)
#undef MS_X
    default: return delta_block_any(bw, blk, l, q, carry, c, cf, cnt, sum, bad);
    }
}

__host__ __device__ inline unsigned bwarp_meta_bytes(unsigned S) {
    return (8u * S + unsigned(sizeof(BStage)) * S + 127u) / 128u * 128u;
}

template <int W>
__global__ void __launch_bounds__(32 * W, 1)
    k_batch(const BCol *__restrict__ cols, const BItem *__restrict__ items, uint64_t n_items,
            const uint64_t *__restrict__ seeks, unsigned S, unsigned SBw, unsigned long long *head,
            unsigned long long *__restrict__ out_cnt, unsigned long long *__restrict__ out_sum, unsigned *err) {
    extern __shared__ __align__(128) uint8_t smem[];
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    uint8_t *mine = smem + size_t(warp) * (bwarp_meta_bytes(S) + size_t(S) * SBw);
    uint64_t *bar = reinterpret_cast<uint64_t *>(mine);
    BStage *stg = reinterpret_cast<BStage *>(mine + 8u * S);
    uint8_t *ring = mine + bwarp_meta_bytes(S);
    if (lane == 0) {
        for (unsigned s = 0; s < S; s++) mbar_init(bar + s, 1);
        mbar_fence_init();
    }
    __syncwarp();

    bool ok = true, bad = false;
    // producer state
    bool exhausted = false;
    uint32_t it = 0, it_col = 0;
    uint64_t it_start = 0, it_next = 0, it_left = 0;
    uint64_t it_off = 0;  // lane i: byte offset of the item's block i
    unsigned it_bw = 0;   // lane i: its bit width
    const uint8_t *it_data = nullptr;
    unsigned issued = 0, consumed = 0;
    // consumer state: delta carry of lane l (threads (l, q) all hold it)
    uint64_t carry = 0;

    // Look-ahead: the next item is taken off the queue and its description
    // and block locations loaded one step per issued tile, so the chain of
    // dependent loads (queue atomic -> item -> column -> block index) overlaps
    // the current item's copies instead of stalling the warp between items.
    enum : unsigned { kLaNone = 0, kLaId = 1, kLaItem = 2, kLaCol = 3, kLaReady = 4, kLaEmpty = 5 };
    unsigned la = kLaNone;
    unsigned long long la_id = 0;  // lane 0 holds the atomic's result until it is broadcast
    BItem la_bi{};
    const uint64_t *la_index = nullptr;
    unsigned la_cbw = 0;
    const uint8_t *la_data = nullptr;
    uint64_t la_off = 0;
    unsigned la_bw = 0;
    auto la_step = [&]() {
        if (la == kLaNone) {
            if (lane == 0) la_id = atomicAdd(head, 1ull);
            la = kLaId;
        } else if (la == kLaId) {
            la_id = __shfl_sync(0xFFFFFFFFu, la_id, 0);
            if (la_id >= n_items) {
                la = kLaEmpty;
                return;
            }
            la_bi = items[la_id];
            la = kLaItem;
        } else if (la == kLaItem) {
            if (la_bi.kind <= kItDelta) {
                const BCol &c = cols[la_bi.col];
                la_index = c.index;
                la_cbw = c.bw;
                la_data = c.data;
            }
            la = kLaCol;
        } else if (la == kLaCol) {
            la_off = 0;
            la_bw = 0;
            if (la_bi.kind <= kItDelta && lane < la_bi.count) {
                if (la_index) {
                    const uint64_t e = __ldg(la_index + la_bi.start + lane);
                    la_off = idx_off(e);
                    la_bw = idx_bw(e);
                } else {
                    la_bw = la_cbw;
                    la_off = (la_bi.start + lane) * 64ull * la_cbw;
                }
            }
            la = kLaReady;
        }
    };

    auto issue = [&]() {
        if (it_left == 0) {
            while (la != kLaReady && la != kLaEmpty) la_step();  // finish the look-ahead if it is behind
            if (la == kLaEmpty) {
                exhausted = true;
                return;
            }
            it = uint32_t(la_id);
            const BItem bi = la_bi;
            it_col = bi.col;
            it_data = la_data;
            it_off = la_off;
            it_bw = la_bw;
            la = kLaNone;
            la_step();  // request the following item now
            if (bi.kind == kItRest || bi.kind == kItRle) {  // read in place: no copy
                const unsigned s = issued % S;
                if (lane == 0) {
                    stg[s].item = it;
                    stg[s].nblk = 0;
                    stg[s].b0 = bi.start;
                    mbar_arrive(bar + s);
                }
                __syncwarp();
                issued++;
                return;
            }
            it_start = it_next = bi.start;
            it_left = bi.count;
        } else if (la != kLaReady && la != kLaEmpty) {
            la_step();
        }
        const unsigned s = issued % S;
        const unsigned k0 = unsigned(it_next - it_start);  // first block of the tile within the item
        const bool valid = lane < it_left;
        const uint64_t off = __shfl_sync(0xFFFFFFFFu, it_off, (k0 + lane) & 31u);
        const unsigned bw = __shfl_sync(0xFFFFFFFFu, it_bw, (k0 + lane) & 31u);
        const uint64_t x0 = __shfl_sync(0xFFFFFFFFu, off, 0);
        const uint64_t len = valid ? off + 64ull * bw - x0 : 0;
        const bool fits = valid && bw >= 1 && bw <= 64 && len <= SBw;
        const unsigned fb = __ballot_sync(0xFFFFFFFFu, fits);
        const unsigned T = fb == 0xFFFFFFFFu ? 32u : unsigned(__ffs(~fb) - 1);  // leading lanes that fit
        if (T == 0) {  // corrupt width or a block larger than a stage: drop the item
            if (lane == 0) atomicOr(err, kErrCorrupt);
            it_left = 0;
            return;
        }
        const uint64_t tl = __shfl_sync(0xFFFFFFFFu, len, T - 1);
        if (lane < T) {
            stg[s].off[lane] = uint32_t(off - x0);
            stg[s].bw[lane] = uint8_t(bw);
        }
        if (lane == 0) {
            stg[s].item = it;
            stg[s].nblk = T;
            stg[s].b0 = it_next;
        }
        __syncwarp();
        if (lane == 0) {
            fence_proxy_async();  // the stage's previous contents were read through the generic proxy
            mbar_arrive_expect_tx(bar + s, unsigned(tl));
            bulk_g2s(ring + size_t(s) * SBw, it_data + x0, unsigned(tl), bar + s);
        }
        __syncwarp();
        it_next += T;
        it_left -= T;
        issued++;
    };

    for (;;) {
        while (!exhausted && issued - consumed < S) issue();
        if (consumed == issued) break;
        const unsigned s = consumed % S;
        if (!mbar_wait(bar + s, (consumed / S) & 1u)) {
            ok = false;
            break;
        }
        const BStage &sd = stg[s];
        const BItem bi = items[sd.item];
        const BCol &c = cols[bi.col];
        const uint8_t *base = ring + size_t(s) * SBw;
        uint64_t cnt = 0, sum = 0;
        if (bi.kind == kItVbp || bi.kind == kItFor) {
            // two blocks at a time, one per half-warp, 32 values per thread
            const unsigned hb = lane >> 4, h = (lane >> 3) & 1u;
            for (unsigned j0 = 0; j0 < sd.nblk; j0 += 2) {
                const unsigned j = j0 + hb;
                if (j >= sd.nblk) continue;  // the second half-warp when the tile has an odd count
                const uint64_t *blk = reinterpret_cast<const uint64_t *>(base + sd.off[j]);
                const unsigned bw = sd.bw[j];
                if (bi.kind == kItVbp) {
                    unsigned k = 0;
                    sum += self_sum32_block_rt(bw, blk, l, h, c.pred, k, bad);
                    cnt += k;
                    continue;
                }
                const uint64_t ref = __ldg(c.aux + ((sd.b0 + j) >> 1));
                Pred pd;
                if (bw <= 32 && rel_pred(ref, uint64_t(1) << bw, c.c, c.pred.cmp, pd)) {
                    // values ref + d: select and sum on d in the bit-width switch
                    unsigned k = 0;
                    const uint64_t sd_ = self_sum32_block_rt(bw, blk, l, h, pd, k, bad);
                    cnt += k;
                    sum += sd_ + uint64_t(k) * ref;
                } else {
                    // every row of the compressed part precedes the scalar remainder
                    for (unsigned qq = 2 * h; qq < 2 * h + 2; qq++) {
                        uint64_t v[16];
                        bad |= !vbp_decode16_rt<true>(bw, blk, l, qq, v);
#pragma unroll
                        for (int k = 0; k < 16; k++) {
                            const uint64_t x = v[k] + ref;
                            const bool hit = cmp_bits(x, c.c, c.cf, true);
                            cnt += hit;
                            sum += hit ? x : 0;
                        }
                    }
                }
            }
        } else if (bi.kind == kItDelta) {
            if (sd.b0 == bi.start) carry = __ldg(seeks + bi.seek * 8 + l);
            for (unsigned j = 0; j < sd.nblk; j++)
                carry = delta_block_rt(sd.bw[j], reinterpret_cast<const uint64_t *>(base + sd.off[j]), l, q, carry,
                                       c.c, c.pred.cmp, c.cf, cnt, sum, bad);
        } else if (bi.kind == kItRest) {
            for (uint64_t r = bi.start + lane; r < bi.start + bi.count; r += 32) {
                const uint64_t v = __ldg(c.rest + (r - c.n_compr));
                const bool hit = cmp_bits(v, c.c, c.cf, r < c.sfrom);
                cnt += hit;
                sum += hit ? v : 0;
            }
        } else {  // rle_f runs, decompressed: rows before sfrom compare signed, the rest unsigned
            const uint64_t *pairs = reinterpret_cast<const uint64_t *>(c.data);
            uint64_t row = bi.seek;
            for (uint64_t r0 = bi.start; r0 < bi.start + bi.count; r0 += 32) {
                const uint64_t r = r0 + lane;
                const bool in = r < bi.start + bi.count;
                const uint64_t v = in ? __ldg(pairs + 2 * r) : 0, len = in ? __ldg(pairs + 2 * r + 1) : 0;
                uint64_t incl = len;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                    if (int(lane) >= d) incl += o;
                }
                const uint64_t rs = row + incl - len;
                const uint64_t nsig = c.sfrom > rs ? minu(c.sfrom - rs, len) : 0;
                const uint64_t add =
                    (cmp_bits(v, c.c, c.cf, true) ? nsig : 0) + (cmp_bits(v, c.c, c.cf, false) ? len - nsig : 0);
                cnt += add;
                sum += v * add;
                row += __shfl_sync(0xFFFFFFFFu, incl, 31);
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, d);
            sum += __shfl_xor_sync(0xFFFFFFFFu, sum, d);
        }
        if (lane == 0) {
            if (cnt) atomicAdd(out_cnt + bi.col, (unsigned long long)cnt);
            if (sum) atomicAdd(out_sum + bi.col, (unsigned long long)sum);
        }
        __syncwarp();
        consumed++;
    }
    // a failed wait leaves copies in flight, the one it gave up on included:
    // wait for them (bounded) before leaving
    if (!ok)
        for (unsigned t = consumed; t < issued; t++) mbar_wait(bar + t % S, (t / S) & 1u);
    if (!ok && lane == 0) atomicOr(err, kErrTimeout);
    if (bad && lane == 0) atomicOr(err, kErrCorrupt);
}

__global__ void k_pick_seeks(const uint64_t *__restrict__ carry, uint64_t nb, uint64_t first_slot,
                             uint64_t *__restrict__ seeks) {
    const uint64_t n_it = (nb + kBItemBlocks - 1) / kBItemBlocks;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_it * 8;
         i += uint64_t(gridDim.x) * blockDim.x)
        seeks[(first_slot + i / 8) * 8 + i % 8] = carry[(i / 8) * kBItemBlocks * 8 + i % 8];
}

// bit width of every column's first block (the decoder its items take)
__global__ void k_first_bw(const BCol *__restrict__ cols, uint64_t n, uint8_t *__restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const BCol &c = cols[i];
        out[i] = c.index && c.n_compr ? uint8_t(idx_bw(c.index[0])) : uint8_t(c.bw);
    }
}

// run lengths summed per item of kBItemRuns runs
__global__ void k_rle_item_rows(const uint64_t *__restrict__ pairs, uint64_t runs, uint64_t *__restrict__ out) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t n_it = (runs + kBItemRuns - 1) / kBItemRuns;
    for (uint64_t i = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; i < n_it;
         i += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t s = 0;
        for (uint64_t r = i * kBItemRuns + lane; r < minu(runs, (i + 1) * kBItemRuns); r += 32) s += pairs[2 * r + 1];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, d);
        if (lane == 0) out[i] = s;
    }
}

}  // namespace
}  // namespace ms

using namespace ms;

constexpr int kBatchKinds = 5;  // kItVbp, kItFor, kItDelta, kItRest, kItRle

struct ms_batch {
    ms_arena *arena;
    uint64_t n_cols, n_items, plan_bytes;
    BCol *d_cols;
    BItem *d_items;
    uint64_t *d_seeks;
    unsigned long long *d_head;  // one queue head per kind segment
    ms_tuning cfg;               // warps, stages, stage_bytes (per warp), ctas_per_sm
    ms_tuning kcfg[kBatchKinds]; // per-kind configuration (kset: set apart from cfg)
    bool kset[kBatchKinds];
    uint64_t seg[kBatchKinds + 1];  // items of kind k: [seg[k], seg[k+1]) (the queue is sorted by kind)
    cudaStream_t side[kBatchKinds];
    cudaEvent_t fork, join[kBatchKinds];
    bool streams;
    cudaGraphExec_t graph;
    uint64_t *g_cnt, *g_sum;  // outputs the graph was captured for
};

namespace {

size_t batch_shm(const ms_tuning &t) {
    return size_t(t.warps) * (bwarp_meta_bytes(t.stages) + size_t(t.stages) * t.stage_bytes);
}

// One persistent launch over items [i0, i1) with configuration t and queue head `head`.
int batch_launch_range(ms_batch *b, const ms_tuning &t, uint64_t i0, uint64_t i1, unsigned long long *head,
                       uint64_t *d_cnt, uint64_t *d_sum, cudaStream_t st) {
    if (i1 <= i0) return MS_OK;
    const unsigned S = t.stages, SB = t.stage_bytes;
    const size_t shm = batch_shm(t);
    const unsigned grid = unsigned(sm_count()) * t.ctas_per_sm;
#define MS_B(Wn)                                                                                                 \
    case Wn:                                                                                                     \
        k_batch<Wn><<<grid, 32 * Wn, shm, st>>>(b->d_cols, b->d_items + i0, i1 - i0, b->d_seeks, S, SB, head,    \
                                                (unsigned long long *)d_cnt, (unsigned long long *)d_sum,         \
                                                b->arena->d_err);                                                \
        break;
    switch (t.warps) {
        MS_B(4) MS_B(8) MS_B(12) MS_B(16)
    default: return ms_fail(MS_ERR_INVALID, "batch: warps must be 4, 8, 12 or 16");
    }
#undef MS_B
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

const ms_tuning &kind_cfg(const ms_batch *b, int k) { return b->kset[k] ? b->kcfg[k] : b->cfg; }

bool same_cfg(const ms_tuning &x, const ms_tuning &y) {
    return x.warps == y.warps && x.stages == y.stages && x.stage_bytes == y.stage_bytes &&
           x.ctas_per_sm == y.ctas_per_sm;
}

int batch_launch(ms_batch *b, uint64_t *d_cnt, uint64_t *d_sum, cudaStream_t st) {
    MS_CUDA_TRY(cudaMemsetAsync(b->d_head, 0, 8 * kBatchKinds, st));
    if (!b->n_cols) return MS_OK;
    MS_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, 8 * b->n_cols, st));
    MS_CUDA_TRY(cudaMemsetAsync(d_sum, 0, 8 * b->n_cols, st));
    if (!b->n_items) return MS_OK;
    bool any = false;
    for (int k = 0; k < kBatchKinds; k++) any |= b->kset[k] && b->seg[k + 1] > b->seg[k];
    if (!any) return batch_launch_range(b, b->cfg, 0, b->n_items, b->d_head, d_cnt, d_sum, st);
    // kind segments with their own configuration: consecutive segments of one
    // configuration share a launch; the launches run on forked streams, so
    // one's tail overlaps the next one's start (the joins bring them back)
    if (!b->streams) {
        MS_CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        for (int k = 0; k < kBatchKinds; k++) {
            MS_CUDA_TRY(cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
            MS_CUDA_TRY(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
        }
        b->streams = true;
    }
    MS_CUDA_TRY(cudaEventRecord(b->fork, st));
    int g = 0;
    for (int k = 0; k < kBatchKinds;) {
        int e = k + 1;
        while (e < kBatchKinds && same_cfg(kind_cfg(b, e), kind_cfg(b, k))) e++;
        if (b->seg[e] > b->seg[k]) {
            MS_CUDA_TRY(cudaStreamWaitEvent(b->side[g], b->fork, 0));
            const int rc = batch_launch_range(b, kind_cfg(b, k), b->seg[k], b->seg[e], b->d_head + g, d_cnt, d_sum,
                                              b->side[g]);
            if (rc) return rc;
            MS_CUDA_TRY(cudaEventRecord(b->join[g], b->side[g]));
            MS_CUDA_TRY(cudaStreamWaitEvent(st, b->join[g], 0));
            g++;
        }
        k = e;
    }
    return MS_OK;
}

int batch_set_attr(const ms_tuning &t, size_t at_least = 0) {
    const size_t shm = batch_shm(t) > at_least ? batch_shm(t) : at_least;
    int dev = 0, maxb = 0, maxsm = 0;
    MS_CUDA_TRY(cudaGetDevice(&dev));
    MS_CUDA_TRY(cudaDeviceGetAttribute(&maxb, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    MS_CUDA_TRY(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    if (shm > size_t(maxb) || (shm + 1024) * t.ctas_per_sm > size_t(maxsm))
        return ms_fail(MS_ERR_INVALID, "batch: warps x stages x stage_bytes exceed shared memory");
#define MS_B(Wn)                                                                                               \
    case Wn:                                                                                                   \
        MS_CUDA_TRY(cudaFuncSetAttribute(k_batch<Wn>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm))); \
        break;
    switch (t.warps) {
        MS_B(4) MS_B(8) MS_B(12) MS_B(16)
    default: return ms_fail(MS_ERR_INVALID, "batch: warps must be 4, 8, 12 or 16");
    }
#undef MS_B
    return MS_OK;
}

// The dynamic shared-memory attribute of every kernel variant: the largest
// need among the configurations that use it.
int batch_set_attrs(const ms_batch *b) {
    for (int w = 4; w <= 16; w += 4) {
        size_t need = 0;
        const ms_tuning *use = nullptr;
        auto consider = [&](const ms_tuning &t) {
            if (int(t.warps) == w && batch_shm(t) >= need) {
                need = batch_shm(t);
                use = &t;
            }
        };
        consider(b->cfg);
        for (int k = 0; k < kBatchKinds; k++)
            if (b->kset[k]) consider(b->kcfg[k]);
        if (use) {
            const int rc = batch_set_attr(*use, need);
            if (rc) return rc;
        }
    }
    return MS_OK;
}

void batch_release(ms_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->streams) {
        cudaEventDestroy(b->fork);
        for (int k = 0; k < kBatchKinds; k++) {
            cudaStreamDestroy(b->side[k]);
            cudaEventDestroy(b->join[k]);
        }
    }
}

int batch_fail(ms_batch *b, int rc) {
    batch_release(b);
    delete b;
    return rc;
}

}  // namespace

extern "C" int ms_gpu_batch_create(const ms_col *cols, const uint64_t *consts, uint64_t n_cols, int cmp, ms_arena *a,
                                   ms_batch **out, void *stream) {
    if (!out || !a || (n_cols && (!cols || !consts))) return ms_fail(MS_ERR_INVALID, "batch_create: null argument");
    if (cmp < MS_CMP_EQ || cmp > MS_CMP_GE) return ms_fail(MS_ERR_INVALID, "batch_create: comparison");
    *out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<BCol> hc(n_cols);
    std::vector<BItem> hi;
    std::vector<uint64_t> rle_cols, delta_cols, first_item(n_cols, 0);
    uint64_t n_seek = 0;
    for (uint64_t i = 0; i < n_cols; i++) {
        const ms_col &c = cols[i];
        int rc = check_col(&c, false);
        if (rc) return rc;
        BCol b{};
        b.c = consts[i];
        b.pred = make_pred(cmp, consts[i]);
        b.cf = cmp_flags(cmp);
        b.n = c.count_values;
        if (c.format == MS_FMT_RLE) {
            b.data = (const uint8_t *)c.data;
            b.sfrom = c.count_values - c.count_values % kStep;  // as the decompressed column
            const uint64_t runs = c.size_used_byte / 16;
            first_item[i] = hi.size();
            for (uint64_t r = 0; r < runs; r += kBItemRuns)
                hi.push_back(BItem{uint32_t(i), kItRle, r, uint32_t(minu(kBItemRuns, runs - r)), 0, 0});
            rle_cols.push_back(i);
            hc[i] = b;
            continue;
        }
        if (c.format == MS_FMT_DELTA_DVBP && c.index_aux)
            return ms_fail(MS_ERR_UNSUPPORTED, "batch_create: delta_f views with a carry-in are not batched");
        ColView v;
        const uint64_t mark = a->used;
        const bool had_index = c.format == MS_FMT_STATIC_VBP || c.format == MS_FMT_UNCOMPR ||
                               (c.index && c.n_index >= (c.count_values - count_rest(c)) / kBlock &&
                                (c.format != MS_FMT_FOR_DVBP || c.index_aux));
        rc = prepare_view(&c, a, st, &v);  // builds a missing block index in the arena (kept)
        if (rc) return rc;
        if (c.format == MS_FMT_DELTA_DVBP && had_index) a->used = mark;  // delta carries: recomputed below
        b.data = v.data;
        b.index = v.index;
        b.aux = v.aux;
        b.rest = v.rest;
        b.n_compr = v.n_compr;
        b.sfrom = v.sfrom;
        b.bw = v.bw;
        const uint32_t kind = c.format == MS_FMT_FOR_DVBP ? kItFor : c.format == MS_FMT_DELTA_DVBP ? kItDelta : kItVbp;
        const uint64_t nb = v.nb();
        for (uint64_t s = 0; s < nb; s += kBItemBlocks)
            hi.push_back(BItem{uint32_t(i), kind, s, uint32_t(minu(kBItemBlocks, nb - s)), 0,
                               kind == kItDelta ? n_seek + s / kBItemBlocks : 0});
        if (kind == kItDelta && nb) {
            delta_cols.push_back(i);
            first_item[i] = n_seek;  // its first seek slot
            n_seek += (nb + kBItemBlocks - 1) / kBItemBlocks;
        }
        for (uint64_t r = v.n_compr; r < v.n; r += kBItemRest)
            hi.push_back(BItem{uint32_t(i), kItRest, r, uint32_t(minu(kBItemRest, v.n - r)), 0, 0});
        hc[i] = b;
    }
    ms_batch *b = new ms_batch{};
    b->arena = a;
    b->n_cols = n_cols;
    b->n_items = hi.size();
    b->cfg = ms_tuning{1, 12, 2, 8192, 1, 16};
    b->d_cols = arena_take_t<BCol>(a, n_cols + 1);
    b->d_items = arena_take_t<BItem>(a, hi.size() + 1);
    b->d_seeks = arena_take_t<uint64_t>(a, 8 * n_seek + 8);
    b->d_head = arena_take_t<unsigned long long>(a, kBatchKinds);
    if (!b->d_cols || !b->d_items || !b->d_seeks || !b->d_head)
        return batch_fail(b, ms_fail(MS_ERR_NOMEM, "arena exhausted (batch plan)"));
    b->plan_bytes = sizeof(BCol) * n_cols + sizeof(BItem) * hi.size() + 64 * n_seek;
    // delta_f seeks: the carry into each item's first block
    for (uint64_t i : delta_cols) {
        const uint64_t mark = a->used;
        ColView v;
        int rc = prepare_view(&cols[i], a, st, &v);
        if (rc) return batch_fail(b, rc);
        k_pick_seeks<<<64, 256, 0, st>>>(v.carry, v.nb(), first_item[i], b->d_seeks);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        a->used = mark;
    }
    // rle_f: the first row of every item
    for (uint64_t i : rle_cols) {
        const uint64_t runs = cols[i].size_used_byte / 16;
        const uint64_t n_it = (runs + kBItemRuns - 1) / kBItemRuns;
        if (!n_it) continue;
        const uint64_t mark = a->used;
        uint64_t *tot = arena_take_t<uint64_t>(a, n_it);
        if (!tot) return batch_fail(b, ms_fail(MS_ERR_NOMEM, "arena exhausted (batch plan)"));
        k_rle_item_rows<<<64, 256, 0, st>>>((const uint64_t *)cols[i].data, runs, tot);
        MS_CUDA_TRY(cudaGetLastError());
        std::vector<uint64_t> h(n_it);
        MS_CUDA_TRY(cudaMemcpyAsync(h.data(), tot, 8 * n_it, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        a->used = mark;
        uint64_t row = 0;
        for (uint64_t k = 0; k < n_it; k++) {
            hi[first_item[i] + k].seek = row;
            row += h[k];
        }
    }
    if (n_cols) MS_CUDA_TRY(cudaMemcpyAsync(b->d_cols, hc.data(), sizeof(BCol) * n_cols, cudaMemcpyHostToDevice, st));
    // Queue order: items that take the same decoder (kind, bit width) run
    // together, so the warps of an SM share their instructions; the items of
    // a column keep their order.
    if (n_cols) {
        const uint64_t mark = a->used;
        uint8_t *d_bw = arena_take_t<uint8_t>(a, n_cols);
        if (!d_bw) return batch_fail(b, ms_fail(MS_ERR_NOMEM, "arena exhausted (batch plan)"));
        k_first_bw<<<unsigned(minu((n_cols + 255) / 256, 1024)), 256, 0, st>>>(b->d_cols, n_cols, d_bw);
        MS_CUDA_TRY(cudaGetLastError());
        std::vector<uint8_t> fbw(n_cols);
        MS_CUDA_TRY(cudaMemcpyAsync(fbw.data(), d_bw, n_cols, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        a->used = mark;
        std::stable_sort(hi.begin(), hi.end(), [&](const BItem &x, const BItem &y) {
            const uint32_t kx = (x.kind << 8) | (x.kind <= kItDelta ? fbw[x.col] : 0u);
            const uint32_t ky = (y.kind << 8) | (y.kind <= kItDelta ? fbw[y.col] : 0u);
            return kx < ky;
        });
    }
    // kind segments of the sorted queue
    for (int k = 0, i = 0; k <= kBatchKinds; k++) {
        while (i < int(hi.size()) && int(hi[i].kind) < k) i++;
        b->seg[k] = k == kBatchKinds ? hi.size() : uint64_t(i);
    }
    if (!hi.empty())
        MS_CUDA_TRY(cudaMemcpyAsync(b->d_items, hi.data(), sizeof(BItem) * hi.size(), cudaMemcpyHostToDevice, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    int rc = read_err(a, st);
    if (rc) return batch_fail(b, rc);
    rc = batch_set_attr(b->cfg);
    if (rc) return batch_fail(b, rc);
    *out = b;
    return MS_OK;
}

extern "C" int ms_gpu_batch_set_config(ms_batch *b, const ms_tuning *t) {
    if (!b || !t) return ms_fail(MS_ERR_INVALID, "batch_set_config: null argument");
    if (t->stages < 2 || t->stages > 8 || t->stage_bytes < 4096 || t->stage_bytes % 128 || t->ctas_per_sm < 1 ||
        t->ctas_per_sm > 4)
        return ms_fail(MS_ERR_INVALID,
                       "batch_set_config: stages 2..8, stage_bytes >= 4096 (multiple of 128), ctas_per_sm 1..4");
    if (t->warps < 4 || t->warps > 16 || t->warps % 4)
        return ms_fail(MS_ERR_INVALID, "batch: warps must be 4, 8, 12 or 16");
    const ms_tuning prev = b->cfg;
    b->cfg = *t;
    int rc = batch_set_attrs(b);
    if (rc) {
        b->cfg = prev;
        return rc;
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return MS_OK;
}

extern "C" int ms_gpu_batch_set_kind_config(ms_batch *b, int kind, const ms_tuning *t) {
    if (!b || kind < 0 || kind >= kBatchKinds) return ms_fail(MS_ERR_INVALID, "batch_set_kind_config: bad argument");
    if (t && (t->stages < 2 || t->stages > 8 || t->stage_bytes < 4096 || t->stage_bytes % 128 ||
              t->ctas_per_sm < 1 || t->ctas_per_sm > 4))
        return ms_fail(MS_ERR_INVALID,
                       "batch_set_kind_config: stages 2..8, stage_bytes >= 4096 (multiple of 128), ctas_per_sm 1..4");
    if (t && (t->warps < 4 || t->warps > 16 || t->warps % 4))
        return ms_fail(MS_ERR_INVALID, "batch: warps must be 4, 8, 12 or 16");
    const ms_tuning prev = b->kcfg[kind];
    const bool prev_set = b->kset[kind];
    b->kset[kind] = t != nullptr;
    if (t) b->kcfg[kind] = *t;
    int rc = batch_set_attrs(b);
    if (rc) {
        b->kcfg[kind] = prev;
        b->kset[kind] = prev_set;
        return rc;
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return MS_OK;
}

extern "C" int ms_gpu_batch_get_kind_config(const ms_batch *b, int kind, ms_tuning *t, uint64_t *n_items) {
    if (!b || !t || kind < 0 || kind >= kBatchKinds) return ms_fail(MS_ERR_INVALID, "batch_get_kind_config");
    *t = b->kset[kind] ? b->kcfg[kind] : b->cfg;
    if (n_items) *n_items = b->seg[kind + 1] - b->seg[kind];
    return MS_OK;
}

extern "C" int ms_gpu_batch_get_config(const ms_batch *b, ms_tuning *t) {
    if (!b || !t) return ms_fail(MS_ERR_INVALID, "batch_get_config: null argument");
    *t = b->cfg;
    return MS_OK;
}

extern "C" int ms_gpu_batch_run(ms_batch *b, uint64_t *d_counts, uint64_t *d_sums, void *stream) {
    if (!b || (b->n_cols && (!d_counts || !d_sums))) return ms_fail(MS_ERR_INVALID, "batch_run: null argument");
    return batch_launch(b, d_counts, d_sums, (cudaStream_t)stream);
}

extern "C" int ms_gpu_batch_run_graph(ms_batch *b, uint64_t *d_counts, uint64_t *d_sums, void *stream) {
    if (!b || (b->n_cols && (!d_counts || !d_sums))) return ms_fail(MS_ERR_INVALID, "batch_run_graph: null argument");
    if (b->graph && (b->g_cnt != d_counts || b->g_sum != d_sums)) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (!b->graph) {
        cudaStream_t cs;
        MS_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        int rc = e == cudaSuccess ? batch_launch(b, d_counts, d_sums, cs) : MS_OK;
        const cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(cs, &g) : cudaSuccess;
        cudaStreamDestroy(cs);
        MS_CUDA_TRY(e);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        MS_CUDA_TRY(e2);
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        MS_CUDA_TRY(e);
        b->g_cnt = d_counts;
        b->g_sum = d_sums;
    }
    MS_CUDA_TRY(cudaGraphLaunch(b->graph, (cudaStream_t)stream));
    return MS_OK;
}

extern "C" int ms_gpu_batch_info(const ms_batch *b, uint64_t *n_items, uint64_t *plan_bytes) {
    if (!b) return ms_fail(MS_ERR_INVALID, "batch_info: null");
    if (n_items) *n_items = b->n_items;
    if (plan_bytes) *plan_bytes = b->plan_bytes;
    return MS_OK;
}

extern "C" void ms_gpu_batch_destroy(ms_batch *b) {
    if (!b) return;
    batch_release(b);
    delete b;
}
