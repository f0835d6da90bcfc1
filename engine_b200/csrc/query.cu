// query.cu -- the fused compressed multi-operator query:
//
//   P1 = select(filter < c)            (select_compr.h:100-260)
//   P2 = semi_join(L, fk)              (join_semi_equi_compr.h:106-300)
//   P  = intersect_sorted(P1, P2)      (intersect_compr.h:190-347)
//   G  = project(gkey, P), M = project(measure, P)
//   (gr, ext) = group(G); S = agg_sum(gr, M, |ext|)   (group_compr.h, scalar/agg_sum_uncompr.h)
//
// in one pass over the fact table: per 512-row block a warp decodes filter,
// probes fk against the build side's bitmap, and for the surviving rows
// decodes gkey and measure and folds (key, row, measure) into a per-CTA
// shared-memory group table (warp-aggregated for skewed keys), flushed to a
// global table at the end.  Each key keeps its smallest row; after a scan of
// the per-block hit counts, the group's extent -- the position of that row in
// P, which is what the reference's group operator returns -- is the hits
// before its block plus its rank within the block, and ordering groups by
// first row gives the reference's group ids.  The result equals the operator-at-a-time
// pipeline's bit for bit; no intermediate touches HBM.
#include <algorithm>
#include <vector>

#include "fastpath.cuh"
#include "internal.h"
#include "scan.cuh"
#include "stream.cuh"
#include "tma.cuh"

namespace ms {
namespace {

constexpr unsigned kQSlots = 2048;  // per-CTA group table
constexpr uint64_t kQEmpty = ~uint64_t(0);

__device__ __forceinline__ uint64_t qhash(uint64_t k) {
    k ^= k >> 33;
    k *= 0xFF51AFD7ED558CCDull;
    k ^= k >> 33;
    return k;
}

struct GTable {  // global group table (open addressing)
    unsigned long long *keys;
    unsigned long long *first;  // smallest row of the group
    unsigned long long *sums;
    uint64_t mask;
};

__device__ __forceinline__ bool gtable_add(const GTable &t, uint64_t key, uint64_t first, uint64_t sum) {
    uint64_t h = qhash(key) & t.mask;
    for (uint64_t p = 0; p <= t.mask; p++) {
        const unsigned long long old = atomicCAS(t.keys + h, kQEmpty, key);
        if (old == kQEmpty || old == key) {
            atomicMin(t.first + h, first);
            atomicAdd(t.sums + h, sum);
            return true;
        }
        h = (h + 1) & t.mask;
    }
    return false;
}

__global__ void __launch_bounds__(256) k_query3(ColView filt, ColView fk, ColView gkey, ColView meas, int cmp,
                                               uint64_t c, const uint32_t *__restrict__ bits, uint64_t lo,
                                               uint64_t span, GTable gt, uint32_t *__restrict__ blk_hits,
                                               uint64_t b_begin, unsigned *err) {
    __shared__ unsigned long long s_key[kQSlots], s_first[kQSlots], s_sum[kQSlots];
    for (unsigned i = threadIdx.x; i < kQSlots; i += blockDim.x) {
        s_key[i] = kQEmpty;
        s_first[i] = ~0ull;
        s_sum[i] = 0;
    }
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true, fit = true;
    for (uint64_t b = b_begin + (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < filt.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(filt, b, l, q, v, valid);
        unsigned m = select_mask(filt, b, l, q, v, valid, cmp, c);
        if (__any_sync(0xFFFFFFFFu, m != 0)) {
            unsigned vk;
            ok &= decode_block(fk, b, l, q, v, vk);
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (!((m >> k) & 1u)) continue;
                const uint64_t d = v[k] - lo;
                const bool in = v[k] >= lo && d < span && ((bits[d >> 5] >> (d & 31u)) & 1u);
                if (!in) m &= ~(1u << k);
            }
        }
        const unsigned total = __reduce_add_sync(0xFFFFFFFFu, __popc(m));
        if (lane == 0) blk_hits[b] = total;
        if (total == 0) continue;
        uint64_t g[16], w[16];
        unsigned vg, vm;
        ok &= decode_block(gkey, b, l, q, g, vg);
        ok &= decode_block(meas, b, l, q, w, vm);
        const uint64_t row0 = b * kBlock;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const bool hit = (m >> k) & 1u;
            const uint64_t key = g[k];
            const uint64_t first = row0 + (16u * q + k) * 8u + l;
            // lanes with the same key combine first: one table update per key
            const unsigned hm = __ballot_sync(0xFFFFFFFFu, hit);
            if (!hit) continue;
            const unsigned peers = __match_any_sync(hm, key);
            uint64_t s = w[k], f = first;
            for (unsigned rest = peers; rest;) {
                const int src = __ffs(rest) - 1;
                rest &= rest - 1;
                const uint64_t so = __shfl_sync(peers, w[k], src);
                const uint64_t fo = __shfl_sync(peers, first, src);
                if (src != int(lane)) {
                    s += so;
                    f = minu(f, fo);
                }
            }
            if (int(lane) != __ffs(peers) - 1) continue;
            // per-CTA table, then the global one when the key does not fit
            uint64_t h = qhash(key) & (kQSlots - 1);
            bool done = false;
            if (key != kQEmpty) {
                for (unsigned p = 0; p < 16; p++) {
                    const unsigned long long old = atomicCAS(s_key + h, kQEmpty, key);
                    if (old == kQEmpty || old == key) {
                        atomicMin(s_first + h, (unsigned long long)f);
                        atomicAdd(s_sum + h, (unsigned long long)s);
                        done = true;
                        break;
                    }
                    h = (h + 1) & (kQSlots - 1);
                }
            }
            if (!done) fit &= gtable_add(gt, key, f, s);
        }
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < kQSlots; i += blockDim.x)
        if (s_key[i] != kQEmpty) fit &= gtable_add(gt, s_key[i], s_first[i], s_sum[i]);
    if (!ok) atomicOr(err, kErrCorrupt);
    if (!fit) atomicOr(err, kErrCapacity);
}

// ---------------------------------------------------------------------------
// Staged variant.  One persistent CTA per SM: warp 0 forms tiles of
// consecutive 512-row blocks whose bytes in all four fact columns fit one
// stage buffer and brings each column's range into shared memory with one
// bulk copy; consumer warps take the tile's blocks round-robin.  Per block
// the filter is decoded and compared inside the bit-width switch (all 512
// rows); the foreign key, group key and measure are not decoded as blocks:
// only the values of rows still alive are extracted from the staged words
// (about 10%, 1% and 1% of the rows in the star query), so the consumers stay
// below the memory time.  Requires the filter in uncompr/static_vbp/
// dynamic_vbp and the other three columns in those or for_f (delta_f and
// rows in the uncompressed rests go through k_query3).
// ---------------------------------------------------------------------------
constexpr unsigned kQTile = 32;  // blocks per tile (one producer lane each)
constexpr unsigned kQCols = 4;   // filter, fk, group key, measure

struct QStage {
    uint64_t b0;
    unsigned nblk;
    unsigned pad;
};

struct QCfg {
    unsigned stages;
    unsigned stage_bytes;
};

// value of slot s (0..63) of lane l in a vbp block of width bw
__device__ __forceinline__ uint64_t vbp_extract(const uint64_t *blk, unsigned bw, unsigned l, unsigned s) {
    const unsigned p = s * bw, w = p >> 6, sh = p & 63u;
    uint64_t x = blk[w * 8u + l] >> sh;
    if (sh + bw > 64u) x |= blk[(w + 1u) * 8u + l] << (64u - sh);
    return bw >= 64u ? x : x & ((uint64_t(1) << bw) - 1u);
}

__host__ __device__ inline uint64_t q3_meta_bytes(unsigned S) {
    return (uint64_t(16) * S + sizeof(QStage) * S + 5ull * kQCols * S * kQTile + 127) / 128 * 128;
}

// Where the probes read the build side's bitmap (nwords words):
enum : int {
    kBmGlobal = 0,   // global memory (an L2 round trip per probe)
    kBmShared = 1,   // the whole bitmap in this CTA's shared memory
    kBmCluster = 2,  // split over the two CTAs of a cluster: words [0, half) in
                     // rank 0, [half, nwords) in rank 1, read through
                     // distributed shared memory (ld.shared::cluster)
};

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// every thread of both CTAs of the cluster; shared-memory writes before it
// are visible to the other CTA after it
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

__device__ __forceinline__ uint32_t dsmem_ld32(const uint32_t *local_base, uint32_t idx, unsigned rank) {
    uint32_t a, v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(local_base + idx)), "r"(rank));
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}

// kBM: where the bitmap lives (kBmGlobal / kBmShared / kBmCluster); in
// shared memory it follows the group table, so a probe costs a shared-memory
// load (local or in the partner CTA) instead of an L2 round trip.
template <int W, int kBM>
__global__ void __launch_bounds__(32 * (W + 1), 1)
    k_query3_tma(ColView fk, ColView gkey, ColView meas, StreamCol c0, StreamCol c1, StreamCol c2, StreamCol c3,
                 Pred pred, const uint32_t *__restrict__ bits, uint64_t nwords, uint64_t lo, uint64_t span, QCfg cfg,
                 GTable gt, uint32_t *__restrict__ blk_hits, unsigned *err) {
    constexpr bool kSB = kBM != kBmGlobal;
    extern __shared__ __align__(128) uint8_t smem[];
    const unsigned S = cfg.stages, SB = cfg.stage_bytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + S;
    QStage *desc = reinterpret_cast<QStage *>(empty + S);
    uint32_t *offs = reinterpret_cast<uint32_t *>(desc + S);                 // [S][kQCols][kQTile]
    uint8_t *bws = reinterpret_cast<uint8_t *>(offs + S * kQCols * kQTile);  // [S][kQCols][kQTile]
    uint8_t *ring = smem + q3_meta_bytes(S);
    unsigned long long *s_key = reinterpret_cast<unsigned long long *>(ring + size_t(S) * SB);
    unsigned long long *s_first = s_key + kQSlots;
    unsigned long long *s_sum = s_first + kQSlots;

    uint32_t *s_bits = reinterpret_cast<uint32_t *>(s_sum + kQSlots);
    const uint32_t *pbits = kSB ? s_bits : bits;
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (unsigned i = threadIdx.x; i < kQSlots; i += blockDim.x) {
        s_key[i] = kQEmpty;
        s_first[i] = ~0ull;
        s_sum[i] = 0;
    }
    const uint32_t half = uint32_t((nwords + 1) / 2);  // words per CTA in a cluster
    if (kBM == kBmShared)
        for (uint64_t i = threadIdx.x; i < nwords; i += blockDim.x) s_bits[i] = __ldg(bits + i);
    if (kBM == kBmCluster) {
        const uint64_t w0 = uint64_t(cluster_rank()) * half;
        for (uint64_t i = threadIdx.x; i < half; i += blockDim.x) s_bits[i] = w0 + i < nwords ? __ldg(bits + w0 + i) : 0u;
    }
    if (threadIdx.x == 0) {
        for (unsigned st = 0; st < S; st++) {
            mbar_init(full + st, 1);
            mbar_init(empty + st, W);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (kBM == kBmCluster) cluster_sync();  // both halves of the bitmap are in place

    const uint64_t nbs = minu(minu(c0.nb, c1.nb), minu(c2.nb, c3.nb));
    const uint64_t b_lo = nbs * blockIdx.x / gridDim.x, b_hi = nbs * (blockIdx.x + 1) / gridDim.x;
    bool ok = true, fit = true, bad = false;

    if (warp == 0) {
        // ---------------- producer ----------------
        const StreamCol *cols[kQCols] = {&c0, &c1, &c2, &c3};
        uint64_t b = b_lo;
        unsigned t = 0;
        for (;; t++) {
            const unsigned st = t % S, use = t / S;
            // the next tile's block locations are requested before waiting
            // for its stage, so the index loads overlap the wait
            const uint64_t blk = b + lane;
            const bool valid = blk < b_hi;
            uint64_t off[kQCols], len[kQCols], x0[kQCols];
            unsigned bw[kQCols];
#pragma unroll
            for (unsigned c = 0; c < kQCols; c++) {
                off[c] = 0;
                bw[c] = 0;
                if (valid) blk_loc(*cols[c], blk, off[c], bw[c]);
            }
            if (use > 0 && !mbar_wait(empty + st, (use - 1) & 1u)) {
                ok = false;
                break;
            }
            if (b >= b_hi) {
                if (lane == 0) {
                    desc[st].nblk = 0;
                    mbar_arrive(full + st);
                }
                t++;
                break;
            }
            uint64_t need = 0;
#pragma unroll
            for (unsigned c = 0; c < kQCols; c++) {
                x0[c] = __shfl_sync(0xFFFFFFFFu, off[c], 0);
                len[c] = valid ? off[c] + 64ull * bw[c] - x0[c] : 0;
                need += align_up(len[c], 128);
            }
            const bool fits = valid && need <= SB;
            const unsigned T = __popc(__ballot_sync(0xFFFFFFFFu, fits));
            if (T == 0) {  // one block larger than a stage: configuration error
                if (lane == 0) {
                    atomicOr(err, kErrCapacity);
                    desc[st].nblk = 0;
                    mbar_arrive(full + st);
                }
                ok = false;
                t++;
                break;
            }
            uint32_t cbase[kQCols];
            uint64_t clen[kQCols];
            uint32_t acc = 0;
#pragma unroll
            for (unsigned c = 0; c < kQCols; c++) {
                clen[c] = __shfl_sync(0xFFFFFFFFu, len[c], T - 1);
                cbase[c] = acc;
                acc += uint32_t(align_up(clen[c], 128));
            }
            if (lane < T) {
#pragma unroll
                for (unsigned c = 0; c < kQCols; c++) {
                    offs[(st * kQCols + c) * kQTile + lane] = st * SB + cbase[c] + uint32_t(off[c] - x0[c]);
                    bws[(st * kQCols + c) * kQTile + lane] = uint8_t(bw[c]);
                }
            }
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                desc[st].b0 = b;
                desc[st].nblk = T;
                __threadfence_block();
                uint64_t total = 0;
#pragma unroll
                for (unsigned c = 0; c < kQCols; c++) total += clen[c];
                mbar_arrive_expect_tx(full + st, unsigned(total));
#pragma unroll
                for (unsigned c = 0; c < kQCols; c++)
                    bulk_g2s(ring + st * SB + cbase[c], cols[c]->base + x0[c], unsigned(clen[c]), full + st);
            }
            __syncwarp();
            b += T;
        }
        const unsigned issued = t;
        for (unsigned st = 0; st < S && st < issued; st++) {
            const unsigned uses = (issued - st + S - 1) / S;
            if (!mbar_wait(full + st, (uses - 1) & 1u)) ok = false;
        }
    } else {
        // ---------------- consumers ----------------
        const unsigned cw = warp - 1, l = lane & 7u, q = lane >> 3;
        const bool fk_for = fk.fmt == MS_FMT_FOR_DVBP, g_for = gkey.fmt == MS_FMT_FOR_DVBP,
                   m_for = meas.fmt == MS_FMT_FOR_DVBP;
        for (unsigned t = 0;; t++) {
            const unsigned st = t % S, use = t / S;
            if (!mbar_wait(full + st, use & 1u)) {
                ok = false;
                break;
            }
            const unsigned T = desc[st].nblk;
            if (T == 0) break;
            const uint64_t b0 = desc[st].b0;
            const unsigned j0 = unsigned((cw + W - (b0 - b_lo) % W) % W);
            const uint32_t *o = offs + st * kQCols * kQTile;
            const uint8_t *w = bws + st * kQCols * kQTile;
            for (unsigned j = j0; j < T; j += W) {
                const uint64_t blk = b0 + j;
                unsigned m = mask_block_rt(w[j], reinterpret_cast<const uint64_t *>(ring + o[j]), l, q, pred, bad);
                // semi-join probe of the surviving rows
                if (__any_sync(0xFFFFFFFFu, m != 0)) {
                    const uint64_t *kb = reinterpret_cast<const uint64_t *>(ring + o[kQTile + j]);
                    const unsigned kbw = w[kQTile + j];
                    if (kbw - 1u >= 64u) {
                        bad = true;
                        m = 0;
                    }
                    const uint64_t kref = fk_for ? __ldg(fk.aux + (blk >> 1)) : 0;
                    // four probes in flight per thread: the bitmap words are
                    // requested together, then tested
                    for (unsigned r = m; r;) {
                        unsigned kk[4];
                        uint32_t word[4], bit[4];
                        bool had[4], inr[4];
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            had[i] = r != 0;
                            kk[i] = had[i] ? unsigned(__ffs(r) - 1) : 0u;
                            r &= r - 1;
                            const uint64_t v = vbp_extract(kb, kbw, l, 16u * q + kk[i]) + kref;
                            const uint64_t d = v - lo;
                            inr[i] = had[i] && v >= lo && d < span;
                            if (kBM == kBmCluster) {
                                const uint32_t wi = uint32_t(d >> 5);
                                const unsigned own = wi >= half;
                                word[i] = inr[i] ? dsmem_ld32(s_bits, wi - own * half, own) : 0u;
                            } else {
                                word[i] = inr[i] ? (kSB ? pbits[d >> 5] : __ldg(pbits + (d >> 5))) : 0u;
                            }
                            bit[i] = unsigned(d & 31u);
                        }
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            if (had[i] && !(inr[i] && ((word[i] >> bit[i]) & 1u))) m &= ~(1u << kk[i]);
                    }
                }
                const unsigned total = __reduce_add_sync(0xFFFFFFFFu, __popc(m));
                if (lane == 0) blk_hits[blk] = total;
                if (total == 0) continue;
                const uint64_t *gb = reinterpret_cast<const uint64_t *>(ring + o[2 * kQTile + j]);
                const uint64_t *mb = reinterpret_cast<const uint64_t *>(ring + o[3 * kQTile + j]);
                const unsigned gbw = w[2 * kQTile + j], mbw = w[3 * kQTile + j];
                if (gbw - 1u >= 64u || mbw - 1u >= 64u) {
                    bad = true;
                    continue;
                }
                const uint64_t gref = g_for ? __ldg(gkey.aux + (blk >> 1)) : 0;
                const uint64_t mref = m_for ? __ldg(meas.aux + (blk >> 1)) : 0;
                const uint64_t row0 = blk * kBlock;
                for (unsigned r = m; __any_sync(0xFFFFFFFFu, r != 0); r &= r - 1) {
                    const bool hit = r != 0;
                    const unsigned hm = __ballot_sync(0xFFFFFFFFu, hit);
                    if (!hit) continue;
                    const unsigned k = __ffs(r) - 1;
                    const uint64_t key = vbp_extract(gb, gbw, l, 16u * q + k) + gref;
                    const uint64_t val = vbp_extract(mb, mbw, l, 16u * q + k) + mref;
                    const uint64_t first = row0 + (16u * q + k) * 8u + l;
                    const unsigned peers = __match_any_sync(hm, key);
                    uint64_t sm = val, f = first;
                    for (unsigned rest = peers; rest;) {
                        const int src = __ffs(rest) - 1;
                        rest &= rest - 1;
                        const uint64_t so = __shfl_sync(peers, val, src);
                        const uint64_t fo = __shfl_sync(peers, first, src);
                        if (src != int(lane)) {
                            sm += so;
                            f = minu(f, fo);
                        }
                    }
                    if (int(lane) != __ffs(peers) - 1) continue;
                    uint64_t h = qhash(key) & (kQSlots - 1);
                    bool done = false;
                    if (key != kQEmpty) {
                        for (unsigned p = 0; p < 16; p++) {
                            const unsigned long long old = atomicCAS(s_key + h, kQEmpty, key);
                            if (old == kQEmpty || old == key) {
                                atomicMin(s_first + h, (unsigned long long)f);
                                atomicAdd(s_sum + h, (unsigned long long)sm);
                                done = true;
                                break;
                            }
                            h = (h + 1) & (kQSlots - 1);
                        }
                    }
                    if (!done) fit &= gtable_add(gt, key, f, sm);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + st);
        }
    }
    __syncthreads();
    for (unsigned i = threadIdx.x; i < kQSlots; i += blockDim.x)
        if (s_key[i] != kQEmpty) fit &= gtable_add(gt, s_key[i], s_first[i], s_sum[i]);
    if (!ok) atomicOr(err, kErrTimeout);
    if (bad) atomicOr(err, kErrCorrupt);
    if (!fit) atomicOr(err, kErrCapacity);
    if (kBM == kBmCluster) cluster_sync();  // the partner may still read this CTA's half
}

// bitmap of the build side's keys (dense range)
__global__ void k_q3_bits(ColView l, uint64_t lo, uint32_t *bits, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, ll = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < l.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(l, b, ll, q, v, valid);
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((valid >> k) & 1u) {
                const uint64_t d = v[k] - lo;
                atomicOr(bits + (d >> 5), 1u << (d & 31u));
            }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

__global__ void k_minmax_q(ColView c, unsigned long long *mn, unsigned long long *mx, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    uint64_t lo = ~uint64_t(0), hi = 0;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < c.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(c, b, l, q, v, valid);
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((valid >> k) & 1u) {
                lo = minu(lo, v[k]);
                hi = maxu(hi, v[k]);
            }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
    atomicMin(mn, (unsigned long long)lo);
    atomicMax(mx, (unsigned long long)hi);
}

// Extent of every group: its first row's position in P, i.e. the hits in
// earlier blocks (scan of the per-block counts) plus the row's rank among the
// hits of its own block, which one warp per group recomputes by decoding that
// block of the filter and the foreign key again.  Results are compacted to
// dense records (key, extent, sum, first row) in arrival order.
__global__ void __launch_bounds__(256) k_q3_extents(GTable gt, ColView filt, ColView fk, int cmp, uint64_t c,
                                                   const uint32_t *__restrict__ bits, uint64_t lo, uint64_t span,
                                                   const uint64_t *__restrict__ blk_off,
                                                   unsigned long long *__restrict__ cnt,
                                                   uint64_t *__restrict__ o, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t h = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; h <= gt.mask;
         h += uint64_t(gridDim.x) * blockDim.x / 32) {
        const uint64_t key = gt.keys[h];
        if (key == kQEmpty) continue;
        const uint64_t row = gt.first[h];
        const uint64_t b = row / kBlock;
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(filt, b, l, q, v, valid);
        unsigned m = select_mask(filt, b, l, q, v, valid, cmp, c);
        ok &= decode_block(fk, b, l, q, v, valid);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint64_t d = v[k] - lo;
            if (!(v[k] >= lo && d < span && ((bits[d >> 5] >> (d & 31u)) & 1u))) m &= ~(1u << k);
        }
        unsigned rank[16];
        block_ranks(m, l, q, rank);
        const unsigned s = unsigned(row % kBlock) / 8u;  // slot of the row within its lane
        unsigned rk = 0;
#pragma unroll
        for (unsigned k = 0; k < 16; k++) rk = (16u * q + k == s) ? rank[k] : rk;
        rk = __shfl_sync(0xFFFFFFFFu, rk, int((s / 16u) * 8u + unsigned(row % 8)));
        if (lane == 0) {
            const unsigned long long i = atomicAdd(cnt, 1ull);
            o[4 * i] = key;
            o[4 * i + 1] = blk_off[b] + rk;
            o[4 * i + 2] = gt.sums[h];
            o[4 * i + 3] = row;
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

bool random_access(const ColView &v) { return plain(v) || v.fmt == MS_FMT_FOR_DVBP; }

constexpr uint64_t kQFirstGroups = 4096;  // group records read back with the counts
constexpr size_t kQSmemMax = 232448;  // 227 KiB of dynamic shared memory per CTA

// launch configuration of the staged kernel (consumer warps 8/16/24)
ms_tuning g_q3 = {1, 16, 3, 57344, 1, 16};
// device time of the last call's fact-table pass
cudaEvent_t g_q3_ev[2] = {nullptr, nullptr};
double g_q3_pass_ms = -1;

template <int W, int kBM>
int launch_q3_kern(size_t shm, QCfg cfg, const ColView &kv, const ColView &gv, const ColView &mv,
                   const StreamCol &s0, const StreamCol &s1, const StreamCol &s2, const StreamCol &s3, const Pred &pred,
                   const uint32_t *bits, uint64_t nwords, uint64_t lo, uint64_t span, const GTable &gt, uint32_t *hits,
                   unsigned *d_err, cudaStream_t st) {
    auto kern = k_query3_tma<W, kBM>;
    MS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
    if (kBM != kBmCluster) {
        kern<<<unsigned(sm_count()), 32 * (W + 1), shm, st>>>(kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span,
                                                              cfg, gt, hits, d_err);
        MS_CUDA_TRY(cudaGetLastError());
        return MS_OK;
    }
    // clusters of two CTAs (one per SM), as many as fit at once
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.blockDim = dim3(32 * (W + 1));
    lc.dynamicSmemBytes = shm;
    lc.stream = st;
    lc.attrs = at;
    lc.numAttrs = 1;
    lc.gridDim = dim3(unsigned(sm_count() / 2 * 2));
    int ncl = 0;
    MS_CUDA_TRY(cudaOccupancyMaxActiveClusters(&ncl, kern, &lc));
    lc.gridDim = dim3(unsigned(2 * (ncl > 0 ? ncl : 1)));
    MS_CUDA_TRY(cudaLaunchKernelEx(&lc, kern, kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, cfg, gt, hits,
                                   d_err));
    return MS_OK;
}

template <int W>
int launch_q3_tma_w(const ColView &kv, const ColView &gv, const ColView &mv, const StreamCol &s0, const StreamCol &s1,
                    const StreamCol &s2, const StreamCol &s3, const Pred &pred, const uint32_t *bits, uint64_t nwords,
                    uint64_t lo, uint64_t span, const GTable &gt, uint32_t *hits, unsigned *d_err, cudaStream_t st) {
    QCfg cfg{g_q3.stages, g_q3.stage_bytes};
    const size_t table = 3ull * 8 * kQSlots, bitmap = 4 * nwords, half = 4 * ((nwords + 1) / 2);
    const size_t meta = q3_meta_bytes(cfg.stages);
    const size_t ring = size_t(cfg.stages) * cfg.stage_bytes;
    // staged 1: the bitmap in shared memory beside the configured ring when
    // it fits, else in global memory.  staged 3: split over a 2-CTA cluster,
    // the ring's stages shrunk to make room (down to 24 KiB).  Both ways of
    // making room for a large bitmap were measured slower than reading it
    // from global memory: for a 2^20-key build side a 2 x 25 KiB ring with
    // the whole bitmap lost more to the shallower pipeline than the probes
    // gained, and the cluster split (3 x 38 KiB ring, half the bitmap per
    // CTA) took 242 us at 2^26 fact rows against 198 us, its distributed
    // shared-memory probes stalling longer than the L2 ones.
    const auto fit_stage = [&](size_t words_bytes) -> unsigned {
        if (meta + table + words_bytes >= kQSmemMax) return 0;
        const size_t room = kQSmemMax - meta - table - words_bytes;
        const size_t sb = minu(cfg.stage_bytes, room / cfg.stages / 128 * 128);
        return sb >= 24576 ? unsigned(sb) : 0;
    };
    int mode = kBmGlobal;
    if (g_q3.staged == 1 && meta + ring + table + bitmap <= kQSmemMax) mode = kBmShared;
    else if (g_q3.staged == 3 && fit_stage(half)) mode = kBmCluster;
    if (mode == kBmCluster) cfg.stage_bytes = fit_stage(half);
    const size_t shm = meta + size_t(cfg.stages) * cfg.stage_bytes + table +
                       (mode == kBmShared ? bitmap : mode == kBmCluster ? half : 0);
    switch (mode) {
    case kBmShared:
        return launch_q3_kern<W, kBmShared>(shm, cfg, kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt,
                                            hits, d_err, st);
    case kBmCluster:
        return launch_q3_kern<W, kBmCluster>(shm, cfg, kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt,
                                             hits, d_err, st);
    default:
        return launch_q3_kern<W, kBmGlobal>(shm, cfg, kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt,
                                            hits, d_err, st);
    }
}

int launch_q3_tma(const ColView &kv, const ColView &gv, const ColView &mv, const StreamCol &s0, const StreamCol &s1,
                  const StreamCol &s2, const StreamCol &s3, const Pred &pred, const uint32_t *bits, uint64_t nwords,
                  uint64_t lo, uint64_t span, const GTable &gt, uint32_t *hits, unsigned *d_err, cudaStream_t st) {
    switch (g_q3.warps) {
    case 8: return launch_q3_tma_w<8>(kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt, hits, d_err, st);
    case 24: return launch_q3_tma_w<24>(kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt, hits, d_err, st);
    default: return launch_q3_tma_w<16>(kv, gv, mv, s0, s1, s2, s3, pred, bits, nwords, lo, span, gt, hits, d_err, st);
    }
}

}  // namespace
}  // namespace ms

using namespace ms;

// Launch configuration of the fused query's staged kernel: staged (0 = the
// direct kernel only, 1 = staged with the build-side bitmap in shared memory
// when it fits beside the ring, 2 = staged with the bitmap in global memory,
// 3 = staged with the bitmap split over a 2-CTA cluster), warps
// (consumer warps: 8, 16 or 24), stages and
// stage_bytes (shared-memory ring; stages x stage_bytes + 48 KiB group table
// must fit 227 KiB).  The other fields are ignored.
extern "C" int ms_gpu_set_query_tuning(const ms_tuning *t) {
    if (!t) return ms_fail(MS_ERR_INVALID, "set_query_tuning: null");
    if (t->staged > 3) return ms_fail(MS_ERR_INVALID, "set_query_tuning: staged must be 0, 1, 2 or 3");
    if (t->warps != 8 && t->warps != 16 && t->warps != 24)
        return ms_fail(MS_ERR_INVALID, "set_query_tuning: warps must be 8, 16 or 24");
    if (t->stages < 2 || t->stages > 16 || t->stage_bytes % 128 || t->stage_bytes < 16384)
        return ms_fail(MS_ERR_INVALID, "set_query_tuning: stages in 2..16, stage_bytes a multiple of 128, >= 16 KiB");
    if (q3_meta_bytes(t->stages) + uint64_t(t->stages) * t->stage_bytes + 3ull * 8 * kQSlots > 232448)
        return ms_fail(MS_ERR_INVALID, "set_query_tuning: shared memory above 227 KiB");
    g_q3 = *t;
    return MS_OK;
}

extern "C" int ms_gpu_query3_last_pass_ms(double *ms) {
    if (!ms) return ms_fail(MS_ERR_INVALID, "query3_last_pass_ms: null");
    *ms = g_q3_pass_ms;
    return MS_OK;
}

extern "C" int ms_gpu_get_query_tuning(ms_tuning *t) {
    if (!t) return ms_fail(MS_ERR_INVALID, "get_query_tuning: null");
    *t = g_q3;
    return MS_OK;
}

// The fused query.  Outputs (host arrays of capacity `cap`): group keys, the
// group extents (first position of each group within P, as group_vec
// returns them) and the grouped sums, in group-id order; *n_groups.
// The build side `l` must span at most 2^30 values (a dense bitmap).
extern "C" int ms_gpu_query3(const ms_col *filter, int cmp, uint64_t c, const ms_col *fk, const ms_col *l,
                             const ms_col *gkey, const ms_col *measure, uint64_t cap, uint64_t *h_keys,
                             uint64_t *h_ext, uint64_t *h_sums, uint64_t *n_groups, uint64_t *n_rows_p,
                             ms_arena *a, void *stream) {
    if (!filter || !fk || !l || !gkey || !measure || !n_groups || !a) return ms_fail(MS_ERR_INVALID, "query3: null");
    const uint64_t n = filter->count_values;
    if (fk->count_values != n || gkey->count_values != n || measure->count_values != n)
        return ms_fail(MS_ERR_INVALID, "query3: fact columns differ in length");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t mark0 = a->used;  // everything below is scratch
    ColView fv, kv, gv, mv, lv;
    int rc;
    if ((rc = prepare_view(filter, a, st, &fv)) || (rc = prepare_view(fk, a, st, &kv)) ||
        (rc = prepare_view(gkey, a, st, &gv)) || (rc = prepare_view(measure, a, st, &mv)) ||
        (rc = prepare_view(l, a, st, &lv)))
        return rc;
    // build side bitmap
    unsigned long long *mm = arena_take_t<unsigned long long>(a, 2);
    if (!mm) return ms_fail(MS_ERR_NOMEM, "arena exhausted (query3)");
    const unsigned long long init[2] = {~0ull, 0ull};
    MS_CUDA_TRY(cudaMemcpyAsync(mm, init, 16, cudaMemcpyHostToDevice, st));
    const unsigned grid = unsigned(maxu(1, minu((lv.nblocks_total() + 7) / 8, persistent_grid(256, 8))));
    if (lv.n) {
        k_minmax_q<<<grid, 256, 0, st>>>(lv, mm, mm + 1, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    unsigned long long hmm[2];
    MS_CUDA_TRY(cudaMemcpyAsync(hmm, mm, 16, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t lo = 0, span = 0;
    if (lv.n) {
        lo = hmm[0];
        if (hmm[1] - hmm[0] >= (uint64_t(1) << 30))
            return ms_fail(MS_ERR_UNSUPPORTED, "query3: build keys span more than 2^30");
        span = hmm[1] - hmm[0] + 1;
    }
    const uint64_t words = (span + 31) / 32 + 1;
    uint32_t *bits = arena_take_t<uint32_t>(a, words);
    if (!bits) return ms_fail(MS_ERR_NOMEM, "arena exhausted (query3)");
    MS_CUDA_TRY(cudaMemsetAsync(bits, 0, 4 * words, st));
    if (lv.n) {
        k_q3_bits<<<grid, 256, 0, st>>>(lv, lo, bits, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    const uint64_t nbt = fv.nblocks_total();
    // The global group table starts at 2^16 slots and grows by 16x (up to
    // 2^24) when it fills, re-running the pass.
    uint64_t slots = uint64_t(1) << 16;
    std::vector<uint64_t> rec;  // (key, extent, sum, first row) per group
    uint64_t ng = 0, np = 0;
    for (;;) {
        const uint64_t mark = a->used;
        uint32_t *hits = arena_take_t<uint32_t>(a, nbt + 1);
        uint64_t *boff = arena_take_t<uint64_t>(a, nbt + 1);
        uint64_t *tot = arena_take_t<uint64_t>(a, 1);
        uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nbt, 1));
        GTable gt{arena_take_t<unsigned long long>(a, slots), arena_take_t<unsigned long long>(a, slots),
                  arena_take_t<unsigned long long>(a, slots), slots - 1};
        unsigned long long *cnt = arena_take_t<unsigned long long>(a, 1);
        uint64_t *out = arena_take_t<uint64_t>(a, 4 * slots);
        if (!hits || !boff || !tot || !scr || !gt.keys || !gt.first || !gt.sums || !cnt || !out)
            return ms_fail(MS_ERR_NOMEM, "arena exhausted (query3)");
        MS_CUDA_TRY(cudaMemsetAsync(gt.keys, 0xFF, 8 * slots, st));
        MS_CUDA_TRY(cudaMemsetAsync(gt.first, 0xFF, 8 * slots, st));
        MS_CUDA_TRY(cudaMemsetAsync(gt.sums, 0, 8 * slots, st));
        MS_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8, st));
        MS_CUDA_TRY(cudaMemsetAsync(tot, 0, 8, st));
        if (!g_q3_ev[0]) {
            MS_CUDA_TRY(cudaEventCreate(&g_q3_ev[0]));
            MS_CUDA_TRY(cudaEventCreate(&g_q3_ev[1]));
        }
        MS_CUDA_TRY(cudaEventRecord(g_q3_ev[0], st));
        if (nbt) {
            uint64_t nbs = 0;  // blocks through the staged kernel
            if (g_q3.staged && plain(fv) && random_access(kv) && random_access(gv) && random_access(mv)) {
                const StreamCol s0 = stream_of(fv), s1 = stream_of(kv), s2 = stream_of(gv), s3 = stream_of(mv);
                nbs = minu(minu(s0.nb, s1.nb), minu(s2.nb, s3.nb));
                if (nbs) {
                    rc = launch_q3_tma(kv, gv, mv, s0, s1, s2, s3, make_pred(cmp, c), bits, words, lo, span, gt,
                                       hits, a->d_err, st);
                    if (rc) return rc;
                }
            }
            if (nbt > nbs) {
                const unsigned g2 = unsigned(maxu(1, minu((nbt - nbs + 7) / 8, persistent_grid(256, 4))));
                k_query3<<<g2, 256, 0, st>>>(fv, kv, gv, mv, cmp, c, bits, lo, span, gt, hits, nbs, a->d_err);
                MS_CUDA_TRY(cudaGetLastError());
            }
            MS_CUDA_TRY(cudaEventRecord(g_q3_ev[1], st));
            MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(hits, nbt, boff, tot, scr, st)));
            k_q3_extents<<<unsigned(minu(slots / 8, 4096)), 256, 0, st>>>(
                gt, fv, kv, cmp, c, bits, lo, span, boff, cnt, out, a->d_err);
            MS_CUDA_TRY(cudaGetLastError());
        }
        // counts, error word and the first kQFirstGroups records in one
        // read-back; more groups take a second copy
        unsigned herr = 0;
        uint64_t hc[2] = {0, 0};
        const uint64_t first = minu(slots, kQFirstGroups);
        rec.resize(4 * first);
        MS_CUDA_TRY(cudaMemcpyAsync(&herr, a->d_err, sizeof herr, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaMemcpyAsync(hc, cnt, 8, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaMemcpyAsync(hc + 1, tot, 8, cudaMemcpyDeviceToHost, st));
        if (nbt) MS_CUDA_TRY(cudaMemcpyAsync(rec.data(), out, 32 * first, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        if (herr == kErrCapacity && slots < (uint64_t(1) << 24)) {
            MS_CUDA_TRY(cudaMemsetAsync(a->d_err, 0, sizeof herr, st));
            a->used = mark;
            slots <<= 4;
            continue;
        }
        rc = read_err(a, st);
        if (rc) return rc;
        float pass_ms = 0;
        if (nbt && cudaEventElapsedTime(&pass_ms, g_q3_ev[0], g_q3_ev[1]) == cudaSuccess) g_q3_pass_ms = pass_ms;
        ng = hc[0];
        np = hc[1];
        if (ng > first) {
            rec.resize(4 * ng);
            MS_CUDA_TRY(cudaMemcpyAsync(rec.data() + 4 * first, out + 4 * first, 32 * (ng - first),
                                        cudaMemcpyDeviceToHost, st));
            MS_CUDA_TRY(cudaStreamSynchronize(st));
        }
        break;
    }
    a->used = mark0;
    // group ids follow the first occurrence: order by first row
    std::vector<uint64_t> idx(ng);
    for (uint64_t i = 0; i < ng; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return rec[4 * x + 3] < rec[4 * y + 3]; });
    *n_groups = ng;
    if (n_rows_p) *n_rows_p = np;
    if (ng > cap) return ms_fail(MS_ERR_NOMEM, "query3: more groups than the output capacity");
    for (uint64_t i = 0; i < ng; i++) {
        if (h_keys) h_keys[i] = rec[4 * idx[i]];
        if (h_ext) h_ext[i] = rec[4 * idx[i] + 1];
        if (h_sums) h_sums[i] = rec[4 * idx[i] + 2];
    }
    return MS_OK;
}
