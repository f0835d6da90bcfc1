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
// global table at the end.  Each key keeps the smallest (row, rank of the row
// among P in its block) pair, so after a scan of the per-block hit counts the
// group's extent -- its first position in P, which is what the reference's
// group operator returns -- is exact, and ordering groups by first row gives
// the reference's group ids.  The result equals the operator-at-a-time
// pipeline's bit for bit; no intermediate touches HBM.
#include <algorithm>
#include <vector>

#include "internal.h"
#include "scan.cuh"

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
    unsigned long long *first;  // (row << 9) | rank of the row among the block's hits
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
                                               unsigned *err) {
    __shared__ unsigned long long s_key[kQSlots], s_first[kQSlots], s_sum[kQSlots];
    for (unsigned i = threadIdx.x; i < kQSlots; i += blockDim.x) {
        s_key[i] = kQEmpty;
        s_first[i] = ~0ull;
        s_sum[i] = 0;
    }
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true, fit = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < filt.nblocks_total();
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
        unsigned rank[16];
        block_ranks(m, l, q, rank);
        uint64_t g[16], w[16];
        unsigned vg, vm;
        ok &= decode_block(gkey, b, l, q, g, vg);
        ok &= decode_block(meas, b, l, q, w, vm);
        const uint64_t row0 = b * kBlock;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const bool hit = (m >> k) & 1u;
            const uint64_t key = g[k];
            const uint64_t first = ((row0 + (16u * q + k) * 8u + l) << 9) | rank[k];
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

// extent of every group: hits in earlier blocks + rank within its block
__global__ void k_q3_extents(GTable gt, const uint64_t *__restrict__ blk_off, unsigned long long *__restrict__ ext,
                             unsigned long long *__restrict__ row) {
    for (uint64_t h = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; h <= gt.mask; h += uint64_t(gridDim.x) * blockDim.x) {
        if (gt.keys[h] == kQEmpty) continue;
        const uint64_t f = gt.first[h];
        const uint64_t r = f >> 9;
        ext[h] = blk_off[r / kBlock] + (f & 511u);
        row[h] = r;
    }
}

}  // namespace
}  // namespace ms

using namespace ms;

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
        span = hmm[1] - hmm[0] + 1;
        if (span > (uint64_t(1) << 30)) return ms_fail(MS_ERR_UNSUPPORTED, "query3: build keys span more than 2^30");
    }
    const uint64_t words = (span + 31) / 32 + 1;
    uint32_t *bits = arena_take_t<uint32_t>(a, words);
    const uint64_t nbt = fv.nblocks_total();
    uint32_t *hits = arena_take_t<uint32_t>(a, nbt + 1);
    uint64_t *boff = arena_take_t<uint64_t>(a, nbt + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 1);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nbt, 1));
    const uint64_t slots = 1 << 16;
    GTable gt{arena_take_t<unsigned long long>(a, slots), arena_take_t<unsigned long long>(a, slots),
              arena_take_t<unsigned long long>(a, slots), slots - 1};
    unsigned long long *ext = arena_take_t<unsigned long long>(a, slots);
    unsigned long long *row = arena_take_t<unsigned long long>(a, slots);
    if (!bits || !hits || !boff || !tot || !scr || !gt.keys || !gt.first || !gt.sums || !ext || !row)
        return ms_fail(MS_ERR_NOMEM, "arena exhausted (query3)");
    MS_CUDA_TRY(cudaMemsetAsync(bits, 0, 4 * words, st));
    MS_CUDA_TRY(cudaMemsetAsync(gt.keys, 0xFF, 8 * slots, st));
    MS_CUDA_TRY(cudaMemsetAsync(gt.first, 0xFF, 8 * slots, st));
    MS_CUDA_TRY(cudaMemsetAsync(gt.sums, 0, 8 * slots, st));
    if (lv.n) {
        k_q3_bits<<<grid, 256, 0, st>>>(lv, lo, bits, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    if (nbt) {
        const unsigned g2 = unsigned(maxu(1, minu((nbt + 7) / 8, persistent_grid(256, 4))));
        k_query3<<<g2, 256, 0, st>>>(fv, kv, gv, mv, cmp, c, bits, lo, span, gt, hits, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(hits, nbt, boff, tot, scr, st)));
        k_q3_extents<<<64, 256, 0, st>>>(gt, boff, ext, row);
        MS_CUDA_TRY(cudaGetLastError());
    }
    rc = read_err(a, st);
    if (rc) return rc;
    // collect on the host (at most `slots` groups) and order by first row
    std::vector<uint64_t> k(slots), e(slots), s(slots), r(slots);
    uint64_t np = 0;
    if (nbt) {
        MS_CUDA_TRY(cudaMemcpy(k.data(), gt.keys, 8 * slots, cudaMemcpyDeviceToHost));
        MS_CUDA_TRY(cudaMemcpy(e.data(), ext, 8 * slots, cudaMemcpyDeviceToHost));
        MS_CUDA_TRY(cudaMemcpy(s.data(), gt.sums, 8 * slots, cudaMemcpyDeviceToHost));
        MS_CUDA_TRY(cudaMemcpy(r.data(), row, 8 * slots, cudaMemcpyDeviceToHost));
        MS_CUDA_TRY(cudaMemcpy(&np, tot, 8, cudaMemcpyDeviceToHost));
    }
    std::vector<uint64_t> idx;
    for (uint64_t h = 0; h < (nbt ? slots : 0); h++)
        if (k[h] != kQEmpty) idx.push_back(h);
    std::sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return r[x] < r[y]; });
    *n_groups = idx.size();
    if (n_rows_p) *n_rows_p = np;
    if (idx.size() > cap) return ms_fail(MS_ERR_NOMEM, "query3: more groups than the output capacity");
    for (size_t i = 0; i < idx.size(); i++) {
        if (h_keys) h_keys[i] = k[idx[i]];
        if (h_ext) h_ext[i] = e[idx[i]];
        if (h_sums) h_sums[i] = s[idx[i]];
    }
    return MS_OK;
}
