// join_group.cu -- semi_join, intersect_sorted, group and grouped agg_sum
// with decompression fused into the probe / grouping kernels.
//
// Membership (semi_join build side): when the build keys span at most 2^27
// values the set is a dense bitmap (exact, one bit per value; kept in
// shared memory when it fits 128 KB), otherwise an open-addressing hash set
// in global memory (linear probing, 64-bit multiplicative hash).  The
// reference uses a vectorised linear-probing hash set
// (vector/datastructures/hash_based/hash_set.h:32-149); results do not
// depend on the table, only on set membership.
//
// Grouping: a global hash table maps each key to the smallest row where it
// occurs (atomicMin); flags at those rows, scanned, give every group its id
// in order of first occurrence -- exactly the reference's ids
// (linear_probing.h:437-443, scalar/group_uncompr.h:105-114) -- and the
// flagged rows in order are the group extents.
#include "internal.h"
#include "scan.cuh"

namespace ms {

int gather_values(const ms_col *data, const uint64_t *d_pos, uint64_t npos, uint64_t *d_out, ms_arena *a,
                  cudaStream_t st);

namespace {

constexpr uint64_t kEmpty = ~uint64_t(0);

__device__ __forceinline__ uint64_t hash64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xFF51AFD7ED558CCDull;
    k ^= k >> 33;
    k *= 0xC4CEB9FE1A85EC53ull;
    k ^= k >> 33;
    return k;
}

struct KeySet {
    // bitmap mode
    const uint32_t *bits;  // global bitmap (nullptr in hash mode)
    uint64_t lo;           // smallest key
    uint64_t span;         // bits in the bitmap
    // hash mode
    const uint64_t *slots;
    uint64_t mask;
    int has_max;           // key 2^64-1 present (it doubles as the empty marker)
};

__device__ __forceinline__ bool set_contains(const KeySet &s, const uint32_t *sbits, uint64_t k) {
    if (s.bits) {
        const uint64_t d = k - s.lo;
        if (k < s.lo || d >= s.span) return false;
        const uint32_t *b = sbits ? sbits : s.bits;
        return (b[d >> 5] >> (d & 31u)) & 1u;
    }
    if (k == kEmpty) return s.has_max;
    uint64_t h = hash64(k) & s.mask;
    for (uint64_t probe = 0; probe <= s.mask; probe++) {
        const uint64_t v = s.slots[h];
        if (v == k) return true;
        if (v == kEmpty) return false;
        h = (h + 1) & s.mask;
    }
    return false;
}

__global__ void k_minmax(ColView c, unsigned long long *mn, unsigned long long *mx, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    uint64_t lo = kEmpty, hi = 0;
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

__global__ void k_build_set(ColView c, uint32_t *bits, uint64_t lo, uint64_t *slots, uint64_t mask,
                            int *has_max, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < c.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(c, b, l, q, v, valid);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (!((valid >> k) & 1u)) continue;
            const uint64_t key = v[k];
            if (bits) {
                const uint64_t d = key - lo;
                atomicOr(bits + (d >> 5), 1u << (d & 31u));
                continue;
            }
            if (key == kEmpty) {
                *has_max = 1;
                continue;
            }
            uint64_t h = hash64(key) & mask;
            bool placed = false;
            for (uint64_t probe = 0; probe <= mask; probe++) {
                const unsigned long long old =
                    atomicCAS((unsigned long long *)(slots + h), (unsigned long long)kEmpty, (unsigned long long)key);
                if (old == kEmpty || old == key) {
                    placed = true;
                    break;
                }
                h = (h + 1) & mask;
            }
            if (!placed) atomicOr(err, kErrCapacity);
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// Probe: per block, hits = rows of r whose value is in the set.  Pass 1
// (blk_off == nullptr) stores per-block counts, pass 2 writes positions.
constexpr unsigned kSmemBitmapWords = 32768;  // 128 KB

template <bool kSmem>
__global__ void __launch_bounds__(256) k_probe(ColView r, KeySet s, uint32_t *__restrict__ blk_counts,
                                              const uint64_t *__restrict__ blk_off, uint64_t *__restrict__ out_pos,
                                              unsigned long long *__restrict__ d_scalar_hits, unsigned *err) {
    extern __shared__ uint32_t sbits[];
    if (kSmem) {
        const uint64_t words = (s.span + 31) / 32;
        for (uint64_t i = threadIdx.x; i < words; i += blockDim.x) sbits[i] = s.bits[i];
        __syncthreads();
    }
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < r.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(r, b, l, q, v, valid);
        unsigned m = 0;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((valid >> k) & 1u) m |= unsigned(set_contains(s, kSmem ? sbits : nullptr, v[k])) << k;
        if (!blk_off) {
            const unsigned tot = __reduce_add_sync(0xFFFFFFFFu, __popc(m));
            if (lane == 0) blk_counts[b] = tot;
            continue;
        }
        if (!__any_sync(0xFFFFFFFFu, m != 0)) continue;
        unsigned rank[16];
        block_ranks(m, l, q, rank);
        const uint64_t base = blk_off[b], row0 = b * kBlock;
        unsigned scal = 0;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((m >> k) & 1u) {
                const uint64_t row = row0 + (16u * q + k) * 8u + l;
                out_pos[base + rank[k]] = row;
                scal += row >= r.sfrom;
            }
        if (scal) atomicAdd(d_scalar_hits, (unsigned long long)scal);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// ---------------------------------------------------------------------------
// Natural equi-join (join_natural_equi_compr.h:116-300): the build side maps
// every key to the position of its first occurrence (the reference's hash
// map keeps the value of the first insert, linear_probing.h:315-366).  Dense
// key ranges use a direct array of positions, others an open-addressing
// table; both are filled with atomicMin, so the result does not depend on the
// order in which warps insert.
// ---------------------------------------------------------------------------
struct KeyMap {
    unsigned long long *dense;  // dense mode: position per key - lo (~0: absent)
    uint64_t lo, span;
    unsigned long long *keys;   // hash mode
    unsigned long long *vals;
    uint64_t mask;
    unsigned long long *max_pos;  // position of key 2^64-1 (it doubles as the empty marker)
};

__device__ __forceinline__ uint64_t map_lookup(const KeyMap &m, uint64_t k) {
    if (m.dense) {
        const uint64_t d = k - m.lo;
        return (k < m.lo || d >= m.span) ? kEmpty : m.dense[d];
    }
    if (k == kEmpty) return *m.max_pos;
    uint64_t h = hash64(k) & m.mask;
    for (uint64_t probe = 0; probe <= m.mask; probe++) {
        const uint64_t v = m.keys[h];
        if (v == k) return m.vals[h];
        if (v == kEmpty) return kEmpty;
        h = (h + 1) & m.mask;
    }
    return kEmpty;
}

__global__ void k_build_map(ColView c, KeyMap m, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < c.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(c, b, l, q, v, valid);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (!((valid >> k) & 1u)) continue;
            const uint64_t key = v[k];
            const unsigned long long row = b * kBlock + (16u * q + k) * 8u + l;
            if (m.dense) {
                atomicMin(m.dense + (key - m.lo), row);
                continue;
            }
            if (key == kEmpty) {
                atomicMin(m.max_pos, row);
                continue;
            }
            uint64_t h = hash64(key) & m.mask;
            bool placed = false;
            for (uint64_t probe = 0; probe <= m.mask; probe++) {
                const unsigned long long old = atomicCAS(m.keys + h, (unsigned long long)kEmpty, (unsigned long long)key);
                if (old == kEmpty || old == key) {
                    atomicMin(m.vals + h, row);
                    placed = true;
                    break;
                }
                h = (h + 1) & m.mask;
            }
            if (!placed) atomicOr(err, kErrCapacity);
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// Probe: per block, hits = rows of r whose value is a key.  Pass 1
// (blk_off == nullptr) stores per-block counts, pass 2 writes the pairs.
__global__ void __launch_bounds__(256) k_probe_map(ColView r, KeyMap m, uint32_t *__restrict__ blk_counts,
                                                  const uint64_t *__restrict__ blk_off, uint64_t *__restrict__ out_r,
                                                  uint64_t *__restrict__ out_l,
                                                  unsigned long long *__restrict__ d_scalar_hits, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < r.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(r, b, l, q, v, valid);
        unsigned mk = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint64_t p = ((valid >> k) & 1u) ? map_lookup(m, v[k]) : kEmpty;
            v[k] = p;  // the build position replaces the value
            mk |= unsigned(p != kEmpty) << k;
        }
        if (!blk_off) {
            const unsigned tot = __reduce_add_sync(0xFFFFFFFFu, __popc(mk));
            if (lane == 0) blk_counts[b] = tot;
            continue;
        }
        if (!__any_sync(0xFFFFFFFFu, mk != 0)) continue;
        unsigned rank[16];
        block_ranks(mk, l, q, rank);
        const uint64_t base = blk_off[b], row0 = b * kBlock;
        unsigned scal = 0;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((mk >> k) & 1u) {
                const uint64_t row = row0 + (16u * q + k) * 8u + l;
                out_r[base + rank[k]] = row;
                out_l[base + rank[k]] = v[k];
                scal += row >= r.sfrom;
            }
        if (scal) atomicAdd(d_scalar_hits, (unsigned long long)scal);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// intersect: rows of l (a sorted position list) whose value occurs in the
// sorted array rv; pass structure as k_probe, output = the values.
__global__ void __launch_bounds__(256) k_intersect(ColView lc, const uint64_t *__restrict__ rv, uint64_t nr,
                                                  uint32_t *__restrict__ blk_counts, const uint64_t *__restrict__ blk_off,
                                                  uint64_t *__restrict__ out, unsigned long long *__restrict__ d_scalar,
                                                  unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < lc.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16];
        unsigned valid;
        ok &= decode_block(lc, b, l, q, v, valid);
        unsigned m = 0;
        // the thread's 16 values ascend: galloping lower-bound searches
        uint64_t j = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (!((valid >> k) & 1u)) continue;
            const uint64_t x = v[k];
            uint64_t step = 1, lo = j, hi = j;
            while (hi < nr && rv[hi] < x) {
                lo = hi + 1;
                hi = j + step;
                step <<= 1;
            }
            if (hi > nr) hi = nr;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (rv[mid] < x) lo = mid + 1;
                else hi = mid;
            }
            j = lo;
            if (j < nr && rv[j] == x) m |= 1u << k;
        }
        if (!blk_off) {
            const unsigned tot = __reduce_add_sync(0xFFFFFFFFu, __popc(m));
            if (lane == 0) blk_counts[b] = tot;
            continue;
        }
        if (!__any_sync(0xFFFFFFFFu, m != 0)) continue;
        unsigned rank[16];
        block_ranks(m, l, q, rank);
        const uint64_t base = blk_off[b], row0 = b * kBlock;
        unsigned scal = 0;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if ((m >> k) & 1u) {
                out[base + rank[k]] = v[k];
                scal += (row0 + (16u * q + k) * 8u + l) >= lc.sfrom;
            }
        if (scal) atomicAdd(d_scalar, (unsigned long long)scal);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// --- group ------------------------------------------------------------------
struct GroupTable {
    uint64_t *ka;               // key (unary) / first key word (binary)
    uint64_t *kb;               // second key word (binary) or nullptr
    unsigned long long *first;  // smallest row of the key
    unsigned *state;            // 0 empty, 1 claimed, 2 key published
    unsigned long long *fill;   // claimed slots
    uint64_t mask;
    uint64_t limit;             // claims allowed before the table counts as full
};

__device__ __forceinline__ uint64_t hash_pair(uint64_t a, uint64_t b) { return hash64(a * 0x9E3779B97F4A7C15ull ^ b); }

enum { kInsOk = 0, kInsFull = 1, kInsTimeout = 2 };

// Insert (key, row): the slot is claimed by CAS 0 -> 1, the key written and
// published (state 2); every inserter lowers `first` with atomicMin.
__device__ __forceinline__ int group_insert(const GroupTable &t, uint64_t a, uint64_t b, uint64_t row) {
    uint64_t h = hash_pair(a, b) & t.mask;
    for (uint64_t probe = 0; probe <= t.mask; probe++) {
        const unsigned st = atomicCAS(t.state + h, 0u, 1u);
        if (st == 0) {
            if (atomicAdd(t.fill, 1ull) >= t.limit) {
                atomicExch(t.state + h, 0u);
                return kInsFull;
            }
            t.ka[h] = a;
            if (t.kb) t.kb[h] = b;
            __threadfence();
            atomicExch(t.state + h, 2u);
            atomicMin(t.first + h, (unsigned long long)row);
            return kInsOk;
        }
        unsigned spins = 0;
        while (*(volatile unsigned *)(t.state + h) == 1u && spins < kSpinLimit) spins++;
        if (spins >= kSpinLimit) return kInsTimeout;
        __threadfence();
        if (*(volatile unsigned *)(t.state + h) == 2u && ((volatile uint64_t *)t.ka)[h] == a &&
            (!t.kb || ((volatile uint64_t *)t.kb)[h] == b)) {
            atomicMin(t.first + h, (unsigned long long)row);
            return kInsOk;
        }
        h = (h + 1) & t.mask;
    }
    return kInsFull;
}

__device__ __forceinline__ bool group_find(const GroupTable &t, uint64_t a, uint64_t b, uint64_t &slot) {
    uint64_t h = hash_pair(a, b) & t.mask;
    for (uint64_t probe = 0; probe <= t.mask; probe++) {
        if (t.state[h] == 0) return false;
        if (t.ka[h] == a && (!t.kb || t.kb[h] == b)) {
            slot = h;
            return true;
        }
        h = (h + 1) & t.mask;
    }
    return false;
}

// pass A: insert every row's key with its row number
__global__ void __launch_bounds__(256) k_group_insert(ColView gin, bool binary, ColView c, GroupTable t,
                                                     unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    int bad = kInsOk;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < c.nblocks_total() && bad == kInsOk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16], g[16];
        unsigned valid, vg;
        ok &= decode_block(c, b, l, q, v, valid);
        if (binary) ok &= decode_block(gin, b, l, q, g, vg);
        const uint64_t row0 = b * kBlock;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (!((valid >> k) & 1u) || bad != kInsOk) continue;
            // unary: the key lives in ka; binary: (group, value) in (ka, kb)
            bad = group_insert(t, binary ? g[k] : v[k], binary ? v[k] : 0, row0 + (16u * q + k) * 8u + l);
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
    if (bad == kInsFull) atomicOr(err, kErrCapacity);
    if (bad == kInsTimeout) atomicOr(err, kErrTimeout);
}

// pass B: flag the first row of every group (bitmap over rows)
__global__ void k_group_flags(GroupTable t, uint32_t *__restrict__ flags) {
    for (uint64_t h = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; h <= t.mask; h += uint64_t(gridDim.x) * blockDim.x)
        if (t.state[h] == 2u) {
            const uint64_t r = t.first[h];
            atomicOr(flags + (r >> 5), 1u << (r & 31u));
        }
}

__global__ void k_popc_words(const uint32_t *__restrict__ flags, uint64_t nwords, uint32_t *__restrict__ cnt) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nwords; i += uint64_t(gridDim.x) * blockDim.x)
        cnt[i] = __popc(flags[i]);
}

// extents: the flagged rows in order
__global__ void k_group_extents(const uint32_t *__restrict__ flags, const uint64_t *__restrict__ woff, uint64_t nwords,
                                uint64_t *__restrict__ ext) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nwords; i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t f = flags[i];
        uint64_t o = woff[i];
        while (f) {
            const int k = __ffs(f) - 1;
            ext[o++] = i * 32 + k;
            f &= f - 1;
        }
    }
}

// pass C: group id of every row = rank of its group's first row
__global__ void __launch_bounds__(256) k_group_ids(ColView gin, bool binary, ColView c, GroupTable t,
                                                  const uint32_t *__restrict__ flags, const uint64_t *__restrict__ woff,
                                                  uint64_t *__restrict__ gr, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < c.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t v[16], g[16];
        unsigned valid, vg;
        ok &= decode_block(c, b, l, q, v, valid);
        if (binary) ok &= decode_block(gin, b, l, q, g, vg);
        const uint64_t row0 = b * kBlock;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (!((valid >> k) & 1u)) continue;
            uint64_t slot = 0;
            if (!group_find(t, binary ? g[k] : v[k], binary ? v[k] : 0, slot)) {
                ok = false;
                continue;
            }
            const uint64_t r = t.first[slot];
            const uint32_t below = flags[r >> 5] & ((1u << (r & 31u)) - 1u);
            gr[row0 + (16u * q + k) * 8u + l] = woff[r >> 5] + __popc(below);
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// --- grouped sum ----------------------------------------------------------------
constexpr unsigned kSmemGroups = 4096;

__global__ void __launch_bounds__(256) k_grouped_sum(ColView gc, ColView dc, uint64_t ngroups,
                                                    unsigned long long *__restrict__ out, unsigned *err) {
    __shared__ unsigned long long acc[kSmemGroups];
    const bool smem = ngroups <= kSmemGroups;
    if (smem)
        for (unsigned i = threadIdx.x; i < ngroups; i += blockDim.x) acc[i] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, q = lane >> 3;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < gc.nblocks_total();
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        uint64_t g[16], d[16];
        unsigned vg, vd;
        ok &= decode_block(gc, b, l, q, g, vg);
        ok &= decode_block(dc, b, l, q, d, vd);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const bool act = (vg >> k) & 1u;
            const uint64_t gid = g[k];
            if (act && gid >= ngroups) {
                ok = false;
                continue;
            }
            // warp-aggregated update: lanes with the same group add once
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, act ? gid : ~uint64_t(0));
            uint64_t s = act ? d[k] : 0;
            // sum over peers: shuffle-free reduction via the leader
            const int leader = __ffs(peers) - 1;
            unsigned rest = peers;
            uint64_t tot = 0;
            while (rest) {
                const int src = __ffs(rest) - 1;
                tot += __shfl_sync(peers, s, src);
                rest &= rest - 1;
            }
            if (act && int(lane) == leader) {
                if (smem) atomicAdd(&acc[gid], (unsigned long long)tot);
                else atomicAdd(out + gid, (unsigned long long)tot);
            }
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
    __syncthreads();
    if (smem)
        for (unsigned i = threadIdx.x; i < ngroups; i += blockDim.x)
            if (acc[i]) atomicAdd(out + i, acc[i]);
}

}  // namespace

static unsigned grid_blocks(uint64_t nbt) {
    return (unsigned)maxu(1, minu((nbt + 7) / 8, persistent_grid(256, 8)));
}

// Shared tail of position-producing operators: pass 1 counts, scan, pass 2
// writes; then the write iterator model.
template <class Launch>
static int positions_two_pass(uint64_t nbt, Launch launch, int out_format, unsigned out_bw, ms_col *out, ms_arena *a,
                              cudaStream_t st) {
    uint32_t *bc = arena_take_t<uint32_t>(a, nbt + 1);
    uint64_t *bo = arena_take_t<uint64_t>(a, nbt + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 2);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nbt, 1));
    if (!bc || !bo || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (positions)");
    MS_CUDA_TRY(cudaMemsetAsync(tot, 0, 16, st));
    if (nbt) {
        launch(bc, nullptr, nullptr, nullptr);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(bc, nbt, bo, tot, scr, st)));
    }
    uint64_t total = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t *pos = arena_take_t<uint64_t>(a, total + 1);
    if (!pos) return ms_fail(MS_ERR_NOMEM, "arena exhausted (positions output)");
    if (total) {
        launch(bc, bo, pos, (unsigned long long *)(tot + 1));
        MS_CUDA_TRY(cudaGetLastError());
    }
    uint64_t scal = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&scal, tot + 1, 8, cudaMemcpyDeviceToHost, st));
    int rc = read_err(a, st);
    if (rc) return rc;
    return write_values(pos, total - scal, scal, out_format, out_bw, out, a, st);
}

static int view_or_decompress(const ms_col *c, ms_arena *a, cudaStream_t st, ColView *v) {
    if (c->format != MS_FMT_RLE) return prepare_view(c, a, st, v);
    uint64_t *tmp = arena_take_t<uint64_t>(a, c->count_values + 1);
    if (!tmp) return ms_fail(MS_ERR_NOMEM, "arena exhausted (rle)");
    int rc = decompress_to(c, tmp, a, st);
    if (rc) return rc;
    *v = ColView{};
    v->fmt = MS_FMT_UNCOMPR;
    v->n = c->count_values;
    v->rest = tmp;
    v->sfrom = v->n - v->n % kStep;
    return MS_OK;
}

}  // namespace ms

using namespace ms;

extern "C" int ms_gpu_semi_join(const ms_col *l, const ms_col *r, int out_format, unsigned out_bw, ms_col *out,
                                ms_arena *a, void *stream) {
    if (!l || !r || !out || !a) return ms_fail(MS_ERR_INVALID, "semi_join: null argument");
    if (r->format == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "semi_join: rle_f probe side");
    cudaStream_t st = (cudaStream_t)stream;
    ColView lv, rv;
    int rc = view_or_decompress(l, a, st, &lv);
    if (rc) return rc;
    rc = prepare_view(r, a, st, &rv);
    if (rc) return rc;
    // build side range
    unsigned long long *mm = arena_take_t<unsigned long long>(a, 2);
    int *has_max = arena_take_t<int>(a, 1);
    if (!mm || !has_max) return ms_fail(MS_ERR_NOMEM, "arena exhausted (semi_join)");
    const unsigned long long init[2] = {~0ull, 0ull};
    MS_CUDA_TRY(cudaMemcpyAsync(mm, init, 16, cudaMemcpyHostToDevice, st));
    MS_CUDA_TRY(cudaMemsetAsync(has_max, 0, 4, st));
    const uint64_t nbl = lv.nblocks_total();
    if (nbl) {
        k_minmax<<<grid_blocks(nbl), 256, 0, st>>>(lv, mm, mm + 1, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    unsigned long long hmm[2];
    MS_CUDA_TRY(cudaMemcpyAsync(hmm, mm, 16, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    KeySet s{};
    const uint64_t nl = l->count_values;
    const bool bitmap = nl > 0 && (hmm[1] - hmm[0]) < (uint64_t(1) << 27);
    if (nl == 0) {
        s.bits = nullptr;
        s.slots = nullptr;
        s.mask = 0;
        uint64_t *one = arena_take_t<uint64_t>(a, 1);
        if (!one) return ms_fail(MS_ERR_NOMEM, "arena exhausted (semi_join)");
        MS_CUDA_TRY(cudaMemsetAsync(one, 0xFF, 8, st));
        s.slots = one;
    } else if (bitmap) {
        s.lo = hmm[0];
        s.span = hmm[1] - hmm[0] + 1;
        const uint64_t words = (s.span + 31) / 32;
        uint32_t *bits = arena_take_t<uint32_t>(a, words);
        if (!bits) return ms_fail(MS_ERR_NOMEM, "arena exhausted (semi_join bitmap)");
        MS_CUDA_TRY(cudaMemsetAsync(bits, 0, 4 * words, st));
        s.bits = bits;
        k_build_set<<<grid_blocks(nbl), 256, 0, st>>>(lv, bits, s.lo, nullptr, 0, has_max, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    } else {
        uint64_t cap = 16;
        while (cap < 2 * nl) cap <<= 1;
        uint64_t *slots = arena_take_t<uint64_t>(a, cap);
        if (!slots) return ms_fail(MS_ERR_NOMEM, "arena exhausted (semi_join table)");
        MS_CUDA_TRY(cudaMemsetAsync(slots, 0xFF, 8 * cap, st));
        s.slots = slots;
        s.mask = cap - 1;
        k_build_set<<<grid_blocks(nbl), 256, 0, st>>>(lv, nullptr, 0, slots, s.mask, has_max, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        int hm = 0;
        MS_CUDA_TRY(cudaMemcpyAsync(&hm, has_max, 4, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        s.has_max = hm;
    }
    const bool smem = s.bits && (s.span + 31) / 32 <= kSmemBitmapWords;
    const size_t shm = smem ? 4 * ((s.span + 31) / 32) : 0;
    if (smem && shm > 48 * 1024)
        MS_CUDA_TRY(cudaFuncSetAttribute(k_probe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm)));
    const uint64_t nbt = rv.nblocks_total();
    auto launch = [&](uint32_t *bc, const uint64_t *bo, uint64_t *pos, unsigned long long *scal) {
        if (smem)
            k_probe<true><<<grid_blocks(nbt), 256, shm, st>>>(rv, s, bc, bo, pos, scal, a->d_err);
        else
            k_probe<false><<<grid_blocks(nbt), 256, 0, st>>>(rv, s, bc, bo, pos, scal, a->d_err);
    };
    return positions_two_pass(nbt, launch, out_format, out_bw, out, a, st);
}

extern "C" int ms_gpu_intersect_sorted(const ms_col *l, const ms_col *r, int out_format, unsigned out_bw, ms_col *out,
                                       ms_arena *a, void *stream) {
    if (!l || !r || !out || !a) return ms_fail(MS_ERR_INVALID, "intersect_sorted: null argument");
    if (l->format == MS_FMT_RLE) return ms_fail(MS_ERR_UNSUPPORTED, "intersect_sorted: rle_f input");
    cudaStream_t st = (cudaStream_t)stream;
    ColView lv;
    int rc = prepare_view(l, a, st, &lv);
    if (rc) return rc;
    const uint64_t *rvals = (const uint64_t *)r->data;
    if (r->format != MS_FMT_UNCOMPR) {
        uint64_t *tmp = arena_take_t<uint64_t>(a, r->count_values + 1);
        if (!tmp) return ms_fail(MS_ERR_NOMEM, "arena exhausted (intersect)");
        rc = decompress_to(r, tmp, a, st);
        if (rc) return rc;
        rvals = tmp;
    } else {
        rc = check_col(r, false);
        if (rc) return rc;
    }
    const uint64_t nr = r->count_values, nbt = lv.nblocks_total();
    auto launch = [&](uint32_t *bc, const uint64_t *bo, uint64_t *pos, unsigned long long *scal) {
        k_intersect<<<grid_blocks(nbt), 256, 0, st>>>(lv, rvals, nr, bc, bo, pos, scal, a->d_err);
    };
    return positions_two_pass(nbt, launch, out_format, out_bw, out, a, st);
}

extern "C" int ms_gpu_group(const ms_col *gr_in, const ms_col *in, int gr_format, ms_col *out_gr, int ext_format,
                            ms_col *out_ext, ms_arena *a, void *stream) {
    if (!in || !out_gr || !out_ext || !a) return ms_fail(MS_ERR_INVALID, "group: null argument");
    if (gr_in && gr_in->count_values != in->count_values)
        return ms_fail(MS_ERR_INVALID, "binary group: inGrCol and inDataCol must contain the same number of data elements");
    cudaStream_t st = (cudaStream_t)stream;
    ColView cv, gv{};
    int rc = view_or_decompress(in, a, st, &cv);
    if (rc) return rc;
    if (gr_in) {
        rc = view_or_decompress(gr_in, a, st, &gv);
        if (rc) return rc;
    }
    const uint64_t n = in->count_values;
    const uint64_t mark = a->used;
    uint64_t cap = 1024;
    for (;;) {
        a->used = mark;
        GroupTable t{};
        t.ka = arena_take_t<uint64_t>(a, cap);
        t.kb = gr_in ? arena_take_t<uint64_t>(a, cap) : nullptr;
        t.first = arena_take_t<unsigned long long>(a, cap);
        t.state = arena_take_t<unsigned>(a, cap);
        t.fill = arena_take_t<unsigned long long>(a, 1);
        t.mask = cap - 1;
        t.limit = cap / 2;
        if (!t.ka || !t.first || !t.state || !t.fill || (gr_in && !t.kb))
            return ms_fail(MS_ERR_NOMEM, "arena exhausted (group table)");
        MS_CUDA_TRY(cudaMemsetAsync(t.first, 0xFF, 8 * cap, st));
        MS_CUDA_TRY(cudaMemsetAsync(t.state, 0, 4 * cap, st));
        MS_CUDA_TRY(cudaMemsetAsync(t.fill, 0, 8, st));
        const uint64_t nbt = cv.nblocks_total();
        if (nbt) {
            k_group_insert<<<grid_blocks(nbt), 256, 0, st>>>(gv, gr_in != nullptr, cv, t, a->d_err);
            MS_CUDA_TRY(cudaGetLastError());
        }
        rc = read_err(a, st);
        if (rc == MS_ERR_NOMEM && cap < 4 * n + 4096) {
            cap *= 8;  // more distinct keys than the table holds: grow and redo
            continue;
        }
        if (rc) return rc;
        // first rows -> flags -> ranks
        const uint64_t nwords = (n + 31) / 32;
        uint32_t *flags = arena_take_t<uint32_t>(a, nwords + 1);
        uint32_t *wcnt = arena_take_t<uint32_t>(a, nwords + 1);
        uint64_t *woff = arena_take_t<uint64_t>(a, nwords + 1);
        uint64_t *ng = arena_take_t<uint64_t>(a, 1);
        uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nwords, 1));
        if (!flags || !wcnt || !woff || !ng || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (group flags)");
        MS_CUDA_TRY(cudaMemsetAsync(flags, 0, 4 * (nwords + 1), st));
        MS_CUDA_TRY(cudaMemsetAsync(ng, 0, 8, st));
        k_group_flags<<<persistent_grid(256, 8), 256, 0, st>>>(t, flags);
        MS_CUDA_TRY(cudaGetLastError());
        if (nwords) {
            k_popc_words<<<persistent_grid(256, 8), 256, 0, st>>>(flags, nwords, wcnt);
            MS_CUDA_TRY(cudaGetLastError());
            MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(wcnt, nwords, woff, ng, scr, st)));
        }
        uint64_t groups = 0;
        MS_CUDA_TRY(cudaMemcpyAsync(&groups, ng, 8, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaStreamSynchronize(st));
        uint64_t *ext = arena_take_t<uint64_t>(a, groups + 1);
        uint64_t *gr = arena_take_t<uint64_t>(a, n + 1);
        if (!ext || !gr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (group output)");
        if (nwords) {
            k_group_extents<<<persistent_grid(256, 8), 256, 0, st>>>(flags, woff, nwords, ext);
            MS_CUDA_TRY(cudaGetLastError());
        }
        if (nbt) {
            k_group_ids<<<grid_blocks(nbt), 256, 0, st>>>(gv, gr_in != nullptr, cv, t, flags, woff, gr, a->d_err);
            MS_CUDA_TRY(cudaGetLastError());
        }
        rc = read_err(a, st);
        if (rc) return rc;
        // outputs through the write iterators (group_compr.h:136-265): rows of
        // the input's scalar remainder, and the groups they open, are appended
        // uncompressed.
        const uint64_t sf = gr_in ? minu(cv.sfrom, gv.sfrom) : cv.sfrom;
        const uint64_t n_scal_rows = n - sf;
        uint64_t n_scal_groups = 0;
        if (n_scal_rows) {
            // extents are ascending: count those at rows >= sf on the host
            uint64_t tail[8] = {0};
            const uint64_t k = minu(groups, 8);
            if (k) MS_CUDA_TRY(cudaMemcpy(tail, ext + groups - k, 8 * k, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < k; i++) n_scal_groups += tail[i] >= sf;
        }
        rc = write_values(gr, n - n_scal_rows, n_scal_rows, gr_format, 0, out_gr, a, st);
        if (rc) return rc;
        return write_values(ext, groups - n_scal_groups, n_scal_groups, ext_format, 0, out_ext, a, st);
    }
}

extern "C" int ms_gpu_agg_sum_grouped(const ms_col *gr, const ms_col *data, uint64_t n_groups, ms_col *out,
                                      ms_arena *a, void *stream) {
    if (!gr || !data || !out || !a) return ms_fail(MS_ERR_INVALID, "agg_sum_grouped: null argument");
    if (gr->count_values != data->count_values)
        return ms_fail(MS_ERR_INVALID, "agg_sum: inGrCol and inDataCol must contain the same number of data elements");
    cudaStream_t st = (cudaStream_t)stream;
    ColView gv, dv;
    int rc = view_or_decompress(gr, a, st, &gv);
    if (rc) return rc;
    rc = view_or_decompress(data, a, st, &dv);
    if (rc) return rc;
    uint64_t *res = arena_take_t<uint64_t>(a, n_groups + 1);
    if (!res) return ms_fail(MS_ERR_NOMEM, "arena exhausted (grouped sum)");
    MS_CUDA_TRY(cudaMemsetAsync(res, 0, 8 * (n_groups + 1), st));
    const uint64_t nbt = gv.nblocks_total();
    if (nbt && n_groups) {
        k_grouped_sum<<<grid_blocks(nbt), 256, 0, st>>>(gv, dv, n_groups, (unsigned long long *)res, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    rc = read_err(a, st);
    if (rc) return rc;
    *out = ms_col{};
    out->format = MS_FMT_UNCOMPR;
    out->count_values = n_groups;
    out->size_used_byte = 8 * n_groups;
    out->size_alloc_byte = 8 * (n_groups + 1);
    out->data = res;
    return MS_OK;
}

// join<ve, outL_f, outR_f, L_f, R_f>(L, R) (join.h:158-187,
// join_natural_equi_compr.h:116-300): (build position, probe position)
// pairs in probe order; the two outputs follow the write iterator model in
// their formats.
extern "C" int ms_gpu_natural_join(const ms_col *l, const ms_col *r, int out_l_format, unsigned out_l_bw,
                                   int out_r_format, unsigned out_r_bw, ms_col *out_l, ms_col *out_r, ms_arena *a,
                                   void *stream) {
    if (!l || !r || !out_l || !out_r || !a) return ms_fail(MS_ERR_INVALID, "natural_join: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    ColView lv, rv;
    int rc = view_or_decompress(l, a, st, &lv);
    if (rc) return rc;
    rc = view_or_decompress(r, a, st, &rv);
    if (rc) return rc;
    unsigned long long *mm = arena_take_t<unsigned long long>(a, 3);
    if (!mm) return ms_fail(MS_ERR_NOMEM, "arena exhausted (natural_join)");
    const unsigned long long init[3] = {~0ull, 0ull, ~0ull};
    MS_CUDA_TRY(cudaMemcpyAsync(mm, init, 24, cudaMemcpyHostToDevice, st));
    const uint64_t nbl = lv.nblocks_total(), nl = l->count_values;
    if (nbl) {
        k_minmax<<<grid_blocks(nbl), 256, 0, st>>>(lv, mm, mm + 1, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    unsigned long long hmm[2];
    MS_CUDA_TRY(cudaMemcpyAsync(hmm, mm, 16, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    KeyMap m{};
    m.max_pos = mm + 2;
    if (nl && hmm[1] - hmm[0] < (uint64_t(1) << 24)) {
        m.lo = hmm[0];
        m.span = hmm[1] - hmm[0] + 1;
        m.dense = arena_take_t<unsigned long long>(a, m.span);
        if (!m.dense) return ms_fail(MS_ERR_NOMEM, "arena exhausted (natural_join array)");
        MS_CUDA_TRY(cudaMemsetAsync(m.dense, 0xFF, 8 * m.span, st));
    } else {
        uint64_t cap = 16;
        while (cap < 2 * nl) cap <<= 1;
        m.keys = arena_take_t<unsigned long long>(a, cap);
        m.vals = arena_take_t<unsigned long long>(a, cap);
        if (!m.keys || !m.vals) return ms_fail(MS_ERR_NOMEM, "arena exhausted (natural_join table)");
        MS_CUDA_TRY(cudaMemsetAsync(m.keys, 0xFF, 8 * cap, st));
        MS_CUDA_TRY(cudaMemsetAsync(m.vals, 0xFF, 8 * cap, st));
        m.mask = cap - 1;
    }
    if (nbl) {
        k_build_map<<<grid_blocks(nbl), 256, 0, st>>>(lv, m, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    // two passes over the probe side: counts, scan, pairs
    const uint64_t nbt = rv.nblocks_total();
    uint32_t *bc = arena_take_t<uint32_t>(a, nbt + 1);
    uint64_t *bo = arena_take_t<uint64_t>(a, nbt + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 2);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nbt, 1));
    if (!bc || !bo || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (natural_join)");
    MS_CUDA_TRY(cudaMemsetAsync(tot, 0, 16, st));
    if (nbt) {
        k_probe_map<<<grid_blocks(nbt), 256, 0, st>>>(rv, m, bc, nullptr, nullptr, nullptr, nullptr, a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
        MS_CUDA_TRY((scan_exclusive<uint32_t, 1>(bc, nbt, bo, tot, scr, st)));
    }
    uint64_t total = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&total, tot, 8, cudaMemcpyDeviceToHost, st));
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t *pr = arena_take_t<uint64_t>(a, total + 1);
    uint64_t *pl = arena_take_t<uint64_t>(a, total + 1);
    if (!pr || !pl) return ms_fail(MS_ERR_NOMEM, "arena exhausted (natural_join output)");
    if (total) {
        k_probe_map<<<grid_blocks(nbt), 256, 0, st>>>(rv, m, bc, bo, pr, pl, (unsigned long long *)(tot + 1),
                                                      a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    uint64_t scal = 0;
    MS_CUDA_TRY(cudaMemcpyAsync(&scal, tot + 1, 8, cudaMemcpyDeviceToHost, st));
    rc = read_err(a, st);
    if (rc) return rc;
    rc = write_values(pl, total - scal, scal, out_l_format, out_l_bw, out_l, a, st);
    if (rc) return rc;
    return write_values(pr, total - scal, scal, out_r_format, out_r_bw, out_r, a, st);
}

