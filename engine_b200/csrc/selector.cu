// selector.cu -- per-block format selection (the exhaustive judge and the
// learned selector's inputs) and the blockwise container.
//
// A column is cut into blocks of 2048 values.  Five candidate formats are
// evaluated per block exactly as the reference's morph_batch writes a
// 2048-value batch (default_formats.h:35-82):
//   static_vbp<bw>  bw = width of the block's largest value, 256*bw bytes
//   dynamic_vbp     one page: 64-B header + four vbp blocks
//   delta+dvbp      two 1024-blocks, each a page of two blocks; the lane-wise
//                   deltas start from zero at the block (delta.h:107-156)
//   for+dvbp        64-B FOR header + two pages (for.h:183-273)
//   rle             16 B per maximal run (rle.h:63-150)
// k_sel_analyze computes, in one read of the block, every sub-block width
// of every candidate, the FOR references and the run count -- i.e. the
// exact byte size of all five candidates (the size-only exhaustive pass).
// k_sel_encode writes a block in one chosen format; compress-all runs it for
// all five candidates into scratch, as the reference's exhaustive selector
// materialises every candidate (exhaustive_size_format_selector.h:56-72).
//
// The blockwise container follows blockwise_individual_f
// (blockwise_individual.h:89-99, 169-311): per block one format-code byte
// (format_selector_commons.h:25-103: static_vbp<bw> = bw, dynamic_vbp = 65,
// delta+dvbp = 67, for+dvbp = 69; rle, which the reference's container does
// not offer, = 71), padding to the next 64-B boundary, then the block's
// payload.
#include "internal.h"
#include "scan.cuh"

namespace ms {

constexpr unsigned kSelBlock = 2048;
constexpr unsigned kSelNF = 32;  // features per block
constexpr unsigned kSelNC = 5;   // candidates

enum : unsigned { kCandStatic = 0, kCandDvbp = 1, kCandDelta = 2, kCandFor = 3, kCandRle = 4 };

struct BlockStats {
    uint8_t raw[4];   // dynamic_vbp widths of the four 512-sub-blocks
    uint8_t dlt[4];   // widths of the deltas
    uint8_t fr[4];    // widths of the FOR offsets
    uint8_t sbw;      // static_vbp width
    uint8_t pad[3];
    uint32_t runs;    // maximal runs
    uint64_t ref[2];  // FOR references of the two 1024-halves
};

__host__ __device__ inline uint32_t cand_size(const BlockStats &s, unsigned c) {
    switch (c) {
    case kCandStatic: return 256u * s.sbw;
    case kCandDvbp: return 64u + 64u * (s.raw[0] + s.raw[1] + s.raw[2] + s.raw[3]);
    case kCandDelta: return 128u + 64u * (s.dlt[0] + s.dlt[1] + s.dlt[2] + s.dlt[3]);
    case kCandFor: return 192u + 64u * (s.fr[0] + s.fr[1] + s.fr[2] + s.fr[3]);
    default: return 16u * s.runs;
    }
}

__host__ __device__ inline uint8_t cand_code(const BlockStats &s, unsigned c) {
    switch (c) {
    case kCandStatic: return s.sbw;
    case kCandDvbp: return 65;
    case kCandDelta: return 67;
    case kCandFor: return 69;
    default: return 71;
    }
}

namespace {

__device__ __forceinline__ uint64_t wor(uint64_t x) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) x |= __shfl_xor_sync(0xFFFFFFFFu, x, s);
    return x;
}

// Analysis of one block by one warp.  Thread `lane` reads rows
// j = k*32 + lane (k = 0..63): row j belongs to sub-block k/16 and TVL lane
// j%8 = lane%8.
// U: unrolling of the four sub-block rounds (4: all 64 loads of a thread in
// flight; 1: a quarter of the registers, for kernels that want occupancy).
template <int U = 4>
__device__ BlockStats analyze_block(const uint64_t *__restrict__ x, unsigned lane) {
    BlockStats s;
    uint64_t prev = 0;       // x[j - 32] of this thread (previous k)
    uint64_t last_prev = 0;  // x[j - 1] for lane 0: lane 31 of the previous k
    unsigned heads = 0;
    // minima of the two 1024-halves; widths packed one byte per sub-block
    // (no register arrays indexed by the loop counter)
    int64_t mn0 = INT64_MAX, mn1 = INT64_MAX;
    uint32_t raw_p = 0, dlt_p = 0, fr_p = 0;
#pragma unroll U
    for (unsigned i = 0; i < 4; i++) {
        uint64_t o_raw = 1, o_dlt = 1;
        int64_t mi = INT64_MAX;
#pragma unroll
        for (unsigned kk = 0; kk < 16; kk++) {
            const unsigned k = i * 16 + kk;
            const uint64_t v = __ldg(x + k * 32 + lane);
            // x[j-8]: lane-8 of this k, or lane+24 of the previous k
            const uint64_t up8 = __shfl_up_sync(0xFFFFFFFFu, v, 8);
            const uint64_t pk = __shfl_sync(0xFFFFFFFFu, prev, (lane + 24) & 31u);
            const uint64_t x8 = lane >= 8 ? up8 : (k ? pk : 0);
            const uint64_t up1 = __shfl_up_sync(0xFFFFFFFFu, v, 1);
            const uint64_t x1 = lane >= 1 ? up1 : last_prev;
            heads += (k == 0 && lane == 0) ? 1u : unsigned(v != x1);
            o_raw |= v;
            o_dlt |= v - x8;
            mi = min(mi, (int64_t)v);
            last_prev = __shfl_sync(0xFFFFFFFFu, v, 31);
            prev = v;
        }
        if (i < 2) mn0 = min(mn0, mi);
        else mn1 = min(mn1, mi);
        raw_p |= uint32_t(effective_bitwidth(wor(o_raw))) << (8 * i);
        dlt_p |= uint32_t(effective_bitwidth(wor(o_dlt))) << (8 * i);
    }
    // FOR references: signed minimum per TVL lane, unsigned across lanes
#pragma unroll
    for (unsigned hh = 0; hh < 2; hh++) {
        int64_t m = hh ? mn1 : mn0;
        m = min(m, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (uint64_t)m, 8));
        m = min(m, (int64_t)__shfl_xor_sync(0xFFFFFFFFu, (uint64_t)m, 16));
        uint64_t um = (uint64_t)m;
        um = minu(um, __shfl_xor_sync(0xFFFFFFFFu, um, 1));
        um = minu(um, __shfl_xor_sync(0xFFFFFFFFu, um, 2));
        um = minu(um, __shfl_xor_sync(0xFFFFFFFFu, um, 4));
        if (um == ~uint64_t(0)) um--;
        s.ref[hh] = um;
    }
    // FOR offsets (second read of the block, from L1/L2)
#pragma unroll U
    for (unsigned i = 0; i < 4; i++) {
        uint64_t o = 1;
        const uint64_t ref = i < 2 ? s.ref[0] : s.ref[1];
#pragma unroll
        for (unsigned kk = 0; kk < 16; kk++) o |= __ldg(x + (i * 16 + kk) * 32 + lane) - ref;
        fr_p |= uint32_t(effective_bitwidth(wor(o))) << (8 * i);
    }
#pragma unroll
    for (unsigned i = 0; i < 4; i++) {
        s.raw[i] = uint8_t(raw_p >> (8 * i));
        s.dlt[i] = uint8_t(dlt_p >> (8 * i));
        s.fr[i] = uint8_t(fr_p >> (8 * i));
    }
    s.runs = __reduce_add_sync(0xFFFFFFFFu, heads);
    s.sbw = uint8_t(max(max(s.raw[0], s.raw[1]), max(s.raw[2], s.raw[3])));
    s.pad[0] = s.pad[1] = s.pad[2] = 0;
    return s;
}

__device__ __forceinline__ unsigned best_cand(const BlockStats &s) {
    unsigned best = 0;
    uint32_t bs = cand_size(s, 0);
    for (unsigned c = 1; c < kSelNC; c++)
        if (cand_size(s, c) < bs) {
            bs = cand_size(s, c);
            best = c;
        }
    return best;
}

__global__ void __launch_bounds__(256) k_sel_analyze(const uint64_t *__restrict__ in, uint64_t nblk,
                                                    BlockStats *__restrict__ st, uint32_t *__restrict__ sizes) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nblk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const BlockStats s = analyze_block(in + b * kSelBlock, lane);
        if (lane == 0) {
            st[b] = s;
            if (sizes)
                for (unsigned c = 0; c < kSelNC; c++) sizes[b * kSelNC + c] = cand_size(s, c);
        }
    }
}

// Exhaustive decision for the blocks the learned selector left open
// (choice 255); the others keep their choice.
// A warp reads the choices of its next 32 blocks (one per lane) in one go
// and analyses only the open ones.
__global__ void __launch_bounds__(256, 2) k_sel_resolve(const uint64_t *__restrict__ in, uint64_t nblk,
                                                       uint8_t *__restrict__ choice) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t W = uint64_t(gridDim.x) * blockDim.x / 32;
    for (uint64_t b0 = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b0 < nblk; b0 += 32 * W) {
        const uint64_t mine = b0 + lane * W;
        const bool open = mine < nblk && choice[mine] == 255;
        for (unsigned todo = __ballot_sync(0xFFFFFFFFu, open); todo; todo &= todo - 1) {
            const uint64_t b = b0 + uint64_t(__ffs(todo) - 1) * W;
            const BlockStats s = analyze_block<1>(in + b * kSelBlock, lane);
            if (lane == 0) choice[b] = uint8_t(best_cand(s));
        }
    }
}

// Footprint of a choice vector given exact sizes.
__global__ void k_sel_footprint(const uint32_t *__restrict__ sizes, const uint8_t *__restrict__ choice, uint64_t nblk,
                                unsigned long long *__restrict__ total) {
    uint64_t t = 0;
    for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < nblk; b += uint64_t(gridDim.x) * blockDim.x)
        t += sizes[b * kSelNC + (choice[b] < kSelNC ? choice[b] : 0)];
    for (int s = 16; s > 0; s >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, s);
    if ((threadIdx.x & 31u) == 0) atomicAdd(total, (unsigned long long)t);
}

// Write block b (values x) in candidate c at out (64-B aligned).  The warp's
// thread t packs lane t%8 of sub-block t/8.
__device__ void encode_block(const uint64_t *__restrict__ x, const BlockStats &s, unsigned c, uint8_t *__restrict__ out,
                             bool &ok) {
    const unsigned lane = threadIdx.x & 31u, i = lane >> 3, l = lane & 7u;
    const uint64_t *sub = x + i * 512;
    if (c == kCandRle) {
        // maximal runs: a head at row j if j == 0 or x[j] != x[j-1]; first
        // the value and start row of every run, then starts -> lengths
        uint64_t *o = reinterpret_cast<uint64_t *>(out);
        unsigned runs = 0;
        uint64_t last_prev = 0;
        for (unsigned k = 0; k < 64; k++) {
            const unsigned j = k * 32 + lane;
            const uint64_t v = __ldg(x + j);
            const uint64_t up1 = __shfl_up_sync(0xFFFFFFFFu, v, 1);
            const uint64_t x1 = lane >= 1 ? up1 : last_prev;
            const bool head = (j == 0) || v != x1;
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, head);
            if (head) {
                const unsigned r = runs + __popc(bal & ((1u << lane) - 1u));
                o[2 * r] = v;
                o[2 * r + 1] = j;
            }
            runs += __popc(bal);
            last_prev = __shfl_sync(0xFFFFFFFFu, v, 31);
        }
        __syncwarp();
        for (unsigned r0 = 0; r0 < runs; r0 += 32) {
            const unsigned r = r0 + lane;
            uint64_t start = 0, next = 0;
            if (r < runs) {
                start = o[2 * r + 1];
                next = r + 1 < runs ? o[2 * r + 3] : kSelBlock;
            }
            __syncwarp();
            if (r < runs) o[2 * r + 1] = next - start;
            __syncwarp();
        }
        return;
    }
    unsigned bw;
    uint64_t off;
    uint64_t ref = 0;
    bool dlt = false;
    switch (c) {
    case kCandStatic:
        bw = s.sbw;
        off = uint64_t(64) * bw * i;
        break;
    case kCandDvbp: {
        bw = s.raw[i];
        uint64_t acc = 0;
        for (unsigned k = 0; k < i; k++) acc += s.raw[k];
        off = 64 + 64 * acc;
        if (lane < 8) {  // page header: four widths, then 0xFF
            uint64_t hw = ~uint64_t(0);
            if (lane == 0)
                hw = (~uint64_t(0) << 32) | uint64_t(s.raw[0]) | (uint64_t(s.raw[1]) << 8) |
                     (uint64_t(s.raw[2]) << 16) | (uint64_t(s.raw[3]) << 24);
            reinterpret_cast<uint64_t *>(out)[lane] = hw;
        }
        break;
    }
    case kCandDelta:
    case kCandFor: {
        const bool isfor = c == kCandFor;
        const uint8_t *w = isfor ? s.fr : s.dlt;
        bw = w[i];
        const unsigned cb = i >> 1;  // 1024-block
        const uint64_t page0 = isfor ? 64 : 0;
        const uint64_t page = page0 + (cb ? 64 + 64 * uint64_t(w[0] + w[1]) : 0);
        off = page + 64 + ((i & 1) ? 64 * uint64_t(w[i - 1]) : 0);
        if (lane < 16) {  // inner headers of both pages (8 words each)
            const unsigned pc = lane >> 3, wi = lane & 7u;
            const uint64_t pg = page0 + (pc ? 64 + 64 * uint64_t(w[0] + w[1]) : 0);
            uint64_t hw = ~uint64_t(0);
            if (wi == 0) hw = (~uint64_t(0) << 16) | uint64_t(w[2 * pc]) | (uint64_t(w[2 * pc + 1]) << 8);
            reinterpret_cast<uint64_t *>(out + pg)[wi] = hw;
        }
        if (isfor) {
            ref = s.ref[cb];
            if (lane >= 16 && lane < 24) {  // FOR header: refs, end marker, zeros
                const unsigned wi = lane - 16;
                const uint64_t hw = wi < 2 ? s.ref[wi] : (wi == 2 ? ~uint64_t(0) : 0);
                reinterpret_cast<uint64_t *>(out)[wi] = hw;
            }
        } else {
            dlt = true;
        }
        break;
    }
    default: return;
    }
    auto get = [&](unsigned v) -> uint64_t {
        const unsigned r = v * 8 + l;
        uint64_t val = __ldg(sub + r);
        if (dlt) {
            const unsigned j = i * 512 + r;
            val -= j >= 8 ? __ldg(x + j - 8) : 0;
        } else {
            val -= ref;
        }
        return val;
    };
    ok &= vbp_pack_lane_rt(bw, get, reinterpret_cast<uint64_t *>(out + off), l);
}

// compress-all: every candidate of every block written to a per-warp scratch
// slot (5 x 32 KB), sizes from the stats.
constexpr unsigned kSlot = 32768;

__global__ void __launch_bounds__(256) k_sel_compress_all(const uint64_t *__restrict__ in, uint64_t nblk,
                                                         BlockStats *__restrict__ st, uint32_t *__restrict__ sizes,
                                                         uint8_t *__restrict__ scratch, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    uint8_t *slot = scratch + gw * kSelNC * kSlot;
    bool ok = true;
    for (uint64_t b = gw; b < nblk; b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const BlockStats s = st[b];
        for (unsigned c = 0; c < kSelNC; c++) encode_block(in + b * kSelBlock, s, c, slot + c * kSlot, ok);
        __syncwarp();
        if (lane < kSelNC) sizes[b * kSelNC + lane] = cand_size(s, lane);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

// Sampled statistics: four runs of 64 consecutive rows at 0, 512, 1024, 1536.
__global__ void __launch_bounds__(256) k_sel_features(const uint64_t *__restrict__ in, uint64_t nblk,
                                                     float *__restrict__ feats) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nblk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const uint64_t *x = in + b * kSelBlock;
        // bit-width histograms: eight 8-bit counters per thread in one word
        // (at most 8 values and 8 deltas per thread)
        uint64_t hv = 0, hd = 0;
        unsigned vmax = 0, vmin = 64, dmax = 0, neg = 0, heads = 0, zd = 0, vsum = 0, nd = 0;
        unsigned cmax[4] = {0}, cdmax[4] = {0};
        uint64_t umax = 0, umin = ~uint64_t(0);
#pragma unroll
        for (unsigned c = 0; c < 4; c++) {
            const uint64_t a = __ldg(x + 512 * c + lane), bq = __ldg(x + 512 * c + 32 + lane);
            // x[j-8] within the chunk and x[j-1]
            const uint64_t a8 = __shfl_up_sync(0xFFFFFFFFu, a, 8);
            const uint64_t b8a = __shfl_sync(0xFFFFFFFFu, a, (lane + 24) & 31u);
            const uint64_t b8b = __shfl_up_sync(0xFFFFFFFFu, bq, 8);
            const uint64_t b8 = lane < 8 ? b8a : b8b;
            const uint64_t a1 = __shfl_up_sync(0xFFFFFFFFu, a, 1);
            const uint64_t b1a = __shfl_sync(0xFFFFFFFFu, a, 31);
            const uint64_t b1b = __shfl_up_sync(0xFFFFFFFFu, bq, 1);
            const uint64_t b1 = lane == 0 ? b1a : b1b;
            const uint64_t vals[2] = {a, bq};
            for (unsigned u = 0; u < 2; u++) {
                const uint64_t v = vals[u];
                const unsigned bw = effective_bitwidth(v);
                hv += uint64_t(1) << (8u * ((bw - 1) >> 3));
                vmax = max(vmax, bw);
                vmin = min(vmin, bw);
                vsum += bw;
                cmax[c] = max(cmax[c], bw);
                umax = maxu(umax, v);
                umin = minu(umin, v);
            }
            if (lane >= 8) {
                const uint64_t d = a - a8;
                const unsigned bw = effective_bitwidth(d);
                hd += uint64_t(1) << (8u * ((bw - 1) >> 3));
                dmax = max(dmax, bw);
                cdmax[c] = max(cdmax[c], bw);
                neg += (int64_t)d < 0;
                zd += d == 0;
                nd++;
            }
            {
                const uint64_t d = bq - b8;
                const unsigned bw = effective_bitwidth(d);
                hd += uint64_t(1) << (8u * ((bw - 1) >> 3));
                dmax = max(dmax, bw);
                cdmax[c] = max(cdmax[c], bw);
                neg += (int64_t)d < 0;
                zd += d == 0;
                nd++;
            }
            if (lane >= 1) heads += a != a1;
            heads += bq != b1;
        }
        float f[kSelNF];
        const float nv = 256.f, ndf = float(__reduce_add_sync(0xFFFFFFFFu, nd));
        const float rnd = 1.f / ndf;  // one division; the delta features multiply by it
        // two counters per 32-bit word (16-bit fields: warp sums stay below 2^16)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const unsigned pv = unsigned((hv >> (16 * k)) & 0xFFu) | (unsigned((hv >> (16 * k + 8)) & 0xFFu) << 16);
            const unsigned pd = unsigned((hd >> (16 * k)) & 0xFFu) | (unsigned((hd >> (16 * k + 8)) & 0xFFu) << 16);
            const unsigned sv = __reduce_add_sync(0xFFFFFFFFu, pv), sd = __reduce_add_sync(0xFFFFFFFFu, pd);
            f[2 * k] = float(sv & 0xFFFFu) / nv;
            f[2 * k + 1] = float(sv >> 16) / nv;
            f[8 + 2 * k] = float(sd & 0xFFFFu) * rnd;
            f[8 + 2 * k + 1] = float(sd >> 16) * rnd;
        }
        f[16] = float(__reduce_max_sync(0xFFFFFFFFu, vmax)) / 64.f;
        f[17] = float(__reduce_min_sync(0xFFFFFFFFu, vmin)) / 64.f;
        {
            // 64-bit warp max / min from 32-bit reductions: high words first,
            // then the low words of the lanes that hold the extreme high word
            const unsigned xh = __reduce_max_sync(0xFFFFFFFFu, unsigned(umax >> 32));
            const unsigned xl = __reduce_max_sync(0xFFFFFFFFu, unsigned(umax >> 32) == xh ? unsigned(umax) : 0u);
            const unsigned nh = __reduce_min_sync(0xFFFFFFFFu, unsigned(umin >> 32));
            const unsigned nl = __reduce_min_sync(0xFFFFFFFFu, unsigned(umin >> 32) == nh ? unsigned(umin) : ~0u);
            umax = uint64_t(xh) << 32 | xl;
            umin = uint64_t(nh) << 32 | nl;
        }
        f[18] = float(effective_bitwidth(umax - umin)) / 64.f;
        f[19] = float(__reduce_max_sync(0xFFFFFFFFu, dmax)) / 64.f;
        f[20] = float(__reduce_add_sync(0xFFFFFFFFu, neg)) * rnd;
        const float hr = float(__reduce_add_sync(0xFFFFFFFFu, heads)) / 252.f;
        f[21] = hr;
        f[22] = float(__reduce_add_sync(0xFFFFFFFFu, zd)) * rnd;
        f[23] = float(__reduce_add_sync(0xFFFFFFFFu, vsum)) / (nv * 64.f);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            f[24 + c] = float(__reduce_max_sync(0xFFFFFFFFu, cmax[c])) / 64.f;
            f[28 + c] = float(__reduce_max_sync(0xFFFFFFFFu, cdmax[c])) / 64.f;
        }
        if (lane == 0)
            for (int k = 0; k < int(kSelNF); k++) feats[b * kSelNF + k] = f[k];
    }
}

// Best candidate by exact size (ties: lowest candidate index).
__global__ void k_sel_argmin(const uint32_t *__restrict__ sizes, uint64_t nblk, uint8_t *__restrict__ choice,
                             unsigned long long *__restrict__ total) {
    uint64_t t = 0;
    for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < nblk; b += uint64_t(gridDim.x) * blockDim.x) {
        unsigned best = 0;
        uint32_t bs = sizes[b * kSelNC];
        for (unsigned c = 1; c < kSelNC; c++)
            if (sizes[b * kSelNC + c] < bs) {
                bs = sizes[b * kSelNC + c];
                best = c;
            }
        if (choice) choice[b] = uint8_t(best);
        t += bs;
    }
    for (int s = 16; s > 0; s >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, s);
    if ((threadIdx.x & 31u) == 0 && total) atomicAdd(total, (unsigned long long)t);
}

// Container layout (blockwise_individual.h:189-311): block b's code byte
// directly follows block b-1's payload, its payload starts at the next 64-B
// boundary after the code byte.  With Q_b = the 64-B boundary at or below
// the code byte, Q_{b+1} = Q_b + 64 + floor64(size_b): a prefix sum.
__global__ void k_bwi_sizes(const BlockStats *__restrict__ st, const uint8_t *__restrict__ choice, uint64_t nblk,
                            uint64_t *__restrict__ bytes) {
    for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < nblk; b += uint64_t(gridDim.x) * blockDim.x)
        bytes[b] = 64 + (cand_size(st[b], choice[b]) & ~63u);
}

__global__ void __launch_bounds__(256) k_bwi_write(const uint64_t *__restrict__ in, uint64_t nblk,
                                                  const BlockStats *__restrict__ st,
                                                  const uint8_t *__restrict__ choice,
                                                  const uint64_t *__restrict__ off, uint8_t *__restrict__ out,
                                                  unsigned *err) {
    const unsigned lane = threadIdx.x & 31u;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nblk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const BlockStats s = st[b];
        const unsigned c = choice[b];
        if (lane == 0) {
            const unsigned prev_tail = b ? cand_size(st[b - 1], choice[b - 1]) & 63u : 0u;
            out[off[b] + prev_tail] = cand_code(s, c);
        }
        encode_block(in + b * kSelBlock, s, c, out + off[b] + 64, ok);
    }
    if (!ok) atomicOr(err, kErrCorrupt);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static unsigned sel_grid(uint64_t nblk) {
    return unsigned(maxu(1, minu((nblk + 7) / 8, uint64_t(persistent_grid(256, 8)))));
}

}  // namespace ms

using namespace ms;

extern "C" uint64_t ms_gpu_sel_block_values(void) { return kSelBlock; }

// Per-block statistics and the exact size of every candidate (size-only
// exhaustive pass).  stats: nblk x 32 bytes (opaque), sizes: nblk x 5 uint32.
extern "C" int ms_gpu_sel_analyze(const uint64_t *d_in, uint64_t nblk, void *d_stats, uint32_t *d_sizes,
                                  void *stream) {
    if ((!d_in || !d_stats) && nblk) return ms_fail(MS_ERR_INVALID, "sel_analyze: null argument");
    if (!nblk) return MS_OK;
    k_sel_analyze<<<sel_grid(nblk), 256, 0, (cudaStream_t)stream>>>(d_in, nblk, (BlockStats *)d_stats, d_sizes);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" uint64_t ms_gpu_sel_stats_bytes(void) { return sizeof(BlockStats); }

// compress-all: analysis, then every candidate materialised in scratch
// (ms_gpu_sel_compress_all_scratch_bytes()), exact sizes out.
extern "C" uint64_t ms_gpu_sel_compress_all_scratch_bytes(void) {
    return uint64_t(persistent_grid(256, 8)) * 8 * kSelNC * kSlot;
}

extern "C" int ms_gpu_sel_compress_all(const uint64_t *d_in, uint64_t nblk, void *d_stats, uint32_t *d_sizes,
                                       uint8_t *d_scratch, unsigned *d_err, void *stream) {
    if ((!d_in || !d_stats || !d_sizes || !d_scratch || !d_err) && nblk)
        return ms_fail(MS_ERR_INVALID, "sel_compress_all: null argument");
    if (!nblk) return MS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    k_sel_analyze<<<sel_grid(nblk), 256, 0, st>>>(d_in, nblk, (BlockStats *)d_stats, nullptr);
    MS_CUDA_TRY(cudaGetLastError());
    k_sel_compress_all<<<persistent_grid(256, 8), 256, 0, st>>>(d_in, nblk, (BlockStats *)d_stats, d_sizes, d_scratch,
                                                                d_err);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_sel_features(const uint64_t *d_in, uint64_t nblk, float *d_feats, void *stream) {
    if ((!d_in || !d_feats) && nblk) return ms_fail(MS_ERR_INVALID, "sel_features: null argument");
    if (!nblk) return MS_OK;
    k_sel_features<<<sel_grid(nblk), 256, 0, (cudaStream_t)stream>>>(d_in, nblk, d_feats);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_sel_argmin(const uint32_t *d_sizes, uint64_t nblk, uint8_t *d_choice, uint64_t *d_total,
                                 void *stream) {
    if (!d_sizes && nblk) return ms_fail(MS_ERR_INVALID, "sel_argmin: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (d_total) MS_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, st));
    if (!nblk) return MS_OK;
    k_sel_argmin<<<sel_grid(nblk), 256, 0, st>>>(d_sizes, nblk, d_choice, (unsigned long long *)d_total);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// Blockwise container of nblk*2048 values with one candidate per block
// (choice[b] in 0..4).  Output storage from the arena; *d_bytes (device) =
// container size.  out->format/meta describe a column of nblk*2048 values.
extern "C" int ms_gpu_bwi_compress(const uint64_t *d_in, uint64_t nblk, const void *d_stats, const uint8_t *d_choice,
                                   uint8_t **d_out, uint64_t **d_offsets, uint64_t *h_bytes, ms_arena *a,
                                   void *stream) {
    if (!d_in || !d_stats || !d_choice || !d_out || !d_offsets || !a) return ms_fail(MS_ERR_INVALID, "bwi_compress");
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t *sz = arena_take_t<uint64_t>(a, nblk + 1);
    uint64_t *off = arena_take_t<uint64_t>(a, nblk + 1);
    uint64_t *tot = arena_take_t<uint64_t>(a, 1);
    uint64_t *scr = arena_take_t<uint64_t>(a, scan_scratch_words(nblk, 1));
    if (!sz || !off || !tot || !scr) return ms_fail(MS_ERR_NOMEM, "arena exhausted (bwi)");
    k_bwi_sizes<<<sel_grid(nblk), 256, 0, st>>>((const BlockStats *)d_stats, d_choice, nblk, sz);
    MS_CUDA_TRY(cudaGetLastError());
    MS_CUDA_TRY((scan_exclusive<uint64_t, 1>(sz, nblk, off, tot, scr, st)));
    uint64_t bytes = 0, last_off = 0;
    uint8_t last_choice = 0;
    BlockStats last_st{};
    if (nblk) {
        MS_CUDA_TRY(cudaMemcpyAsync(&last_off, off + nblk - 1, 8, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaMemcpyAsync(&last_choice, d_choice + nblk - 1, 1, cudaMemcpyDeviceToHost, st));
        MS_CUDA_TRY(cudaMemcpyAsync(&last_st, (const BlockStats *)d_stats + nblk - 1, sizeof(BlockStats),
                                    cudaMemcpyDeviceToHost, st));
    }
    MS_CUDA_TRY(cudaStreamSynchronize(st));
    if (nblk) bytes = last_off + 64 + cand_size(last_st, last_choice);
    uint8_t *out = arena_take_t<uint8_t>(a, bytes + 64);
    if (!out) return ms_fail(MS_ERR_NOMEM, "arena exhausted (bwi output)");
    if (nblk) {
        k_bwi_write<<<sel_grid(nblk), 256, 0, st>>>(d_in, nblk, (const BlockStats *)d_stats, d_choice, off, out,
                                                    a->d_err);
        MS_CUDA_TRY(cudaGetLastError());
    }
    int rc = read_err(a, st);
    if (rc) return rc;
    *d_out = out;
    *d_offsets = off;
    *h_bytes = bytes;
    return MS_OK;
}

// ---------------------------------------------------------------------------
// Mixed synthetic column for the selector: segments of `seg_blocks` blocks
// cycle through four families (by segment index and seed): uniform over b
// bits (b in 1..40), sorted with random gaps, long runs, Zipf (inverse-CDF
// table).  One warp per block; value j of the block is row k*32 + lane.
// ---------------------------------------------------------------------------
namespace ms {
namespace {

__device__ __forceinline__ uint64_t gmix(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(256) k_sel_gen(uint64_t seed, uint64_t nblk, unsigned seg_blocks,
                                                const uint64_t *__restrict__ zipf, uint64_t n_zipf,
                                                uint64_t *__restrict__ out) {
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nblk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const uint64_t seg = b / seg_blocks;
        const uint64_t h = gmix(seed, seg);
        const unsigned fam = unsigned((seg + seed) & 3u);
        uint64_t *o = out + b * kSelBlock;
        const uint64_t rs = gmix(seed ^ 0xA5A5A5A5ull, b);
        if (fam == 0) {  // uniform over b bits
            const unsigned bits = 1 + unsigned(h % 40);
            for (unsigned k = 0; k < 64; k++) o[k * 32 + lane] = gmix(rs, k * 32 + lane) >> (64 - bits);
        } else if (fam == 3) {  // Zipf over the table's range
            for (unsigned k = 0; k < 64; k++) {
                const uint64_t u = gmix(rs, k * 32 + lane);
                uint64_t lo = 0, hi = n_zipf - 1;
                while (lo < hi) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (u < zipf[mid]) hi = mid;
                    else lo = mid + 1;
                }
                o[k * 32 + lane] = lo;
            }
        } else {
            // sorted: prefix sums of gaps in [1, 2g-1]; runs: value changes
            // where a draw hits 1/L, run values over 20 bits
            const unsigned g = 1 + unsigned(h % 16);
            const unsigned L = 64u << unsigned((h >> 8) % 4);
            uint64_t carry = fam == 1 ? (rs >> 24) : 0;
            for (unsigned k = 0; k < 64; k++) {
                const uint64_t u = gmix(rs, k * 32 + lane);
                uint64_t inc = fam == 1 ? 1 + u % (2 * g - 1) : uint64_t(u % L == 0);
                // inclusive warp scan
#pragma unroll
                for (int s = 1; s < 32; s <<= 1) {
                    const uint64_t t = __shfl_up_sync(0xFFFFFFFFu, inc, s);
                    if (lane >= unsigned(s)) inc += t;
                }
                const uint64_t v = carry + inc;
                o[k * 32 + lane] = fam == 1 ? v : (gmix(rs ^ 0x77, v) >> 44);
                carry = __shfl_sync(0xFFFFFFFFu, v, 31);
            }
        }
    }
}

// select(value cmp c) -> sum over a blockwise container.  One warp per
// block; the four 512-row sub-blocks are decoded with the vbp decoder, the
// cascade steps applied per format, rle handled per run.
__global__ void __launch_bounds__(256) k_bwi_select_sum(const uint8_t *__restrict__ data,
                                                       const uint64_t *__restrict__ q, const uint8_t *__restrict__ codes,
                                                       const uint32_t *__restrict__ psz, uint64_t nblk, int cmp,
                                                       uint64_t val,
                                                       unsigned long long *__restrict__ d_sum,
                                                       unsigned long long *__restrict__ d_cnt, unsigned *err) {
    const unsigned lane = threadIdx.x & 31u, l = lane & 7u, qq = lane >> 3;
    uint64_t s_sum = 0, s_cnt = 0;
    bool ok = true;
    for (uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; b < nblk;
         b += uint64_t(gridDim.x) * blockDim.x / 32) {
        const unsigned code = codes[b];
        const uint8_t *p = data + q[b] + 64;
        if (code == 71) {  // rle: (value, length) pairs covering 2048 rows
            const uint64_t *pr = reinterpret_cast<const uint64_t *>(p);
            const unsigned runs = psz[b] / 16;
            uint64_t rows = 0;
            for (unsigned r0 = 0; r0 < runs; r0 += 32) {
                const unsigned r = r0 + lane;
                if (r < runs) {
                    const uint64_t v = pr[2 * r], len = pr[2 * r + 1];
                    rows += len;
                    if (cmp_eval(cmp, v, val, true)) {
                        s_sum += v * len;
                        s_cnt += len;
                    }
                }
            }
            ok &= __reduce_add_sync(0xFFFFFFFFu, unsigned(rows)) == kSelBlock;
            continue;
        }
        // per sub-block location and width
        uint64_t carry = 0;  // delta: running lane sum
        for (unsigned i = 0; i < 4; i++) {
            unsigned bw;
            uint64_t off, ref = 0;
            bool dlt = false;
            if (code >= 1 && code <= 64) {
                bw = code;
                off = uint64_t(64) * bw * i;
            } else if (code == 65) {
                uint64_t acc = 0;
                for (unsigned k = 0; k < i; k++) acc += p[k];
                bw = p[i];
                off = 64 + 64 * acc;
            } else if (code == 67 || code == 69) {
                const bool isfor = code == 69;
                const uint64_t page0 = isfor ? 64 : 0;
                const uint8_t w0 = p[page0], w1 = p[page0 + 1];
                const uint64_t page1 = page0 + 64 + 64 * uint64_t(w0 + w1);
                const uint64_t pg = (i >> 1) ? page1 : page0;
                const uint8_t a = p[pg], c2 = p[pg + 1];
                bw = (i & 1) ? c2 : a;
                off = pg + 64 + ((i & 1) ? 64 * uint64_t(a) : 0);
                if (isfor) ref = reinterpret_cast<const uint64_t *>(p)[i >> 1];
                else dlt = true;
            } else {
                ok = false;
                break;
            }
            uint64_t v[16];
            ok &= vbp_decode16_rt(bw, reinterpret_cast<const uint64_t *>(p + off), l, qq, v);
            if (dlt) {
#pragma unroll
                for (int k = 1; k < 16; k++) v[k] += v[k - 1];
                const uint64_t tot = v[15];
                const uint64_t up = __shfl_up_sync(0xFFFFFFFFu, tot, 8);
                uint64_t pre = qq >= 1 ? up : 0;
                const uint64_t up2 = __shfl_up_sync(0xFFFFFFFFu, tot + pre, 16);
                pre += qq >= 2 ? up2 : 0;
                pre += carry;
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] += pre;
                // lane total of this sub-block: last value of quarter 3
                carry = __shfl_sync(0xFFFFFFFFu, v[15], 24 + l);
            } else {
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] += ref;
            }
#pragma unroll
            for (int k = 0; k < 16; k++)
                if (cmp_eval(cmp, v[k], val, true)) {
                    s_sum += v[k];
                    s_cnt++;
                }
        }
    }
    if (!ok) atomicOr(err, kErrCorrupt);
    for (int s = 16; s > 0; s >>= 1) {
        s_sum += __shfl_xor_sync(0xFFFFFFFFu, s_sum, s);
        s_cnt += __shfl_xor_sync(0xFFFFFFFFu, s_cnt, s);
    }
    if (lane == 0) {
        atomicAdd(d_sum, (unsigned long long)s_sum);
        if (d_cnt) atomicAdd(d_cnt, (unsigned long long)s_cnt);
    }
}

__global__ void k_bwi_codes(const BlockStats *__restrict__ st, const uint8_t *__restrict__ choice, uint64_t nblk,
                            uint8_t *__restrict__ codes, uint32_t *__restrict__ psz) {
    for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b < nblk; b += uint64_t(gridDim.x) * blockDim.x) {
        codes[b] = cand_code(st[b], choice[b]);
        psz[b] = cand_size(st[b], choice[b]);
    }
}

}  // namespace
}  // namespace ms

extern "C" int ms_gpu_sel_gen(uint64_t seed, uint64_t nblk, unsigned seg_blocks, const uint64_t *d_zipf,
                              uint64_t n_zipf, uint64_t *d_out, void *stream) {
    if ((!d_out || !d_zipf || !n_zipf || !seg_blocks) && nblk) return ms_fail(MS_ERR_INVALID, "sel_gen: bad argument");
    if (!nblk) return MS_OK;
    k_sel_gen<<<sel_grid(nblk), 256, 0, (cudaStream_t)stream>>>(seed, nblk, seg_blocks, d_zipf, n_zipf, d_out);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_sel_resolve(const uint64_t *d_in, uint64_t nblk, uint8_t *d_choice, void *stream) {
    if ((!d_in || !d_choice) && nblk) return ms_fail(MS_ERR_INVALID, "sel_resolve: bad argument");
    if (!nblk) return MS_OK;
    k_sel_resolve<<<sel_grid(nblk), 256, 0, (cudaStream_t)stream>>>(d_in, nblk, d_choice);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_sel_footprint(const uint32_t *d_sizes, const uint8_t *d_choice, uint64_t nblk, uint64_t *d_total,
                                    void *stream) {
    if (!d_total || ((!d_sizes || !d_choice) && nblk)) return ms_fail(MS_ERR_INVALID, "sel_footprint: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    MS_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, st));
    if (!nblk) return MS_OK;
    k_sel_footprint<<<sel_grid(nblk), 256, 0, st>>>(d_sizes, d_choice, nblk, (unsigned long long *)d_total);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

// Block index of a container: format code and payload bytes per block.
extern "C" int ms_gpu_bwi_codes(const void *d_stats, const uint8_t *d_choice, uint64_t nblk, uint8_t *d_codes,
                                uint32_t *d_payload_bytes, void *stream) {
    if ((!d_stats || !d_choice || !d_codes || !d_payload_bytes) && nblk)
        return ms_fail(MS_ERR_INVALID, "bwi_codes: bad argument");
    if (!nblk) return MS_OK;
    k_bwi_codes<<<sel_grid(nblk), 256, 0, (cudaStream_t)stream>>>((const BlockStats *)d_stats, d_choice, nblk, d_codes,
                                                                  d_payload_bytes);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}

extern "C" int ms_gpu_bwi_select_sum(const uint8_t *d_data, const uint64_t *d_offsets, const uint8_t *d_codes,
                                     const uint32_t *d_payload_bytes, uint64_t nblk, int cmp, uint64_t val,
                                     uint64_t *d_sum, uint64_t *d_cnt, unsigned *d_err, void *stream) {
    if (!d_sum || !d_err || ((!d_data || !d_offsets || !d_codes || !d_payload_bytes) && nblk))
        return ms_fail(MS_ERR_INVALID, "bwi_select_sum: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    MS_CUDA_TRY(cudaMemsetAsync(d_sum, 0, 8, st));
    if (d_cnt) MS_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, 8, st));
    if (!nblk) return MS_OK;
    k_bwi_select_sum<<<sel_grid(nblk), 256, 0, st>>>(d_data, d_offsets, d_codes, d_payload_bytes, nblk, cmp, val,
                                                    (unsigned long long *)d_sum, (unsigned long long *)d_cnt, d_err);
    MS_CUDA_TRY(cudaGetLastError());
    return MS_OK;
}
