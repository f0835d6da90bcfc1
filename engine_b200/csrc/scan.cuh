// scan.cuh -- exclusive prefix sums over small device arrays (block sizes,
// hit counts, run counts, delta carries).  Reduce-then-scan in three
// launches, recursive over the tile sums; W = elements per item (8 for the
// lane-wise delta carries, scanned lane by lane).
#pragma once

#include "ms_common.cuh"

namespace ms {

constexpr unsigned kScanThreads = 256;
constexpr unsigned kScanPerThread = 8;
constexpr unsigned kScanTile = kScanThreads * kScanPerThread;

template <class T, unsigned W>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const T *__restrict__ in, uint64_t n,
                                                             uint64_t *__restrict__ tile_sums) {
    __shared__ uint64_t sh[kScanThreads];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile;
    for (unsigned w = 0; w < W; w++) {
        uint64_t s = 0;
        for (unsigned i = 0; i < kScanPerThread; i++) {
            const uint64_t idx = base + threadIdx.x * kScanPerThread + i;
            if (idx < n) s += uint64_t(in[idx * W + w]);
        }
        sh[threadIdx.x] = s;
        __syncthreads();
        for (unsigned st = kScanThreads / 2; st > 0; st >>= 1) {
            if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) tile_sums[blockIdx.x * W + w] = sh[0];
        __syncthreads();
    }
}

// Exclusive scan of one tile (plus a per-tile offset); optionally writes the
// grand total (last tile) to *total.
template <class T, unsigned W>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const T *__restrict__ in, uint64_t n,
                                                           const uint64_t *__restrict__ tile_off,
                                                           uint64_t *__restrict__ out, uint64_t *__restrict__ total) {
    __shared__ uint64_t sh[kScanThreads];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile;
    for (unsigned w = 0; w < W; w++) {
        uint64_t v[kScanPerThread];
        uint64_t s = 0;
        for (unsigned i = 0; i < kScanPerThread; i++) {
            const uint64_t idx = base + threadIdx.x * kScanPerThread + i;
            v[i] = idx < n ? uint64_t(in[idx * W + w]) : 0;
            s += v[i];
        }
        sh[threadIdx.x] = s;
        __syncthreads();
        // Hillis-Steele inclusive scan over thread sums
        for (unsigned st = 1; st < kScanThreads; st <<= 1) {
            uint64_t add = threadIdx.x >= st ? sh[threadIdx.x - st] : 0;
            __syncthreads();
            sh[threadIdx.x] += add;
            __syncthreads();
        }
        uint64_t run = (threadIdx.x ? sh[threadIdx.x - 1] : 0) + (tile_off ? tile_off[blockIdx.x * W + w] : 0);
        for (unsigned i = 0; i < kScanPerThread; i++) {
            const uint64_t idx = base + threadIdx.x * kScanPerThread + i;
            if (idx < n) out[idx * W + w] = run;
            run += v[i];
        }
        if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) total[w] = run;
        __syncthreads();
    }
}

// Scratch needed by scan_exclusive for n items of width W (in uint64 words).
inline uint64_t scan_scratch_words(uint64_t n, unsigned W) {
    uint64_t words = 0;
    while (n > kScanTile) {
        const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
        words += 2 * tiles * W;
        n = tiles;
    }
    return words + W;
}

// out[i] = sum_{j<i} in[j] (lane-wise for W > 1); total[0..W) = grand total.
// `scratch` holds scan_scratch_words(n, W) words.
template <class T, unsigned W>
cudaError_t scan_exclusive(const T *in, uint64_t n, uint64_t *out, uint64_t *total, uint64_t *scratch,
                           cudaStream_t st) {
    if (n == 0) {
        return cudaMemsetAsync(total, 0, sizeof(uint64_t) * W, st);
    }
    const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        k_scan_tile<T, W><<<1, kScanThreads, 0, st>>>(in, n, nullptr, out, total);
        return cudaGetLastError();
    }
    uint64_t *tile_sums = scratch;
    uint64_t *tile_off = scratch + tiles * W;
    k_scan_reduce<T, W><<<unsigned(tiles), kScanThreads, 0, st>>>(in, n, tile_sums);
    cudaError_t e = scan_exclusive<uint64_t, W>(tile_sums, tiles, tile_off, total, scratch + 2 * tiles * W, st);
    if (e != cudaSuccess) return e;
    k_scan_tile<T, W><<<unsigned(tiles), kScanThreads, 0, st>>>(in, n, tile_off, out, nullptr);
    return cudaGetLastError();
}

}  // namespace ms
