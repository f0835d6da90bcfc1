// ref_bwi.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's blockwise_individual_f container (blockwise_individual.h:
// 60-311) and its exhaustive_size_format_selector (exhaustive_size_format_
// selector.h:36-141), compiled from the reference's headers where they lie,
// with the two cascade macros they need supplied by ref_missing_formats.h.
//   ref_bwi_compress: morph_batch<ve, blockwise_individual_f<2048,
//     fixed_choice_selector, ve>, uncompr_f> of nblk 2048-value blocks, the
//     selector returning the given format code for each block in turn;
//   ref_exhaustive_choose: the reference selector's format code per block.
// Built by oracle/Makefile into libmsref_<isa>.so beside ref_shim.cpp.
#include <core/memory/mm_glob.h>
#include <core/format_selection/exhaustive_size_format_selector.h>
#include <core/morphing/blockwise_individual.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

using namespace morphstore;
using namespace vectorlib;

#ifndef VE
#define VE avx512<v512<uint64_t>>
#endif
using bwi_ve = VE;

namespace {

thread_local const uint8_t *g_codes = nullptr;
thread_local size_t g_next = 0;

// A format selector that returns prescribed codes (the GPU's per-block picks).
template <class t_vector_extension> struct fixed_choice_selector : public format_selector<t_vector_extension> {
    static format_code choose(const typename t_vector_extension::base_t *, size_t) {
        return static_cast<format_code>(g_codes[g_next++]);
    }
};

constexpr size_t kBwiBlock = 2048;

}  // namespace

extern "C" {

// A 64-byte aligned copy: the reference's packers load their input with
// aligned vector loads (its columns are always 64-byte aligned).
static uint64_t *aligned_copy(const uint64_t *in, size_t n) {
    void *mem = nullptr;
    if (posix_memalign(&mem, 64, std::max<size_t>(8 * n, 64))) return nullptr;
    std::memcpy(mem, in, 8 * n);
    return static_cast<uint64_t *>(mem);
}

// out receives the container bytes (compressed through a 64-byte aligned,
// zeroed buffer, as the reference aligns payloads by address); *bytes = size.
int ref_bwi_compress(const uint64_t *in, uint64_t nblk, const uint8_t *codes, uint8_t *out, uint64_t cap,
                     uint64_t *bytes) {
    using f = blockwise_individual_f<kBwiBlock, fixed_choice_selector, bwi_ve>;
    const size_t worst = f::get_size_max_byte(nblk * kBwiBlock) + 64;
    void *mem = nullptr;
    if (posix_memalign(&mem, 64, (worst + 63) / 64 * 64)) return 4;
    uint8_t *buf = static_cast<uint8_t *>(mem);
    uint64_t *src = aligned_copy(in, nblk * kBwiBlock);
    if (!src) {
        std::free(buf);
        return 4;
    }
    std::memset(buf, 0, worst);
    g_codes = codes;
    g_next = 0;
    const uint8_t *in8 = reinterpret_cast<const uint8_t *>(src);
    uint8_t *out8 = buf;
    morph_batch<bwi_ve, f, uncompr_f>(in8, out8, nblk * kBwiBlock);
    const uint64_t n = uint64_t(out8 - buf);
    int rc = 0;
    if (n > cap)
        rc = 4;
    else
        std::memcpy(out, buf, n);
    *bytes = n;
    std::free(buf);
    std::free(src);
    return rc;
}

int ref_exhaustive_choose(const uint64_t *in, uint64_t nblk, uint8_t *codes) {
    uint64_t *src = aligned_copy(in, nblk * kBwiBlock);
    if (!src) return 4;
    for (uint64_t b = 0; b < nblk; b++)
        codes[b] = static_cast<uint8_t>(
            exhaustive_size_format_selector_helper<true>::selector<bwi_ve>::choose(src + b * kBwiBlock, kBwiBlock));
    std::free(src);
    return 0;
}

}  // extern "C"
