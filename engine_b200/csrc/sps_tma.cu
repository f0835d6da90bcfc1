// sps_tma.cu -- entry of the staged select -> project -> sum pipeline: checks
// the launch configuration and dispatches to the launcher for the
// consumer-warp count (the kernels are in sps_tma.cuh, instantiated per warp
// count in sps_tma_w<W>.cu).
#include "sps_tma.cuh"

namespace ms {

// Fused select -> project -> agg_sum through the staged pipeline.  Columns
// must be uncompr / static_vbp or carry a block index (dynamic_vbp, for_f)
// or a prepared delta view.  warps: consumer warps per CTA (4, 8, 12, 16, 20, 24).
int sps_tma(const ColView &x, const ColView &y, bool has_y, int cmp, uint64_t val, unsigned warps, unsigned stages,
            unsigned stage_bytes, unsigned ctas_per_sm, unsigned vpt, uint64_t *d_sum, uint64_t *d_cnt,
            unsigned *d_err, cudaStream_t st) {
    if (stage_bytes < 2 * 4096 + 128 || stage_bytes % 128) return ms_fail(MS_ERR_INVALID, "sps_tma: stage_bytes");
    if (stages < 2 || stages > 32) return ms_fail(MS_ERR_INVALID, "sps_tma: stages");
    TmaCfg cfg{stages, stage_bytes, kMaxTile};
    const unsigned grid = unsigned(sm_count()) * (ctas_per_sm ? ctas_per_sm : 1);
#define MS_L(Wn) \
    if (warps == Wn) return sps_tma_launch_w##Wn(x, y, has_y, cmp, val, cfg, vpt, d_sum, d_cnt, d_err, grid, st);
    MS_L(4) MS_L(8) MS_L(12) MS_L(16) MS_L(20) MS_L(24)
#undef MS_L
    return ms_fail(MS_ERR_INVALID, "sps_tma: warps must be 4, 8, 12, 16, 20 or 24");
}

}  // namespace ms
