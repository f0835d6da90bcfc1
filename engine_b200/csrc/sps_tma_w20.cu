// sps_tma_w20.cu -- the staged select -> project -> sum kernels with 20
// consumer warps (see sps_tma.cuh).
#include "sps_tma.cuh"

namespace ms {

MS_SPS_TMA_LAUNCHER(20) {
    return has_y ? launch_tma<20, true>(x, y, cmp, val, cfg, vpt, d_sum, d_cnt, d_err, grid, st)
                 : launch_tma<20, false>(x, x, cmp, val, cfg, vpt, d_sum, d_cnt, d_err, grid, st);
}

}  // namespace ms
