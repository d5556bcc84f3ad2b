// lbm_fast.cu - the fused interior kernels with the fast arithmetic policy
// (lbm_fast.cuh).  A translation unit of its own so that it is compiled
// with multiply-add contraction while the rest of the library keeps the
// reference's rounding (-fmad=false).
#define LBM_AUX_TU
#include <cuda_runtime.h>

#include "lbm_launch.h"
#include "lbm_stages.cuh"
#include "lbm_tile.cuh"
#include "lbm_fast.cuh"
#include "lbm_batch_tile.cuh"

namespace lbm {

template <int S>
static bool launch_fast_s(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st) {
    if (A.P.collision == LBM_COLLIDE_KBC) return launch_tile_tma_t<S, ArFast<LBM_COLLIDE_KBC>>(A, m24, m20, st);
    return launch_tile_tma_t<S, ArFast<LBM_COLLIDE_REGULARIZED>>(A, m24, m20, st);
}

bool launch_tile_tma_fast(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F32: return launch_fast_s<LBM_STORE_F32>(A, m24, m20, st);
        case LBM_STORE_F16S: return launch_fast_s<LBM_STORE_F16S>(A, m24, m20, st);
        case LBM_STORE_BF16S: return launch_fast_s<LBM_STORE_BF16S>(A, m24, m20, st);
        default: return false;
    }
}

// the interior grid of an ensemble group: the group's collision model picks the policy
void launch_batch_tile_fast(int which, int storage, const BatchGroup &G, bool les, int collision, int tile_blocks,
                            cudaStream_t st) {
    if (collision == LBM_COLLIDE_KBC)
        launch_batch_tile_any<ArFast<LBM_COLLIDE_KBC>>(which, storage, G, les, tile_blocks, st);
    else
        launch_batch_tile_any<ArFast<LBM_COLLIDE_REGULARIZED>>(which, storage, G, les, tile_blocks, st);
}

int batch_tile_blocks_fast(int storage, bool les, int collision, bool tma) {
    if (collision == LBM_COLLIDE_KBC) return batch_tile_blocks_any<ArFast<LBM_COLLIDE_KBC>>(storage, les, tma);
    return batch_tile_blocks_any<ArFast<LBM_COLLIDE_REGULARIZED>>(storage, les, tma);
}

}  // namespace lbm
