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

typedef ArFast<LBM_COLLIDE_KBC> ArFastK;
typedef ArFast<LBM_COLLIDE_REGULARIZED> ArFastR;

void launch_batch_tile_fast(int which, int storage, const BatchLaunch &L, int q, unsigned long long step, int flags,
                            cudaStream_t st) {
    switch (storage) {
        case LBM_STORE_F16S: launch_batch_tile_t<LBM_STORE_F16S, ArFastK, ArFastR>(which, L, q, step, flags, st); break;
        case LBM_STORE_BF16S: launch_batch_tile_t<LBM_STORE_BF16S, ArFastK, ArFastR>(which, L, q, step, flags, st); break;
        default: launch_batch_tile_t<LBM_STORE_F32, ArFastK, ArFastR>(which, L, q, step, flags, st); break;
    }
}

int batch_tile_blocks_fast(int storage) {
    switch (storage) {
        case LBM_STORE_F16S: return batch_tile_blocks_t<LBM_STORE_F16S, ArFastK, ArFastR>();
        case LBM_STORE_BF16S: return batch_tile_blocks_t<LBM_STORE_BF16S, ArFastK, ArFastR>();
        default: return batch_tile_blocks_t<LBM_STORE_F32, ArFastK, ArFastR>();
    }
}

}  // namespace lbm
