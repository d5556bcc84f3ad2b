// lbm_batch_tile.cuh - the interior planes of an ensemble as one work queue
// (kb_tile) and its host-side launch, shared by the exact translation unit
// (lbm_device.cu, ArExact) and the fast one (lbm_fast.cu, ArFast).  A grid of
// resident blocks takes (domain, tile x, tile y, z chunk) items from a
// counter until none is left; a block copies its domain's step arguments into
// shared memory when the domain changes and runs the cp.async-staged tile
// body of a domain's own launch, so the results equal stepping the domains
// one by one.
#pragma once

#include "lbm_tile.cuh"

namespace lbm {

// copy a domain's step arguments into shared memory (all threads of the block)
LBM_DEV void batch_load_args(StepArgs &dst, const StepArgs &src) {
    const int nw = (int)(sizeof(StepArgs) / 4);
    const unsigned *s = (const unsigned *)&src;
    unsigned *d = (unsigned *)&dst;
    const int t = threadIdx.x + threadIdx.y * blockDim.x, nt = blockDim.x * blockDim.y;
    for (int w = t; w < nw; w += nt) d[w] = s[w];
}
static_assert(sizeof(StepArgs) % 4 == 0, "step arguments copy as words");

template <int S>
constexpr int batch_tile_smem() {
    return S == LBM_STORE_F32 ? PIPE_SMEM_BYTES : P16_SMEM_BYTES;
}

// the interior planes of every domain as a work queue; ArK / ArR: the
// arithmetic policies of KBC and regularized domains
template <int S, int IN, class ArK, class ArR>
__global__ void __launch_bounds__(256, 2) kb_tile(BatchLaunch L, int q, unsigned long long step, int flags) {
    extern __shared__ __align__(16) float smem[];
    __shared__ __align__(16) StepArgs sA;
    __shared__ int s_item;
    int cur = -1;
    for (;;) {
        __syncthreads();   // every thread is done with the last item's shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(L.queue, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= L.nitems) break;
        const int4 it = L.items[item];
        if (it.x != cur) {
            batch_load_args(sA, L.tab[q * L.ndom + it.x]);
            __syncthreads();
            if (threadIdx.x == 0) {
                sA.step = step;
                sA.flags = flags;
            }
            __syncthreads();
            cur = it.x;
        }
        const bool kbc = sA.P.collision == LBM_COLLIDE_KBC;
        if constexpr (S == LBM_STORE_F32) {
            if (sA.P.use_les) {
                if (kbc) tile_pipe_body<IN, true, ArK>(sA, smem, it.y, it.z, it.w);
                else tile_pipe_body<IN, true, ArR>(sA, smem, it.y, it.z, it.w);
            } else {
                if (kbc) tile_pipe_body<IN, false, ArK>(sA, smem, it.y, it.z, it.w);
                else tile_pipe_body<IN, false, ArR>(sA, smem, it.y, it.z, it.w);
            }
        } else {
            if (sA.P.use_les) {
                if (kbc) tile_pipe16_body<S, IN, true, ArK>(sA, smem, it.y, it.z, it.w);
                else tile_pipe16_body<S, IN, true, ArR>(sA, smem, it.y, it.z, it.w);
            } else {
                if (kbc) tile_pipe16_body<S, IN, false, ArK>(sA, smem, it.y, it.z, it.w);
                else tile_pipe16_body<S, IN, false, ArR>(sA, smem, it.y, it.z, it.w);
            }
        }
    }
}

template <int S, class ArK, class ArR>
static bool batch_tile_ready_t() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        ok[dev] = cudaFuncSetAttribute(kb_tile<S, 0, ArK, ArR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       batch_tile_smem<S>()) == cudaSuccess &&
                  cudaFuncSetAttribute(kb_tile<S, 1, ArK, ArR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       batch_tile_smem<S>()) == cudaSuccess;
    }
    return ok[dev];
}

// resident blocks of the work-queue grid on the current device (0: refused)
template <int S, class ArK, class ArR>
static int batch_tile_blocks_t() {
    if (!batch_tile_ready_t<S, ArK, ArR>()) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kb_tile<S, 1, ArK, ArR>, 256, batch_tile_smem<S>()) !=
            cudaSuccess)
        return 0;
    return per * sms;
}

template <int S, class ArK, class ArR>
static void launch_batch_tile_t(int which, const BatchLaunch &L, int q, unsigned long long step, int flags,
                                cudaStream_t st) {
    if (!L.nitems || !L.tile_blocks) return;
    cudaMemsetAsync(L.queue, 0, sizeof(int), st);
    const unsigned g = (unsigned)(L.tile_blocks < L.nitems ? L.tile_blocks : L.nitems);
    if (which == KER_TILE_CANON) kb_tile<S, 0, ArK, ArR><<<g, 256, batch_tile_smem<S>(), st>>>(L, q, step, flags);
    else kb_tile<S, 1, ArK, ArR><<<g, 256, batch_tile_smem<S>(), st>>>(L, q, step, flags);
    launch_count_add(1);
}

}  // namespace lbm
