// lbm_batch_tile.cuh - the interior planes of a group of ensemble domains as
// one work queue (kb_tile) and its host-side launch, shared by the exact
// translation unit (lbm_device.cu, ArExact) and the fast one (lbm_fast.cu,
// ArFast).  A grid of resident blocks takes (domain, tile x, tile y, z chunk)
// items from a counter until none is left and runs the cp.async-staged tile
// body of a domain's own launch on each, with the item's step arguments read
// from the launch's parameter space, so the results equal stepping the
// domains one by one.  The group's domains share the LES switch and the
// collision model, which are template arguments here.
#pragma once

#include "lbm_tile.cuh"

namespace lbm {

template <int S>
constexpr int batch_tile_smem() {
    return S == LBM_STORE_F32 ? PIPE_SMEM_BYTES : P16_SMEM_BYTES;
}

template <int S, int IN, bool LES, class Ar>
__global__ void __launch_bounds__(256, 2) kb_tile(const __grid_constant__ BatchGroup G) {
    extern __shared__ __align__(16) float smem[];
    __shared__ int s_item;
    // a tile-copy grid launched behind this one may start once every block
    // runs (the two take disjoint tiles)
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    for (;;) {
        __syncthreads();   // every thread is done with the last item's shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(G.queue, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= G.nmap) break;
        const int4 it = G.map[item];
        const StepArgs &A = G.a[it.x];
        if constexpr (S == LBM_STORE_F32) tile_pipe_body<IN, LES, Ar>(A, smem, it.y, it.z, it.w);
        else tile_pipe16_body<S, IN, LES, Ar>(A, smem, it.y, it.z, it.w);
    }
}

// The fused interior step with LES on the tiles off each domain's edge,
// staged by tile copies (tile_tma_body), as a work queue of (domain, tile x,
// tile y, z chunk) items; the tensor maps of the item's domain come from the
// launch parameters.
template <int S, class Ar>
__global__ void __launch_bounds__(256, 2) kb_tile_tma(const __grid_constant__ BatchGroup G) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    __shared__ int s_item;
    for (;;) {
        __syncthreads();   // every thread is done with the last item's shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(G.queue, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= G.nmap) break;
        const int4 it = G.map[item];
        if (!tile_tma_body<S, Ar>(G.a[it.x], &G.tmap[it.x][0], &G.tmap[it.x][1], tma_smem, it.y * LBM_TILE,
                                  it.z * LBM_TILE, it.w))
            break;   // a wait gave up (status bit 2 of the domain)
    }
    // complete only after the edge grid this one may have been launched
    // behind, so that the work after it sees both grids' results
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

template <int S, class Ar>
static bool batch_tma_ready_t() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        ok[dev] = cudaFuncSetAttribute(kb_tile_tma<S, Ar>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       tma_smem_bytes<S>()) == cudaSuccess;
    }
    return ok[dev];
}

template <int S, class Ar>
static int batch_tma_blocks_t() {
    if (!batch_tma_ready_t<S, Ar>()) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kb_tile_tma<S, Ar>, 256, tma_smem_bytes<S>()) !=
            cudaSuccess)
        return 0;
    return per * sms;
}

template <int S, class Ar>
static void launch_batch_tma_t(const BatchGroup &G, int tile_blocks, cudaStream_t st) {
    if (!G.nmap || tile_blocks <= 0 || !batch_tma_ready_t<S, Ar>()) return;
    if (!G.pdl) cudaMemsetAsync(G.queue, 0, sizeof(int), st);
    const unsigned g = (unsigned)(tile_blocks < G.nmap ? tile_blocks : G.nmap);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = tma_smem_bytes<S>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = G.pdl ? 1 : 0;
    if (cudaLaunchKernelEx(&cfg, kb_tile_tma<S, Ar>, G) != cudaSuccess) {
        cudaGetLastError();
        kb_tile_tma<S, Ar><<<g, 256, tma_smem_bytes<S>(), st>>>(G);
    }
    launch_count_add(1);
}

template <int S, bool LES, class Ar>
static bool batch_tile_ready_t() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        ok[dev] = cudaFuncSetAttribute(kb_tile<S, 0, LES, Ar>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       batch_tile_smem<S>()) == cudaSuccess &&
                  cudaFuncSetAttribute(kb_tile<S, 1, LES, Ar>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       batch_tile_smem<S>()) == cudaSuccess;
    }
    return ok[dev];
}

// resident blocks of the work-queue grid on the current device (0: refused)
template <int S, bool LES, class Ar>
static int batch_tile_blocks_t() {
    if (!batch_tile_ready_t<S, LES, Ar>()) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kb_tile<S, 1, LES, Ar>, 256, batch_tile_smem<S>()) !=
            cudaSuccess)
        return 0;
    return per * sms;
}

template <int S, bool LES, class Ar>
static void launch_batch_tile_t(int which, const BatchGroup &G, int tile_blocks, cudaStream_t st) {
    if (!G.nmap || tile_blocks <= 0 || !batch_tile_ready_t<S, LES, Ar>()) return;
    cudaMemsetAsync(G.queue, 0, (G.pdl ? 2 : 1) * sizeof(int), st);   // with pdl: the tile-copy grid's counter too
    const unsigned g = (unsigned)(tile_blocks < G.nmap ? tile_blocks : G.nmap);
    if (which == KER_TILE_CANON) kb_tile<S, 0, LES, Ar><<<g, 256, batch_tile_smem<S>(), st>>>(G);
    else kb_tile<S, 1, LES, Ar><<<g, 256, batch_tile_smem<S>(), st>>>(G);
    launch_count_add(1);
}

// dispatch on the storage and the LES switch for one arithmetic policy
// (KER_TILE_TMA: the tile-copy grid, LES on)
template <class Ar>
static void launch_batch_tile_any(int which, int storage, const BatchGroup &G, bool les, int tile_blocks,
                                  cudaStream_t st) {
    if (which == KER_TILE_TMA) {
        switch (storage) {
            case LBM_STORE_F16S: launch_batch_tma_t<LBM_STORE_F16S, Ar>(G, tile_blocks, st); break;
            case LBM_STORE_BF16S: launch_batch_tma_t<LBM_STORE_BF16S, Ar>(G, tile_blocks, st); break;
            default: launch_batch_tma_t<LBM_STORE_F32, Ar>(G, tile_blocks, st); break;
        }
        return;
    }
    switch (storage) {
        case LBM_STORE_F16S:
            if (les) launch_batch_tile_t<LBM_STORE_F16S, true, Ar>(which, G, tile_blocks, st);
            else launch_batch_tile_t<LBM_STORE_F16S, false, Ar>(which, G, tile_blocks, st);
            break;
        case LBM_STORE_BF16S:
            if (les) launch_batch_tile_t<LBM_STORE_BF16S, true, Ar>(which, G, tile_blocks, st);
            else launch_batch_tile_t<LBM_STORE_BF16S, false, Ar>(which, G, tile_blocks, st);
            break;
        default:
            if (les) launch_batch_tile_t<LBM_STORE_F32, true, Ar>(which, G, tile_blocks, st);
            else launch_batch_tile_t<LBM_STORE_F32, false, Ar>(which, G, tile_blocks, st);
            break;
    }
}
template <class Ar>
static int batch_tile_blocks_any(int storage, bool les, bool tma = false) {
    if (tma) {
        switch (storage) {
            case LBM_STORE_F16S: return batch_tma_blocks_t<LBM_STORE_F16S, Ar>();
            case LBM_STORE_BF16S: return batch_tma_blocks_t<LBM_STORE_BF16S, Ar>();
            default: return batch_tma_blocks_t<LBM_STORE_F32, Ar>();
        }
    }
    switch (storage) {
        case LBM_STORE_F16S:
            return les ? batch_tile_blocks_t<LBM_STORE_F16S, true, Ar>() : batch_tile_blocks_t<LBM_STORE_F16S, false, Ar>();
        case LBM_STORE_BF16S:
            return les ? batch_tile_blocks_t<LBM_STORE_BF16S, true, Ar>() : batch_tile_blocks_t<LBM_STORE_BF16S, false, Ar>();
        default:
            return les ? batch_tile_blocks_t<LBM_STORE_F32, true, Ar>() : batch_tile_blocks_t<LBM_STORE_F32, false, Ar>();
    }
}

}  // namespace lbm
