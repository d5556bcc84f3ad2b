// lbm_batch.cuh - an ensemble of air domains stepped with one launch per
// phase and group of domains.
//
// The ensemble is split into groups of at most BATCH_GROUP domains that share
// the collision model; each group steps on a stream of its own, so the
// phases of different groups overlap on the device.  Each phase of the air
// step (bed, 3x3 maximum and column cache; general pre-pass; interior planes;
// general collide; the final stream) runs as one grid over the group's
// domains, with each block's domain and coordinates taken from device tables
// built when the ensemble is created:
//   kb_bed / kb_hmax / kb_colgeo   one thread per column of the concatenated
//                                  columns of the group's domains
//   kb_general                     one block of 32 x 8 cells per map entry
//                                  (domain, bx, by, bz): pre-pass, collide or
//                                  stream of the planes next to the bed and
//                                  the top
//   kb_tile                        the interior planes as a work queue: a
//                                  grid of resident blocks, each taking the
//                                  next (domain, tile, z chunk) item from a
//                                  counter until none is left, so domains of
//                                  uneven size share the SMs without a tail
//                                  per domain
//   kb_stream_interior             one block per map entry
// The step arguments of the group's domains travel in the launch's parameter
// space (BatchGroup), and each block runs the same per-block body as a
// domain's own launch (prepass_body, collide_body, stream_body,
// tile_pipe_body / tile_pipe16_body, stream_interior_body) on its domain's
// entry, so an ensemble steps bit for bit like its domains stepped one by one.
#pragma once

#include "lbm_batch_tile.cuh"

namespace lbm {

// domain of concatenated column g: the last d with col0[d] <= g
LBM_DEV int batch_domain(const long long *col0, int ndom, long long g) {
    int lo = 0, hi = ndom - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (col0[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void kb_bed(BatchLaunch L, long long m, int par) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= L.ncols) return;
    const int d = batch_domain(L.col0, L.ndom, g);
    const BatchBed &B = L.bed[par * L.nall + L.d0 + d];
    const float t = (float)((double)(m + 1) * B.P.dt_phys);   // the host's step time, CODEX.py:3874
    bed_column(B.P, B.D, B.h_prev, B.h, B.uw, B.vw, B.ww, B.piecewise, t, (int)(g - L.col0[d]));
}
__global__ void kb_hmax(BatchLaunch L, int par) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= L.ncols) return;
    const int d = batch_domain(L.col0, L.ndom, g);
    const BatchBed &B = L.bed[par * L.nall + L.d0 + d];
    hmax_column(B.D, B.h, B.hmax, (int)(g - L.col0[d]));
}
__global__ void kb_colgeo(BatchLaunch L, int par) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= L.ncols) return;
    const int d = batch_domain(L.col0, L.ndom, g);
    const BatchBed &B = L.bed[par * L.nall + L.d0 + d];
    if (!B.cg) return;
    const int a = (int)(g - L.col0[d]), j = a / B.D.nx, i = a - j * B.D.nx;
    BedView V;
    V.h = B.h; V.hmax = B.hmax; V.uw = B.uw; V.vw = B.vw; V.ww = B.ww; V.cg = B.cg;
    colgeo_column(B.P, B.D, V, j, i, B.cg);
}

// KIND 0: pre-pass, 1: collide, 2: stream (column-cache kernels)
template <int S, int IN, int KIND>
__global__ void __launch_bounds__(256, KIND == 0 ? LBM_CG_PRE_MINB : LBM_CG_MINB)
    kb_general(const __grid_constant__ BatchGroup G) {
    const int4 m = G.map[blockIdx.x];
    const StepArgs &A = G.a[m.x];
    const int gz = A.zcnt[0] + A.zcnt[1] + A.zcnt[2];
    if constexpr (KIND == 0) prepass_body<S, IN, true>(A, m.y, m.z, m.w, gz);
    else if constexpr (KIND == 1) collide_body<S, IN, true>(A, m.y, m.z, m.w, gz);
    else stream_body<S, true>(A, m.y, m.z, m.w);
}

template <int S>
__global__ void __launch_bounds__(256) kb_stream_interior(const __grid_constant__ BatchGroup G) {
    const int4 m = G.map[blockIdx.x];
    stream_interior_body<S>(G.a[m.x], m.y, m.z, m.w);
}

}  // namespace lbm
