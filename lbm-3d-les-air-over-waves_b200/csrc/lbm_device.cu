// lbm_device.cu - every kernel of the B200 D3Q19 step engine and its
// launcher (one translation unit, so the constant-slot parameter copies
// c_params[] exist once).
//
// Kernel map (reference kernel -> here):
//   update_wave_bed_and_velocities           k_bed + k_hmax (2-D)
//   compute_phi / build_lattice_open         recomputed per cell (lbm_geom.cuh)
//   update_bed_populations + macro_step +
//   compute_LES + collide_*                  k_collide<IN=0> (from the post-stream state)
//   stream + x walls + open BCs, then the
//   next step's condition + macro + LES +
//   collide                                  k_collide<IN=1> (air path, one pass per step)
//   stream + x walls + open BCs (+ water
//   post-stream macro_step)                  k_stream
//   velocity stencil of compute_LES          k_prepass (u of every cell)
//   compute_free_surface_column_flux         k_column_flux
//   advect_free_surface_height               k_advect
//   refill_new_free_surface_cells            k_refill
//   init_constants ... init_fields           k_init_* (setup)
#define LBM_DEVICE_TU
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lbm_launch.h"
#include "lbm_stages.cuh"
#include "lbm_tile.cuh"
#include "lbm_vof.cuh"
#include "lbm_diag.cuh"

namespace lbm {

cudaError_t upload_params(int slot, const lbm_params &P) {
    return cudaMemcpyToSymbol(c_params, &P, sizeof(lbm_params), (size_t)slot * sizeof(lbm_params),
                              cudaMemcpyHostToDevice);
}

static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// kernels launched by this library since the process started
static std::atomic<long long> g_launches{0};
long long launch_count() { return g_launches.load(); }
void launch_count_add(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
#define LAUNCHED(n) g_launches.fetch_add((n), std::memory_order_relaxed)

// 3-D launch of the general kernels: block (32, 8) covering x [32 bx, 32 bx
// + 32) and y [8 by, 8 by + 8) of the bz-th plane of the launch's z ranges
// (a domain's own launch: grid (ceil(nx/32), ceil(ny/8), planes))
__device__ __forceinline__ bool cell_xyz(const StepArgs &A, int bx, int by, int bz, int &i, int &j, int &k, int &c) {
    const Dom &D = A.D;
    i = bx * 32 + threadIdx.x;
    j = by * 8 + threadIdx.y;
    if (bz < A.zcnt[0]) k = A.zlo[0] + bz;
    else if (bz < A.zcnt[0] + A.zcnt[1]) k = A.zlo[1] + (bz - A.zcnt[0]);
    else k = A.zlo[2] + (bz - A.zcnt[0] - A.zcnt[1]);
    if (i >= D.nx || j >= D.ny) return false;
    c = (k * D.ny + j) * D.nx + i;
    return true;
}
static inline dim3 grid3(const StepArgs &A) {
    return dim3((A.D.nx + 31) / 32, (A.D.ny + 7) / 8, A.zcnt[0] + A.zcnt[1] + A.zcnt[2]);
}
static const dim3 kBlock3(32, 8, 1);

__device__ __forceinline__ void cell_of(const Dom &D, int c, int &k, int &j, int &i) {
    k = c / (int)D.a;
    int r = c - k * (int)D.a;
    j = r / D.nx;
    i = r - j * D.nx;
}

// ------------------------------------------------- free-surface heights
// solitary_surface_height_at_x, CODEX.py:1165-1181
__device__ __forceinline__ float solitary_h(const lbm_params &P, const Dom &D, float xp, float t) {
    float Lx = (float)D.nx * P.dx;
    float h0 = P.fs_depth_m;
    float ks = sqrtf((float)(3.0 * (double)P.solitary_amp_m) / (4.0f * h0 * h0 * h0));
    float center = P.solitary_x0_m + P.solitary_dir_cel * t;
    float xrel = xp - center;
    if (!P.x_solid) {
        if (xrel > 0.5f * Lx) xrel -= Lx;
        if (xrel < -0.5f * Lx) xrel += Lx;
    }
    float arg = ks * xrel;
    float ep = lbm_expf(arg), em = lbm_expf(-arg);
    float sech = 2.0f / (ep + em);
    return P.fs_base_m + P.solitary_amp_m * sech * sech;
}
// gaussian_surface_height_at_x, CODEX.py:1184-1194
__device__ __forceinline__ float gaussian_h(const lbm_params &P, const Dom &D, float xp) {
    float Lx = (float)D.nx * P.dx;
    float xrel = xp - P.gaussian_center_x_m;
    if (!P.x_solid) {
        if (xrel > 0.5f * Lx) xrel -= Lx;
        if (xrel < -0.5f * Lx) xrel += Lx;
    }
    float arg = xrel / P.gaussian_sigma_m;
    return P.fs_base_m + P.gaussian_amp_m * lbm_expf(-0.5f * arg * arg);
}

// ------------------------------------------------------------- bed (2-D)
// update_wave_bed_and_velocities, CODEX.py:1082-1162, harmonics generalised,
// for column a at time t
__device__ __forceinline__ void bed_column(const lbm_params &P, const Dom &D, const float *__restrict__ h_prev,
                                           float *h, float *uw, float *vw, float *ww,
                                           const float *__restrict__ piecewise, float t, int a) {
    int i = a % D.nx;
    const bool moving = P.bed_profile == LBM_BED_MOVING_SINE;
    float a1 = 0.0f, a2 = 0.0f;
    if (moving) {
        if (t < P.bed_ramp_time) {
            float s = smooth01(t / P.bed_ramp_time);
            a1 = P.bed_amp1 * s;
            a2 = P.bed_amp2 * s;
        } else {
            a1 = P.bed_amp1;
            a2 = P.bed_amp2;
        }
    }
    float x0 = (float)i * P.dx;
    float hl = h_prev[a];
    float eta1 = 0.0f, eta2 = 0.0f, eta = 0.0f, ph1 = 0.0f, ph2 = 0.0f;
    if (moving) {
        float xph1 = x0 - P.bed_c1 * t;
        float xph2 = x0 - P.bed_c2 * t;
        ph1 = P.bed_k1 * xph1;
        ph2 = P.bed_k2 * xph2;
        eta1 = a1 * lbm_sinf(ph1);
        eta2 = a2 * lbm_sinf(ph2);
        eta = eta1 + eta2;
    }
    float bh = P.bed_offset_m + eta;
    if (P.bed_profile == LBM_BED_PIECEWISE) bh = piecewise[i];
    h[a] = bh;
    float us = 0.0f, vs = 0.0f, ws = 0.0f;
    if (moving) {
        float ex1 = a1 * P.bed_k1 * lbm_cosf(ph1);
        float ex2 = a2 * P.bed_k2 * lbm_cosf(ph2);
        float eta_x = ex1 + ex2;
        float eta_y = 0.0f;
        float eta_t = (bh - hl) / P.dt_phys_f;
        if (P.bed_orbital_velocity) us = P.bed_c1 * eta1 / (P.bed_h0 + eta1) + P.bed_c2 * eta2 / (P.bed_h0 + eta2);
        ws = eta_t + us * eta_x + vs * eta_y;
    }
    uw[a] = us / P.vel_scale;
    vw[a] = vs / P.vel_scale;
    ww[a] = ws / P.vel_scale;
}
__global__ void k_bed(lbm_params P, Dom D, const float *__restrict__ h_prev, float *h, float *uw, float *vw,
                      float *ww, const float *__restrict__ piecewise, float t, const long long *clock, long long off) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)D.a) return;
    if (clock) t = (float)((double)(*clock + off + 1) * P.dt_phys);  // the host's step time, CODEX.py:3874
    bed_column(P, D, h_prev, h, uw, vw, ww, piecewise, t, a);
}

// max of the bed over the 3x3 column neighbourhood (periodic): the support
// of every link-endpoint sample of the column
__device__ __forceinline__ void hmax_column(const Dom &D, const float *__restrict__ h, float *hmax, int a) {
    int j = a / D.nx, i = a - j * D.nx;
    float m = -3.4e38f;
    for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
            int jj = (j + dj + D.ny) % D.ny, ii = (i + di + D.nx) % D.nx;
            m = fmaxf(m, h[D.col(jj, ii)]);
        }
    hmax[a] = m;
}
__global__ void k_hmax(Dom D, const float *__restrict__ h, float *hmax) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)D.a) return;
    hmax_column(D, h, hmax, a);
}

// per-column link-endpoint cache of one bed state (bed-only geometry)
__global__ void k_colgeo(lbm_params P, Dom D, BedView B, float *cg) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)D.a) return;
    const int j = a / D.nx, i = a - j * D.nx;
    colgeo_column(P, D, B, j, i, cg);
}

// ------------------------------------------------------- step kernels
// resident blocks per SM requested for the general kernels without the
// column cache (water, VOF, cube, phi geometry, solid x walls): three, which
// spills some registers of their long near-wall paths but triples the warps
// that hide their load latency (water height 256x128x96: 2,251 -> 2,939
// MLUPS, VOF 128x64x128: 334 -> 444 MLUPS, against one block per SM)
#ifndef LBM_GEN_MINB
#define LBM_GEN_MINB 3
#endif
#ifndef LBM_CG_PRE_MINB
#define LBM_CG_PRE_MINB 3   // the column-cache pre-pass: 3 blocks of 256 per SM (85 registers)
#endif
#ifndef LBM_CG_MINB
#define LBM_CG_MINB 2
#endif
template <int S>
__device__ __forceinline__ void load_cell(const StepArgs &A, int c, float f[19]) {
    const typename Store<S>::T *src = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = Store<S>::ld(src, (size_t)q * A.D.n + (size_t)c, q, A.P.rho0);
}
template <int S>
__device__ __forceinline__ void store_cell(const StepArgs &A, int c, const float f[19]) {
    typename Store<S>::T *dst = (typename Store<S>::T *)A.fdst;
#pragma unroll
    for (int q = 0; q < 19; ++q) Store<S>::st(dst, (size_t)q * A.D.n + (size_t)c, f[q], q, A.P.rho0);
}

// Populations entering the collide step, then the condition and macro
// stages on the collide step's geometry.  IN = 0: from the stored
// post-stream state; IN = 1: stream + BC of the previous step from its
// post-collision state.  Cells away from every wall and boundary take the
// plain gather; the general path handles the rest.
// Stream-stage class of a water cell on the height path: 1 = gas cell,
// 2 = cell whose sources are all wet, 0 = anything else; in classes 1 and 2
// the cell is away from the bed (its link endpoints are more than half a
// cell above the 3x3 bed maximum), above the bottom row, below the top row
// (class 2), and there is no cube, phi geometry, fringe or top drive, so
// stream_bc gives:
// the rest equilibrium (gas) or the plain gather (wet sources) on every
// link, except the links through a solid x wall, which carry the cell's own
// opposite population.  Wet sources: the lowest free-surface height over
// the 3x3 columns is more than 1.01 cells above the top source plane's
// bottom, so every source fill exceeds 1e-4.
__device__ __forceinline__ int vof_stream_class(const StepArgs &A, int k, int j, int i);
__device__ __forceinline__ int water_stream_class(const StepArgs &A, int k, int j, int i) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    if (P.fs_mode == LBM_FS_NONE) return 0;
    if (A.flags & F_VOF_STATE) return vof_stream_class(A, k, j, i);
    if (k < 1 || k > D.nz - 1) return 0;
    if (P.enable_x_fringe || P.enable_top_drive || P.include_cube || P.use_phi_open_fraction ||
        P.use_phi_open_flags)
        return 0;
    const float dx = P.dx, hdx = 0.5f * dx;
    if (P.include_bed) {
        const float zc = ((float)k + 0.5f) * dx;
        const float hm = __ldg(A.bed_s.hmax + D.col(j, i));
        const float margin = 1e-4f * dx + 1e-6f * (fabsf(zc) + fabsf(hm));
        if (!((zc - hdx) - hm >= hdx + margin)) return 0;
    }
    int type;
    float fill;
    classify_height(P, __ldg(A.fs_h + D.col(j, i)), k, true, type, fill);
    if (type == LBM_FS_GAS) return 1;   // the top row too: stream_bc gives a gas cell the rest equilibrium
    if (k == D.nz - 1) return 0;
    int im = i == 0 ? D.nx - 1 : i - 1, ip = i + 1 == D.nx ? 0 : i + 1;
    if (P.x_solid) {
        if (i == 0) im = i;
        if (i + 1 == D.nx) ip = i;
    }
    const int jm = j == 0 ? D.ny - 1 : j - 1, jp = j + 1 == D.ny ? 0 : j + 1;
    float hmin = __ldg(A.fs_h + D.col(j, i));
    const int cols[8] = {D.col(jm, im), D.col(jm, i), D.col(jm, ip), D.col(j, im), D.col(j, ip), D.col(jp, im),
                         D.col(jp, i), D.col(jp, ip)};
#pragma unroll
    for (int u = 0; u < 8; ++u) hmin = fminf(hmin, __ldg(A.fs_h + cols[u]));
    return hmin > ((float)k + 1.01f) * dx ? 2 : 0;
}

// The same classes on the VOF path, from the stored cell types, away from
// solid x walls: 1 = open gas cell (stream_bc gives the rest equilibrium and
// no wall bounce-back), 2 = liquid cell below the top row whose 18 sources
// are liquid (every link takes the plain gather: no free-surface link, link
// aperture 1), 0 = anything else.
__device__ __forceinline__ int vof_stream_class(const StepArgs &A, int k, int j, int i) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    if (k < 1 || k > D.nz - 1) return 0;
    if (P.x_solid && (i == 0 || i == D.nx - 1)) return 0;
    if (P.enable_x_fringe || P.enable_top_drive || P.include_cube || P.use_phi_open_fraction ||
        P.use_phi_open_flags)
        return 0;
    const float dx = P.dx, hdx = 0.5f * dx;
    if (P.include_bed) {
        const float zc = ((float)k + 0.5f) * dx;
        const float hm = __ldg(A.bed_s.hmax + D.col(j, i));
        const float margin = 1e-4f * dx + 1e-6f * (fabsf(zc) + fabsf(hm));
        if (!((zc - hdx) - hm >= hdx + margin)) return 0;
    }
    const int type = A.fs_type[D.cell(k, j, i)];
    if (type == LBM_FS_GAS) return 1;
    if (type != LBM_FS_LIQUID || k == D.nz - 1) return 0;
    const int im = i == 0 ? D.nx - 1 : i - 1, ip = i + 1 == D.nx ? 0 : i + 1;
    const int jm = j == 0 ? D.ny - 1 : j - 1, jp = j + 1 == D.ny ? 0 : j + 1;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const int si = cxq(q) > 0 ? im : (cxq(q) < 0 ? ip : i);
        const int sj = cyq(q) > 0 ? jm : (cyq(q) < 0 ? jp : j);
        if (A.fs_type[D.cell(k - czq(q), sj, si)] != LBM_FS_LIQUID) return 0;
    }
    return 2;
}

// Water cell (height or VOF path) whose collide needs no link geometry: farther than
// half a cell from the bed, no cube, phi geometry, fringe or top drive (the
// top and bottom rows included: the domain's z ends close no link).  Its own
// link (q = 0) is open, and every closed link is an x wall, where the water
// path's condition stage applies nothing (only bed links, or any link in
// air physics, are conditioned).
__device__ __forceinline__ bool water_collide_local(const StepArgs &A, int k, int j, int i) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    if (P.fs_mode == LBM_FS_NONE || !P.physics_water) return false;
    if (P.enable_x_fringe || P.enable_top_drive || P.include_cube || P.use_phi_open_fraction ||
        P.use_phi_open_flags)
        return false;
    if (P.include_bed) {
        const float dx = P.dx, hdx = 0.5f * dx;
        const float zc = ((float)k + 0.5f) * dx;
        const float hm = __ldg(A.bed_c.hmax + D.col(j, i));
        const float margin = 1e-4f * dx + 1e-6f * (fabsf(zc) + fabsf(hm));
        if (!((zc - hdx) - hm >= hdx + margin)) return false;
    }
    return true;
}

// gas_free: the caller does not read the populations of a gas cell (the
// velocity pre-pass, whose gas velocity is zero, and the regularized
// collision, whose gas output is the rest equilibrium), so with a free
// surface they are not loaded for gas cells
template <int S, int IN, bool CG>
__device__ __forceinline__ void front(const StepArgs &A, int c, int k, int j, int i, float f[19], bool &fast_c,
                                      bool &open, int &type, float &gbf, float &r, float &vx, float &vy, float &vz,
                                      bool gas_free = false) {
    const lbm_params &P = A.P;
    // the column cache is used in air mode only: CG kernels carry no
    // free-surface code
    const bool water = !CG && P.fs_mode != LBM_FS_NONE;
    if (cell_fast(A, IN == 1, true, k, j, i)) {
        if (IN == 0) load_cell<S>(A, c, f);
        else stream_fast<S>(A, (const typename Store<S>::T *)A.fsrc, k, j, i, c, f);
        fast_c = true;
        open = true;
        type = LBM_FS_LIQUID;
        gbf = 0.0f;
        macro(P, A.D, f, k, false, type, gbf, r, vx, vy, vz);
        return;
    }
    GeoLinks Lc;
    Geo gc = geo_cell<CG>(P, A.slot, A.D, A.bed_c, k, j, i, Lc, true, P.use_link_wall_velocity && P.include_bed);
    fast_c = gc.fast;
    open = (gc.lo & 1u) != 0u;
    type = LBM_FS_LIQUID;
    float fill = 1.0f;
    gbf = 0.0f;
    if (water) {
        fs_state(A, c, k, j, i, open, type, fill);
        gbf = gbf_of(P, k, open, type);
    }
    // A cell with every link closed in the collide geometry (air): the
    // condition stage sets f_q = frac_q f_q + (1 - frac_q) feq_q on every
    // link, with frac_q = 0 for q >= 1, so only the rest population of the
    // stream stage survives (the others enter multiplied by zero).  The
    // stream stage leaves f_0 local here (no fringe, no top drive at this
    // cell), so the gather and the stream geometry are skipped.
    const bool solid_c = gc.lo == 0u && !water && !P.physics_water &&
                         !(P.enable_x_fringe && i < 5 && k > A.D.nz / 2) &&
                         !(P.enable_top_drive && k == A.D.nz - 1);
    if (water && gas_free && type == LBM_FS_GAS) {
        // macro_step gives (rho0, 0) for a gas cell whatever its populations
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = 0.0f;
    } else if (solid_c) {
        f[0] = Store<S>::ld((const typename Store<S>::T *)A.fsrc, (size_t)c, 0, P.rho0);
#pragma unroll
        for (int q = 1; q < 19; ++q) f[q] = 0.0f;
    } else if (IN == 0) {
        load_cell<S>(A, c, f);
    } else {
        GeoLinks Ls;
        Geo gs = geo_cell<CG>(P, A.slot, A.D, A.bed_s, k, j, i, Ls, true, P.use_link_wall_velocity && P.include_bed);
        int cut = 0, fscut = 0, bridge = 0;
        stream_bc<S, CG>(A, (const typename Store<S>::T *)A.fsrc, gs, Ls, k, j, i, c, f, cut, fscut, bridge);
    }
    condition(P, A.D, A.bed_c, gc, Lc, k, j, i, f);
    macro(P, A.D, f, k, water, type, gbf, r, vx, vy, vz);
}

// Bodies of the general kernels, with the block's coordinates explicit (bz
// walks the launch's z ranges, gz is their total), so that one body serves
// a domain's own launch and the batched launches over many domains.
template <int S, int IN, bool CG>
__device__ __forceinline__ void prepass_body(const StepArgs &A, int bx, int by, int bz, int gz) {
    int i, j, k, c;
    if (!cell_xyz(A, bx, by, bz, i, j, k, c)) return;
    float f[19], r, vx, vy, vz, gbf;
    int type;
    bool fast_c, open;
    // with the stash the collide pass reads these populations back; without
    // it only the velocity is used
    const bool gas_free = !(CG && (A.flags & F_STASH));
    front<S, IN, CG>(A, c, k, j, i, f, fast_c, open, type, gbf, r, vx, vy, vz, gas_free);
    A.u_out[c] = vx;
    A.u_out[A.D.n + c] = vy;
    A.u_out[2 * A.D.n + c] = vz;
    // the collide pass of these cells reads the populations back: from its
    // own destination slots (FP32), or from the FP32 stash indexed by the
    // launch's plane (16-bit storage would round them)
    if (CG && (A.flags & F_STASH)) {
        if (S == LBM_STORE_F32) {
            store_cell<S>(A, c, f);
        } else {
            const size_t ng = (size_t)gz * A.D.nx * A.D.ny;
            const size_t g = ((size_t)bz * A.D.ny + j) * A.D.nx + i;
#pragma unroll
            for (int q = 0; q < 19; ++q) A.stash[q * ng + g] = f[q];
        }
    }
}
template <int S, int IN, bool CG>
__global__ void __launch_bounds__(256, CG ? LBM_CG_PRE_MINB : LBM_GEN_MINB) k_prepass(StepArgs A) {
    prepass_body<S, IN, CG>(A, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.z);
}

template <int S, int IN, bool CG>
__device__ __forceinline__ void collide_cell(const StepArgs &A, int k, int j, int i, int c, int bz, int gz) {
    float f[19], r, vx, vy, vz, gbf;
    int type;
    bool fast_c, open;
    if (CG && (A.flags & F_STASH)) {
        // populations after stream, boundary conditions and condition
        // stage, left by the pre-pass in the destination slots (FP32) or
        // in the stash (16-bit storage)
        if (S == LBM_STORE_F32) {
            const float *fd = (const float *)A.fdst;
#pragma unroll
            for (int q = 0; q < 19; ++q) f[q] = fd[(size_t)q * A.D.n + c];
        } else {
            const size_t ng = (size_t)gz * A.D.nx * A.D.ny;
            const size_t g = ((size_t)bz * A.D.ny + j) * A.D.nx + i;
#pragma unroll
            for (int q = 0; q < 19; ++q) f[q] = A.stash[q * ng + g];
        }
        GeoLinks Lc;
        Geo gc = geo_cell<CG>(A.P, A.slot, A.D, A.bed_c, k, j, i, Lc, true, false);
        fast_c = gc.fast;
        open = (gc.lo & 1u) != 0u;
        type = LBM_FS_LIQUID;
        gbf = 0.0f;
        macro(A.P, A.D, f, k, false, type, gbf, r, vx, vy, vz);
    } else {
        front<S, IN, CG>(A, c, k, j, i, f, fast_c, open, type, gbf, r, vx, vy, vz,
                         A.P.collision == LBM_COLLIDE_REGULARIZED);
    }
    const lbm_params &P = A.P;
    const bool water = !CG && P.fs_mode != LBM_FS_NONE;
    const bool gas = water && type == LBM_FS_GAS;
    if (A.flags & F_WRITE_MACRO) {
        A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
    }
    if (!(r == r) || fabsf(r) > 3.0e38f) atomicOr(A.status, 1u);
    float om;
    if (P.use_les) {
        if (open && !gas) {
            om = les_omega(A, k, j, i, c, vx, vy, vz);
            if ((A.flags & F_WRITE_ALL_OMEGA) || !fast_c) A.omega[c] = om;
        } else {
            om = A.omega[c];
        }
    } else {
        om = P.omega0;
    }
    collide(A, c, k, !open, water, gas, gbf, r, vx, vy, vz, om, f);
    store_cell<S>(A, c, f);
}
template <int S, int IN, bool CG>
__device__ __forceinline__ void collide_body(const StepArgs &A, int bx, int by, int bz, int gz) {
    int i, j, k, c;
    if (!cell_xyz(A, bx, by, bz, i, j, k, c)) return;
    collide_cell<S, IN, CG>(A, k, j, i, c, bz, gz);
}
template <int S, int IN, bool CG>
__global__ void __launch_bounds__(256, CG ? LBM_CG_MINB : LBM_GEN_MINB) k_collide(StepArgs A) {
    collide_body<S, IN, CG>(A, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.z);
}

template <int S, bool CG>
__device__ __forceinline__ void stream_cell(const StepArgs &A, int k, int j, int i, int c, int wcls, int &cut,
                                            int &fscut, int &bridge) {
    {
        float f[19];
        if (cell_fast(A, true, false, k, j, i)) {
            stream_fast<S>(A, (const typename Store<S>::T *)A.fsrc, k, j, i, c, f);
            store_cell<S>(A, c, f);
        } else if (wcls != 0) {
            // water, height path, away from the bed and the x walls: a gas
            // cell takes the rest equilibrium, a cell whose sources are all
            // wet the plain gather; then the post-stream macro step
            const bool xwall = A.P.x_solid && (i == 0 || i + 1 == A.D.nx);
            if (wcls == 1) {
                f[0] = feq<0>(A.P.rho0, 0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                for (int q = 1; q < 19; ++q) f[q] = A.P.rho0 * wq(q) * 1.0f;
            } else if (!xwall) {
                stream_fast<S>(A, (const typename Store<S>::T *)A.fsrc, k, j, i, c, f);
            } else {
                // pull from inside the domain (periodic y); the wall links are set below
                const typename Store<S>::T *fs = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const int si = i - cxq(q);
                    if (si < 0 || si >= A.D.nx) continue;
                    const int sj = (j - cyq(q) + A.D.ny) % A.D.ny;
                    f[q] = Store<S>::ld(fs, (size_t)q * A.D.n + A.D.cell(k - czq(q), sj, si), q, A.P.rho0);
                }
            }
            if (xwall) {
                const typename Store<S>::T *fs = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
                for (int q = 1; q < 19; ++q) {
                    if ((i == 0 && cxq(q) > 0) || (i + 1 == A.D.nx && cxq(q) < 0)) {
                        f[q] = Store<S>::ld(fs, (size_t)oppq(q) * A.D.n + c, oppq(q), A.P.rho0);
                        if (wcls == 2) cut++;
                    }
                }
            }
            store_cell<S>(A, c, f);
            int type;
            float fill;
            fs_state(A, c, k, j, i, true, type, fill);
            const float gbf = gbf_of(A.P, k, true, type);
            float r, vx, vy, vz;
            macro(A.P, A.D, f, k, true, type, gbf, r, vx, vy, vz);
            A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
        } else {
            GeoLinks Ls;
            Geo gs = geo_cell<CG>(A.P, A.slot, A.D, A.bed_s, k, j, i, Ls, true, A.P.use_link_wall_velocity && A.P.include_bed);
            stream_bc<S, CG>(A, (const typename Store<S>::T *)A.fsrc, gs, Ls, k, j, i, c, f, cut, fscut, bridge);
            store_cell<S>(A, c, f);
            if (!CG && A.P.fs_mode != LBM_FS_NONE) {
                // post-stream macro_step of the water path, CODEX.py:3897
                int type;
                float fill;
                bool open = (gs.lo & 1u) != 0u;
                fs_state(A, c, k, j, i, open, type, fill);
                float gbf = gbf_of(A.P, k, open, type);
                float r, vx, vy, vz;
                macro(A.P, A.D, f, k, true, type, gbf, r, vx, vy, vz);
                A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
            }
        }
    }
}

// the stream counters of a warp (cut, free-surface cut, bridge links)
__device__ __forceinline__ void stream_counts(const StepArgs &A, int cut, int fscut, int bridge) {
    if (A.flags & F_COUNT) {
        unsigned m = __activemask();
        int s0 = __reduce_add_sync(m, cut), s1 = __reduce_add_sync(m, fscut), s2 = __reduce_add_sync(m, bridge);
        if ((threadIdx.x & 31) == 0) {
            if (s0) atomicAdd(A.counters + 0, s0);
            if (s1) atomicAdd(A.counters + 1, s1);
            if (s2) atomicAdd(A.counters + 2, s2);
        }
    }
}

template <int S, bool CG>
__device__ __forceinline__ void stream_body(const StepArgs &A, int bx, int by, int bz) {
    int i, j, k, c;
    int cut = 0, fscut = 0, bridge = 0;
    if (cell_xyz(A, bx, by, bz, i, j, k, c)) {
        const int wcls = CG ? 0 : water_stream_class(A, k, j, i);
        stream_cell<S, CG>(A, k, j, i, c, wcls, cut, fscut, bridge);
    }
    stream_counts(A, cut, fscut, bridge);
}
template <int S, bool CG>
__global__ void __launch_bounds__(256, CG ? LBM_CG_MINB : LBM_GEN_MINB) k_stream(StepArgs A) {
    stream_body<S, CG>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ------------------------------------------------ compact kernels of water
// The cells that water_collide_local (collide) or water_stream_class (stream)
// admit take the same stage functions as in the general kernels, in kernels
// that carry none of the near-wall, free-surface-cut or VOF code, so they are
// small enough to run without register spills or instruction-cache misses.
// They list the other cells, and the general collide / stream run over the
// list only (k_collide_list, k_stream_list).
// list / count: the cells left to the general collide are appended, for k_collide_list
template <int S, int COLL>
__device__ __forceinline__ void collide_water_cell(const StepArgs &A, int k, int j, int i, int c);
#ifndef LBM_WATER_MINB
#define LBM_WATER_MINB 3   // resident blocks per SM of the compact water collide (80 registers, a few spilled)
#endif
template <int S, int COLL>
__global__ void __launch_bounds__(256, LBM_WATER_MINB) k_collide_water(StepArgs A, int *list, int *count) {
    int i, j, k, c;
    bool local = false, general = false;
    if (cell_xyz(A, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k, c)) {
        local = water_collide_local(A, k, j, i);
        general = !local;
    }
    const unsigned lanes = __ballot_sync(0xffffffffu, general);
    if (lanes) {
        const int lane = threadIdx.x & 31, lead = __ffs(lanes) - 1;
        int base = 0;
        if (lane == lead) base = atomicAdd(count, __popc(lanes));
        base = __shfl_sync(0xffffffffu, base, lead);
        if (general) list[base + __popc(lanes & ((1u << lane) - 1u))] = c;
    }
    if (local) collide_water_cell<S, COLL>(A, k, j, i, c);
}
// the general collide over the cells k_collide_water left (grid-stride over the list)
template <int S>
__global__ void __launch_bounds__(256, 2) k_collide_list(StepArgs A, const int *list, const int *count) {
    const int nl = *count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nl; e += gridDim.x * blockDim.x) {
        const int c = list[e];
        int k, j, i;
        cell_of(A.D, c, k, j, i);
        collide_cell<S, 0, false>(A, k, j, i, c, 0, 1);
    }
}
template <int S, int COLL>
__device__ __forceinline__ void collide_water_cell(const StepArgs &A, int k, int j, int i, int c) {
    const lbm_params &P = A.P;
    // front() for such a cell: open, no closed link to condition
    const bool fast_c = !(P.x_solid && (i == 0 || i == A.D.nx - 1));
    int type;
    float fill;
    fs_state(A, c, k, j, i, true, type, fill);
    const float gbf = gbf_of(P, k, true, type);
    const bool gas = type == LBM_FS_GAS;
    float f[19];
    if (gas && COLL == LBM_COLLIDE_REGULARIZED) {
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = 0.0f;   // macro_step gives (rho0, 0) for a gas cell
    } else {
        load_cell<S>(A, c, f);
    }
    float r, vx, vy, vz;
    macro(P, A.D, f, k, true, type, gbf, r, vx, vy, vz);
    if (A.flags & F_WRITE_MACRO) {
        A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
    }
    if (!(r == r) || fabsf(r) > 3.0e38f) atomicOr(A.status, 1u);
    float om;
    if (P.use_les) {
        if (!gas) {
            om = les_omega(A, k, j, i, c, vx, vy, vz);
            if ((A.flags & F_WRITE_ALL_OMEGA) || !fast_c) A.omega[c] = om;
        } else {
            om = A.omega[c];
        }
    } else {
        om = P.omega0;
    }
    collide<COLL>(A, c, k, false, true, gas, gbf, r, vx, vy, vz, om, f);
    store_cell<S>(A, c, f);
}

// list / count: the cells left to the general path are appended (one
// warp-aggregated atomic per warp), for k_stream_list
template <int S>
__global__ void __launch_bounds__(256, 2) k_stream_water(StepArgs A, int *list, int *count) {
    int i, j, k, c;
    int cut = 0;
    bool general = false;
    if (cell_xyz(A, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k, c)) {
        const int wcls = water_stream_class(A, k, j, i);
        general = wcls == 0;
        if (wcls != 0) {
            // the water branch of stream_body: a gas cell takes the rest
            // equilibrium, a cell whose sources are all wet the plain gather
            // (links through a solid x wall carry the cell's own opposite
            // population); then the post-stream macro step
            float f[19];
            const typename Store<S>::T *fs = (const typename Store<S>::T *)A.fsrc;
            const bool xwall = A.P.x_solid && (i == 0 || i + 1 == A.D.nx);
            if (wcls == 1) {
                f[0] = feq<0>(A.P.rho0, 0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                for (int q = 1; q < 19; ++q) f[q] = A.P.rho0 * wq(q) * 1.0f;
            } else if (!xwall) {
                stream_fast<S>(A, fs, k, j, i, c, f);
            } else {
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const int si = i - cxq(q);
                    if (si < 0 || si >= A.D.nx) continue;
                    const int sj = (j - cyq(q) + A.D.ny) % A.D.ny;
                    f[q] = Store<S>::ld(fs, (size_t)q * A.D.n + A.D.cell(k - czq(q), sj, si), q, A.P.rho0);
                }
            }
            if (xwall) {
#pragma unroll
                for (int q = 1; q < 19; ++q) {
                    if ((i == 0 && cxq(q) > 0) || (i + 1 == A.D.nx && cxq(q) < 0)) {
                        f[q] = Store<S>::ld(fs, (size_t)oppq(q) * A.D.n + c, oppq(q), A.P.rho0);
                        if (wcls == 2) cut++;
                    }
                }
            }
            store_cell<S>(A, c, f);
            int type;
            float fill;
            fs_state(A, c, k, j, i, true, type, fill);
            const float gbf = gbf_of(A.P, k, true, type);
            float r, vx, vy, vz;
            macro(A.P, A.D, f, k, true, type, gbf, r, vx, vy, vz);
            A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
        }
    }
    const unsigned lanes = __ballot_sync(0xffffffffu, general);
    if (lanes) {
        const int lane = threadIdx.x & 31, lead = __ffs(lanes) - 1;
        int base = 0;
        if (lane == lead) base = atomicAdd(count, __popc(lanes));
        base = __shfl_sync(0xffffffffu, base, lead);
        if (general) list[base + __popc(lanes & ((1u << lane) - 1u))] = c;
    }
    if (A.flags & F_COUNT) {
        const int s0 = __reduce_add_sync(0xffffffffu, cut);
        if ((threadIdx.x & 31) == 0 && s0) atomicAdd(A.counters + 0, s0);
    }
}

// the general stream over the cells k_stream_water left (grid-stride over the list)
template <int S>
__global__ void __launch_bounds__(256, 2) k_stream_list(StepArgs A, const int *list, const int *count) {
    const int nl = *count;
    int cut = 0, fscut = 0, bridge = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nl; e += gridDim.x * blockDim.x) {
        const int c = list[e];
        int k, j, i;
        cell_of(A.D, c, k, j, i);
        stream_cell<S, false>(A, k, j, i, c, 0, cut, fscut, bridge);
    }
    stream_counts(A, cut, fscut, bridge);
}

}  // namespace lbm

#include "lbm_batch.cuh"

namespace lbm {

// -------------------------------------------- height-function free surface
// compute_free_surface_column_flux, CODEX.py:2376-2388.  A block covers 32
// columns of one row (x fastest, so the velocity loads coalesce) with 8
// warps over z: the terms fill u vel_scale dx of FLUX_KC planes are formed in
// parallel into shared memory, then one warp per component adds them in
// plane order, so each column's sum is the reference's sequential one.  A
// gas or closed cell adds +0, which leaves a sum that starts at +0 unchanged.
constexpr int FLUX_KC = 64;
__global__ void __launch_bounds__(256, 4) k_column_flux(StepArgs A, float *qx_out, float *qy_out) {
    __shared__ float sq[2][FLUX_KC][33];
    const Dom &D = A.D;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int nbx = (D.nx + 31) / 32;
    const int j = blockIdx.x / nbx, i = (blockIdx.x - j * nbx) * 32 + tx;
    const bool live = i < D.nx;
    const int a = j * D.nx + i;
    const float h = live ? A.fs_h[a] : 0.0f;
    float q = 0.0f;   // warp 0: x flux, warp 1: y flux
    for (int k0 = 0; k0 < D.nz; k0 += FLUX_KC) {
        for (int kk = ty; kk < FLUX_KC; kk += 8) {
            const int k = k0 + kk;
            float tqx = 0.0f, tqy = 0.0f;
            if (live && k < D.nz) {
                int type;
                float fill;
                classify_height(A.P, h, k, true, type, fill);
                if (type != LBM_FS_GAS && cell_open(A.P, A.slot, D, A.bed_s, k, j, i)) {
                    const int c = D.cell(k, j, i);
                    tqx = fill * A.ux[c] * A.P.vel_scale * A.P.dx;
                    tqy = fill * A.uy[c] * A.P.vel_scale * A.P.dx;
                }
            }
            sq[0][kk][tx] = tqx;
            sq[1][kk][tx] = tqy;
        }
        __syncthreads();
        if (ty < 2) {
            const int kn = min(FLUX_KC, D.nz - k0);
#pragma unroll 8
            for (int kk = 0; kk < kn; ++kk) q += sq[ty][kk][tx];
        }
        __syncthreads();
    }
    if (live) {
        if (ty == 0) qx_out[a] = q;
        else if (ty == 1) qy_out[a] = q;
    }
}

// advect_free_surface_height, CODEX.py:2391-2429
__global__ void k_advect(lbm_params P, Dom D, const float *__restrict__ bed_h, const float *__restrict__ qx,
                         const float *__restrict__ qy, const float *h_in, float *h_out, float *h_last, float t) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)D.a) return;
    int j = a / D.nx, i = a - j * D.nx;
    float Lz = (float)D.nz * P.dx;
    float ho = h_in[a];
    float h = ho;
    if (P.fs_mode == LBM_FS_PRESCRIBED_SOLITARY) {
        float x = ((float)i + 0.5f) * P.dx;
        h = solitary_h(P, D, x, t);
    } else if (P.fs_mode == LBM_FS_HEIGHT_KINEMATIC) {
        float dqdx;
        if (P.x_solid) {
            float fl = 0.0f, fr = 0.0f;
            if (i > 0) fl = 0.5f * (qx[D.col(j, i - 1)] + qx[a]);
            if (i < D.nx - 1) fr = 0.5f * (qx[a] + qx[D.col(j, i + 1)]);
            dqdx = (fr - fl) / P.dx;
        } else {
            int ip = (i + 1) % D.nx, im = (i - 1 + D.nx) % D.nx;
            dqdx = (qx[D.col(j, ip)] - qx[D.col(j, im)]) * P.half_inv_dx;
        }
        int jp = (j + 1) % D.ny, jm = (j - 1 + D.ny) % D.ny;
        float dqdy = (qy[D.col(jp, i)] - qy[D.col(jm, i)]) * P.half_inv_dx;
        float dhdt = -(dqdx + dqdy);
        h = ho + P.dt_phys_f * dhdt;
        float mn = bed_h[a] + 0.5f * P.dx;
        float mx = Lz - 0.5f * P.dx;
        if (h < mn) h = mn;
        if (h > mx) h = mx;
    }
    h_last[a] = ho;
    h_out[a] = h;
}

// refill_new_free_surface_cells, CODEX.py:2163-2316.  Height path: the
// before/after states come from h_last/h; VOF path: from the stored
// type_prev/type (F_VOF_STATE).  refill_cell handles one cell and returns 1
// if it refilled it; tp / tn are the cell's types before and after.
template <int S>
__device__ __forceinline__ int refill_cell(const StepArgs &A, const int8_t *type_prev_v, int c, int k, int j, int i,
                                           int tp, int tn) {
    int did = 0;
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const bool vofm = (A.flags & F_VOF_STATE) != 0;
    {
        bool cand = tp == LBM_FS_GAS && tn != LBM_FS_GAS;
        if (cand && cell_open(P, A.slot, D, A.bed_s, k, j, i)) {
            typename Store<S>::T *fb = (typename Store<S>::T *)A.fdst;
            float ws = 0.0f, fws = 0.0f, ra = 0.0f, xa = 0.0f, ya = 0.0f, za = 0.0f;
            float fra = 0.0f, fxa = 0.0f, fya = 0.0f, fza = 0.0f;
            float na[19], nfa[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) { na[q] = 0.0f; nfa[q] = 0.0f; }
#pragma unroll
            for (int qn = 1; qn < 19; ++qn) {
                int nir = i + cxq(qn);
                int nj = pymod(j + cyq(qn) + D.ny, D.ny);
                int nk = k + czq(qn);
                int ni = nir;
                bool valid = true;
                if (!P.x_solid) ni = pymod(nir + D.nx, D.nx);
                else if (nir < 0 || nir >= D.nx) valid = false;
                if (nk < 0 || nk >= D.nz) valid = false;
                if (!valid) continue;
                int nb = D.cell(nk, nj, ni);
                int ntp, ntn;
                float nfl;
                if (vofm) {
                    ntp = type_prev_v[nb];
                    ntn = A.fs_type[nb];
                    nfl = A.fs_fill[nb];
                } else {
                    float dummy;
                    classify_height(P, A.fs_h_last[D.col(nj, ni)], nk, true, ntp, dummy);
                    classify_height(P, A.fs_h[D.col(nj, ni)], nk, true, ntn, nfl);
                }
                if (!(ntp != LBM_FS_GAS && ntn != LBM_FS_GAS)) continue;
                if (!cell_open(P, A.slot, D, A.bed_s, nk, nj, ni)) continue;
                float wn = wq(qn);
                float rn = A.rho[nb], uxn = A.ux[nb], uyn = A.uy[nb], uzn = A.uz[nb];
                fws += wn;
                fra += wn * rn; fxa += wn * uxn; fya += wn * uyn; fza += wn * uzn;
                float lw = wn * nfl;
                ws += lw;
                ra += lw * rn; xa += lw * uxn; ya += lw * uyn; za += lw * uzn;
                if (P.fs_refill == LBM_REFILL_NONEQ) {
                    float u2n = usq(uxn, uyn, uzn);
#pragma unroll
                    for (int qq = 0; qq < 19; ++qq) {
                        float fe = 0.0f;
                        switch (qq) {
#define FQ(Q) case Q: fe = feq<Q>(rn, uxn, uyn, uzn, u2n); break;
                            FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13)
                            FQ(14) FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                        }
                        float fneq = Store<S>::ld_rw(fb, (size_t)qq * D.n + nb, qq, P.rho0) - fe;
                        na[qq] += lw * fneq;
                        nfa[qq] += wn * fneq;
                    }
                }
            }
            float rr = P.rho0;
            if (!vofm) {
                // gravity fraction of the state at the start of the step
                float gbf = gbf_of(P, k, true, tp);
                rr = fs_density_cell(P, A.fs_h[D.col(j, i)], k, gbf);
            }
            float urx = P.u_current_lb, ury = 0.0f, urz = 0.0f;
            if (ws > 0.0f) {
                float iw = 1.0f / ws;
                if (vofm) rr = ra * iw;
                urx = xa * iw; ury = ya * iw; urz = za * iw;
            } else if (fws > 0.0f) {
                float iw = 1.0f / fws;
                if (vofm) rr = fra * iw;
                urx = fxa * iw; ury = fya * iw; urz = fza * iw;
            } else if (vofm) {
                rr = P.rho0;
            }
            float fr[19];
            float rp = 0.0f;
            float u2r = usq(urx, ury, urz);
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                float v = 0.0f;
                switch (q) {
#define FQ(Q) case Q: v = feq<Q>(rr, urx, ury, urz, u2r); break;
                    FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                    FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                }
                if (P.fs_refill == LBM_REFILL_NONEQ) {
                    if (ws > 0.0f) v += na[q] / ws;
                    else if (fws > 0.0f) v += nfa[q] / fws;
                } else if (P.fs_refill == LBM_REFILL_DIRECTIONAL) {
                    int sir = i - cxq(q);
                    int si = sir;
                    int sj = pymod(j - cyq(q) + D.ny, D.ny);
                    int sk = k - czq(q);
                    bool sv = true;
                    if (!P.x_solid) si = pymod(sir + D.nx, D.nx);
                    else if (sir < 0 || sir >= D.nx) sv = false;
                    if (sk < 0 || sk >= D.nz) sv = false;
                    if (sv) {
                        int s = D.cell(sk, sj, si);
                        int stp, stn;
                        float sfl;
                        if (vofm) {
                            stp = type_prev_v[s];
                            stn = A.fs_type[s];
                        } else {
                            classify_height(P, A.fs_h_last[D.col(sj, si)], sk, true, stp, sfl);
                            classify_height(P, A.fs_h[D.col(sj, si)], sk, true, stn, sfl);
                        }
                        if (stp != LBM_FS_GAS && stn != LBM_FS_GAS && cell_open(P, A.slot, D, A.bed_s, sk, sj, si))
                            v = Store<S>::ld_rw(fb, (size_t)q * D.n + s, q, P.rho0);
                    }
                }
                fr[q] = v;
                rp += v;
            }
            if (P.fs_refill == LBM_REFILL_DIRECTIONAL) {
                float scale = 1.0f;
                if (rp > 1.0e-8f) scale = rr / rp;
                rp = 0.0f;
                float mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    float fv = fr[q] * scale;
                    fr[q] = fv;
                    rp += fv;
                    if (cxq(q) > 0) mx += fv; else if (cxq(q) < 0) mx += -fv;
                    if (cyq(q) > 0) my += fv; else if (cyq(q) < 0) my += -fv;
                    if (czq(q) > 0) mz += fv; else if (czq(q) < 0) mz += -fv;
                }
                A.rho[c] = rp;
                if (rp > 1.0e-8f) { A.ux[c] = mx / rp; A.uy[c] = my / rp; A.uz[c] = mz / rp; }
                else { A.ux[c] = urx; A.uy[c] = ury; A.uz[c] = urz; }
            } else {
                A.rho[c] = rr; A.ux[c] = urx; A.uy[c] = ury; A.uz[c] = urz;
            }
            // a refilled cell is never a source for another refilled cell
            // (sources need type_prev != GAS), so writing in place is safe
            store_cell<S>(A, c, fr);
            did = 1;
        }
    }
    return did;
}

// VOF path: one thread per cell, types from the stored fields
template <int S>
__global__ void __launch_bounds__(256) k_refill(StepArgs A, const int8_t *type_prev_v, int *count) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    int did = 0;
    if (c < (int)A.D.n) {
        int k, j, i;
        cell_of(A.D, c, k, j, i);
        did = refill_cell<S>(A, type_prev_v, c, k, j, i, type_prev_v[c], A.fs_type[c]);
    }
    const int s = __reduce_add_sync(0xffffffffu, did);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(count, s);
}

// VOF path in two passes: the cells that turned wet (type_prev gas, type
// not gas) are listed (one warp-aggregated atomic per warp) and their coarse
// blocks marked for the coalescence repair (vof_mark_near), then the refill
// runs over the list only.
__global__ void __launch_bounds__(256) k_refill_vof_mark(StepArgs A, VofArgs V, const int8_t *type_prev, int *list,
                                                           int *lcount) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool cand = false;
    if (c < (int)A.D.n) {
        cand = type_prev[c] == LBM_FS_GAS && A.fs_type[c] != LBM_FS_GAS;
        if (cand) {
            int k, j, i;
            cell_of(A.D, c, k, j, i);
            vof_mark_near(V, k, j, i);
        }
    }
    const unsigned lanes = __ballot_sync(0xffffffffu, cand);
    if (lanes) {
        const int lane = threadIdx.x & 31, lead = __ffs(lanes) - 1;
        int base = 0;
        if (lane == lead) base = atomicAdd(lcount, __popc(lanes));
        base = __shfl_sync(0xffffffffu, base, lead);
        if (cand) list[base + __popc(lanes & ((1u << lane) - 1u))] = c;
    }
}
template <int S>
__global__ void __launch_bounds__(256) k_refill_vof_list(StepArgs A, const int8_t *type_prev, const int *list,
                                                          const int *lcount, int *count) {
    const int nl = *lcount;
    int did = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nl; e += gridDim.x * blockDim.x) {
        const int c = list[e];
        int k, j, i;
        cell_of(A.D, c, k, j, i);
        did += refill_cell<S>(A, type_prev, c, k, j, i, type_prev[c], A.fs_type[c]);
    }
    const int s = __reduce_add_sync(0xffffffffu, did);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(count, s);
}

// Height path: one thread per column.  A cell is refilled only if it was gas
// under the height before advection and is not gas under the new one, which
// needs k dx within a cell of the two heights: the planes from two below the
// lower height to two above the higher one are tested (every plane if a
// height is not finite); every other plane is liquid or gas under both.
template <int S>
__global__ void __launch_bounds__(256) k_refill_height(StepArgs A, int *count) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    int did = 0;
    const Dom &D = A.D;
    if (a < (int)D.a) {
        const int j = a / D.nx, i = a - j * D.nx;
        const float hl = A.fs_h_last[a], hn = A.fs_h[a];
        int k0 = 0, k1 = D.nz - 1;
        if (hl == hl && hn == hn) {
            const float lo = fminf(fmaxf(fminf(hl, hn) / A.P.dx, -4.0f), (float)D.nz + 4.0f);
            const float hi = fminf(fmaxf(fmaxf(hl, hn) / A.P.dx, -4.0f), (float)D.nz + 4.0f);
            k0 = max(0, (int)floorf(lo) - 2);
            k1 = min(D.nz - 1, (int)floorf(hi) + 2);
        }
        for (int k = k0; k <= k1; ++k) {
            int tp, tn;
            float fl;
            classify_height(A.P, hl, k, true, tp, fl);
            classify_height(A.P, hn, k, true, tn, fl);
            if (tp == LBM_FS_GAS && tn != LBM_FS_GAS) did += refill_cell<S>(A, nullptr, D.cell(k, j, i), k, j, i, tp, tn);
        }
    }
    const int s = __reduce_add_sync(0xffffffffu, did);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(count, s);
}

// free-surface fields of the height path after a call: fill and type from
// the new height, type_prev from the height before advection
__global__ void k_height_types(StepArgs A, float *fill, int8_t *type, int8_t *type_prev) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)A.D.n) return;
    int k, j, i;
    cell_of(A.D, c, k, j, i);
    bool open = cell_open(A.P, A.slot, A.D, A.bed_s, k, j, i);
    int tp, tn;
    float fp, fn;
    classify_height(A.P, A.fs_h_last[A.D.col(j, i)], k, open, tp, fp);
    classify_height(A.P, A.fs_h[A.D.col(j, i)], k, open, tn, fn);
    fill[c] = fn;
    type[c] = (int8_t)tn;
    type_prev[c] = (int8_t)tp;
}

// ======================================================== initialisation
// init_constants, CODEX.py:1022-1080
__global__ void k_init_constants(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = I.D;
    const lbm_params &P = I.P;
    if (c < (int)D.n) {
        I.rho[c] = P.rho0; I.ux[c] = 0.0f; I.uy[c] = 0.0f; I.uz[c] = 0.0f;
        I.omega[c] = P.omega0;
        I.fs_fill[c] = 1.0f;
        I.fs_type[c] = LBM_FS_LIQUID;
        I.fs_type_prev[c] = LBM_FS_LIQUID;
        I.fs_mass[c] = P.rho0;
        I.fs_mass_excess[c] = 0.0f;
        I.fs_excess_dir[c] = 0;
    }
    if (c < (int)D.a) {
        int i = c % D.nx;
        float bh = P.bed_offset_m;
        if (P.bed_profile == LBM_BED_PIECEWISE) bh = I.piecewise[i];
        I.water_h[c] = bh;
        I.water_h_last[c] = bh;
        I.u_wave[c] = 0.0f; I.v_wave[c] = 0.0f; I.w_wave[c] = 0.0f;
        I.fs_h[c] = P.fs_base_m;
        I.fs_h_last[c] = P.fs_base_m;
        I.fs_flux_x[c] = 0.0f;
        I.fs_flux_y[c] = 0.0f;
    }
}

// initialize_free_surface_height, CODEX.py:1197-1207
__global__ void k_fs_height_init(InitArgs I) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)I.D.a) return;
    const lbm_params &P = I.P;
    int i = a % I.D.nx;
    float x = ((float)i + 0.5f) * P.dx;
    float h = P.fs_base_m;
    if (P.fs_initial == LBM_FSINIT_SOLITARY || P.fs_mode == LBM_FS_PRESCRIBED_SOLITARY) h = solitary_h(P, I.D, x, 0.0f);
    else if (P.fs_initial == LBM_FSINIT_GAUSSIAN) h = gaussian_h(P, I.D, x);
    I.fs_h[a] = h;
    I.fs_h_last[a] = h;
}

// classify_free_surface_cells, CODEX.py:1210-1235 (stored form)
__global__ void k_classify_store(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    int8_t old = I.fs_type[c];
    float fl = 1.0f;
    int ct = LBM_FS_LIQUID;
    if (I.P.fs_mode != LBM_FS_NONE) {
        bool open = cell_open(I.P, I.slot, I.D, I.bed, k, j, i);
        classify_height(I.P, I.fs_h[I.D.col(j, i)], k, open, ct, fl);
    }
    I.fs_fill[c] = fl;
    I.fs_type_prev[c] = old;
    I.fs_type[c] = (int8_t)ct;
}

__device__ __forceinline__ float overlap(float cmin, float cmax, float bmin, float bmax) {
    float lo = cmin;
    if (bmin > lo) lo = bmin;
    float hi = cmax;
    if (bmax < hi) hi = bmax;
    float ov = hi - lo;
    if (ov < 0.0f) ov = 0.0f;
    return ov / (cmax - cmin);
}
// apply_vof_initial_disconnected_shape, CODEX.py:1253-1286
__global__ void k_vof_block(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    const lbm_params &P = I.P;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    if (!cell_open(P, I.slot, I.D, I.bed, k, j, i)) return;
    float dx = P.dx;
    float x0 = (float)i * dx, x1 = x0 + dx, y0 = (float)j * dx, y1 = y0 + dx, z0 = (float)k * dx, z1 = z0 + dx;
    float fx = overlap(x0, x1, P.vof_block_xmin, P.vof_block_xmax);
    float fy = overlap(y0, y1, P.vof_block_ymin, P.vof_block_ymax);
    float fz = overlap(z0, z1, P.vof_block_zmin, P.vof_block_zmax);
    float bf = fx * fy * fz;
    if (bf > 1e-4f) {
        int8_t old = I.fs_type[c];
        float fl = I.fs_fill[c];
        if (bf > fl) fl = bf;
        int ct = LBM_FS_INTERFACE;
        if (fl >= (float)(1.0 - 1e-4)) { fl = 1.0f; ct = LBM_FS_LIQUID; }
        I.fs_fill[c] = fl;
        I.fs_type_prev[c] = old;
        I.fs_type[c] = (int8_t)ct;
    }
}

// log-law inlet profile of init_fields, CODEX.py:2718-2742 (sequential)
__global__ void k_profile(InitArgs I) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const lbm_params &P = I.P;
    const int nz = I.D.nz;
    float B = 5.0f;
    float u_tau = P.u_tau_init;
    float nu_lbm = P.nu_lbm_init;
    for (int k = 0; k < nz; ++k) {
        float y = (float)k;
        float yp = y * u_tau / nu_lbm;
        if (yp <= 1.0f) yp = 1.0f;
        I.u_inlet_profile[k] = P.inv_kappa * lbm_logf(yp) + B;
    }
    float top = I.u_inlet_profile[nz - 1];
    if (top == 0.0f) top = 1.0f;
    for (int k = 0; k < nz; ++k) I.u_inlet_profile[k] = I.u_inlet_profile[k] / top * P.u_top_lb;
}

// velocity and equilibrium populations of init_fields, CODEX.py:2744-2825
template <int S>
__global__ void k_init_fields(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    const lbm_params &P = I.P;
    const Dom &D = I.D;
    int k, j, i;
    cell_of(D, c, k, j, i);
    GeoLinks L;
    Geo g = geo_cell(P, I.slot, D, I.bed, k, j, i, L);
    bool open = (g.lo & 1u) != 0u;
    const bool water = P.fs_mode != LBM_FS_NONE;
    float r = I.rho[c], vx, vy, vz;
    if (P.init_velocity_mode == LBM_INITVEL_UNIFORM) {
        float amp = P.init_noise_amp;
        vx = P.init_u0x + I.noise[c] * amp;
        vy = P.init_u0y + I.noise[D.n + c] * amp;
        vz = P.init_u0z + I.noise[2 * D.n + c] * amp;
    } else {
        float kick = I.noise[c];
        vx = I.u_inlet_profile[k] * (1.0f + kick * P.ti_kick);
        vy = 0.0f;
        vz = 0.0f;
    }
    int type = water ? I.fs_type[c] : LBM_FS_LIQUID;
    if (water) {
        if (type == LBM_FS_GAS) {
            r = P.rho0; vx = 0.0f; vy = 0.0f; vz = 0.0f;
        } else {
            r = I.rho_initial[c];
            vx = P.u_current_lb;
            if (P.fs_initial == LBM_FSINIT_SOLITARY && P.solitary_velocity_mode != LBM_SOLVEL_NONE) {
                float eta_fs = I.fs_h[D.col(j, i)] - P.fs_base_m;
                if (eta_fs < 0.0f) eta_fs = 0.0f;
                float hd = P.fs_depth_m;
                float usol = P.solitary_direction * P.solitary_celerity * eta_fs / (hd + eta_fs);
                vx += usol / P.vel_scale;
                if (P.solitary_velocity_mode == LBM_SOLVEL_SHALLOW_DIVFREE) {
                    float xc = ((float)i + 0.5f) * P.dx;
                    float Lxs = (float)D.nx * P.dx;
                    float xrel = xc - P.solitary_x0_m;
                    if (!P.x_solid) {
                        if (xrel > 0.5f * Lxs) xrel -= Lxs;
                        if (xrel < -0.5f * Lxs) xrel += Lxs;
                    }
                    float arg = P.solitary_kappa_inv * xrel;
                    float ep = lbm_expf(arg), em = lbm_expf(-arg);
                    float den = ep + em;
                    float sech = 2.0f / den;
                    float th = (ep - em) / den;
                    float eta_x = -2.0f * P.solitary_amp_m * P.solitary_kappa_inv * sech * sech * th;
                    float dudx = P.solitary_direction * P.solitary_celerity * hd * eta_x / ((hd + eta_fs) * (hd + eta_fs));
                    float zc = ((float)k + 0.5f) * P.dx;
                    float zrel = zc - I.bed.h[D.col(j, i)];
                    if (zrel < 0.0f) zrel = 0.0f;
                    vz += (-zrel * dudx) / P.vel_scale;
                }
            }
        }
    }
    if (!open) {
        vx = 0.0f; vy = 0.0f; vz = 0.0f;
        r = P.rho0;
        if (L.wt[0] == LBM_WALL_BED) {
            int a = D.col(j, i);
            vx = I.bed.uw[a]; vy = I.bed.vw[a]; vz = I.bed.ww[a];
        }
    }
    I.rho[c] = r; I.ux[c] = vx; I.uy[c] = vy; I.uz[c] = vz;
    float ez = vz;
    if (water && open && type != LBM_FS_GAS) ez += 0.5f * g_local(P, gbf_of(P, k, open, type));
    float u2 = usq(vx, vy, ez);
    typename Store<S>::T *dst = (typename Store<S>::T *)I.f_cur;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float v = 0.0f;
        switch (q) {
#define FQ(Q) case Q: v = feq<Q>(r, vx, vy, ez, u2); break;
            FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14) FQ(15)
            FQ(16) FQ(17) FQ(18)
#undef FQ
        }
        Store<S>::st(dst, (size_t)q * D.n + c, v, q, P.rho0);
    }
}

// initialize_free_surface_boundary_populations, CODEX.py:2828-2875:
// f_other = f_cur, plus the atmospheric projection when enabled
template <int S>
__global__ void k_fs_boundary_pop(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    const lbm_params &P = I.P;
    const Dom &D = I.D;
    typedef typename Store<S>::T ST;
    const ST *fo = (const ST *)I.f_cur;
    ST *fn = (ST *)I.f_other;
    float f[19], out[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        f[q] = Store<S>::ld_rw(fo, (size_t)q * D.n + c, q, P.rho0);
        out[q] = f[q];
    }
    if (P.fs_mode != LBM_FS_NONE && P.init_fs_populations) {
        int k, j, i;
        cell_of(D, c, k, j, i);
        bool open = cell_open(P, I.slot, D, I.bed, k, j, i);
        int type = I.fs_type[c];
        if (open && type != LBM_FS_GAS) {
            float vx = I.ux[c], vy = I.uy[c], vz = I.uz[c];
            float u2 = usq(vx, vy, vz);
            float gbf = gbf_of(P, k, open, type);
            float hcol = I.fs_h[D.col(j, i)];
#pragma unroll
            for (int q = 1; q < 19; ++q) {
                int sir = i - cxq(q);
                int si = sir;
                bool sf = true;
                if (!P.x_solid) si = pymod(sir + D.nx, D.nx);
                else if (sir < 0) { si = 0; sf = false; }
                else if (sir >= D.nx) { si = D.nx - 1; sf = false; }
                int sj = pymod(j - cyq(q) + D.ny, D.ny);
                int sk = k - czq(q);
                bool src_gas = false;
                if (!sf) src_gas = false;
                else if (sk >= D.nz) src_gas = true;
                else if (sk >= 0) {
                    int s = D.cell(sk, sj, si);
                    if (I.fs_type[s] == LBM_FS_GAS && cell_open(P, I.slot, D, I.bed, sk, sj, si)) src_gas = true;
                }
                if (src_gas) {
                    float rfs = P.rho0;
                    if (P.use_hydrostatic_balanced_pressure || P.fs_boundary == LBM_FSB_HYDROSTATIC)
                        rfs = fs_density_link(P, hcol, k, czq(q), gbf);
                    switch (q) {
#define FQ(Q) case Q: out[q] = feq<Q>(rfs, vx, vy, vz, u2) + feq<oppq(Q)>(rfs, vx, vy, vz, u2) - f[oppq(Q)]; break;
                        FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                        FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                    }
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) Store<S>::st(fn, (size_t)q * D.n + c, out[q], q, P.rho0);
}

// initialize_vof_mass_from_fill, CODEX.py:1289-1302
__global__ void k_vof_mass_init(InitArgs I) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    bool open = cell_open(I.P, I.slot, I.D, I.bed, k, j, i);
    if (open && I.fs_type[c] != LBM_FS_GAS) {
        I.fs_mass[c] = I.fs_fill[c] * I.rho[c];
    } else {
        I.fs_mass[c] = 0.0f;
        I.fs_fill[c] = 0.0f;
        I.fs_type[c] = LBM_FS_GAS;
    }
    I.fs_type_prev[c] = I.fs_type[c];
    I.fs_mass_excess[c] = 0.0f;
    I.fs_excess_dir[c] = 0;
}

// ------------------------------------------------------------------ export
__global__ void k_export(InitArgs I, ExportArgs E) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)I.D.n) return;
    const lbm_params &P = I.P;
    const Dom &D = I.D;
    int k, j, i;
    cell_of(D, c, k, j, i);
    GeoLinks L;
    Geo g = geo_cell(P, I.slot, D, I.bed, k, j, i, L, false);
    bool open = (g.lo & 1u) != 0u;
    if (E.phi) E.phi[c] = phi_cell(P, D, I.bed.h, k, j, i);
    if (E.obstacle) E.obstacle[c] = open ? 0 : 1;
    if (E.near_obstacle) E.near_obstacle[c] = g.near ? 1 : 0;
    for (int q = 0; q < 19; ++q) {
        if (E.lattice_open) E.lattice_open[(size_t)q * D.n + c] = (int8_t)((g.lo >> q) & 1u);
        if (E.lattice_open_frac) E.lattice_open_frac[(size_t)q * D.n + c] = L.lf[q];
        if (E.lattice_wall_type) E.lattice_wall_type[(size_t)q * D.n + c] = (int8_t)L.wt[q];
    }
    // update_pressure_reference_fields ran at the start of the last step
    // (types of that moment = fs_type_prev now) or, before any step, at init
    int tp = E.types_are_prev ? I.fs_type_prev[c] : I.fs_type[c];
    if (E.prh) E.prh[c] = prh_of(P, k, open, tp);
    if (E.gbf) E.gbf[c] = gbf_of(P, k, open, tp);
}

// ---------------------------------------------------------------- launchers
__global__ void k_clock_set(long long *clock, long long value) { *clock = value; }

void launch_clock_set(long long *clock, long long value, cudaStream_t st) {
    k_clock_set<<<1, 1, 0, st>>>(clock, value); LAUNCHED(1);
}

void launch_bed(const lbm_params &P, const Dom &D, const float *h_prev, float *h, float *hmax, float *uw, float *vw,
                float *ww, const float *piecewise, float t, cudaStream_t st, const long long *clock, long long off) {
    k_bed<<<blocks_for(D.a, 256), 256, 0, st>>>(P, D, h_prev, h, uw, vw, ww, piecewise, t, clock, off); LAUNCHED(1);
    k_hmax<<<blocks_for(D.a, 256), 256, 0, st>>>(D, h, hmax); LAUNCHED(1);
}
void launch_colgeo(const lbm_params &P, const Dom &D, const BedView &B, float *cg, cudaStream_t st) {
    k_colgeo<<<blocks_for(D.a, 128), 128, 0, st>>>(P, D, B, cg); LAUNCHED(1);
}
void launch_hmax(const Dom &D, const float *h, float *hmax, cudaStream_t st) {
    k_hmax<<<blocks_for(D.a, 256), 256, 0, st>>>(D, h, hmax); LAUNCHED(1);
}

// the pipelined interior kernel takes more than 48 KB of shared memory:
// raise the per-kernel limit once per device
static bool pipe_smem_ready() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        ok[dev] = cudaFuncSetAttribute(k_tile_pipe<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       PIPE_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       PIPE_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       PIPE_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       PIPE_SMEM_BYTES) == cudaSuccess;
    }
    return ok[dev];
}
template <int S>
static bool pipe16_smem_ready() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        ok[dev] = cudaFuncSetAttribute(k_tile_pipe16<S, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       P16_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe16<S, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       P16_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe16<S, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       P16_SMEM_BYTES) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_pipe16<S, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       P16_SMEM_BYTES) == cudaSuccess;
    }
    return ok[dev];
}

bool launch_tile_tma(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F32: return launch_tile_tma_t<LBM_STORE_F32, ArExact>(A, m24, m20, st);
        case LBM_STORE_F16S: return launch_tile_tma_t<LBM_STORE_F16S, ArExact>(A, m24, m20, st);
        case LBM_STORE_BF16S: return launch_tile_tma_t<LBM_STORE_BF16S, ArExact>(A, m24, m20, st);
        default: return false;
    }
}

template <int S>
static void launch_step_kernel_s(int which, const StepArgs &A, cudaStream_t st) {
    dim3 g = grid3(A);
    const int ni = A.zi1 - A.zi0 + 1;
    const bool tile_kernel = which == KER_TILE_CANON || which == KER_TILE_FUSED || which == KER_STREAM_INTERIOR;
    if (!tile_kernel && g.z == 0) return;
    if (tile_kernel && (ni <= 0 || A.chunk <= 0)) return;
    const unsigned tz = tile_kernel ? (unsigned)((ni + A.chunk - 1) / A.chunk) : 0u;
    dim3 gt(A.D.nx / LBM_TILE, A.D.ny / LBM_TILE, tz);
    dim3 gs(A.D.nx / LBM_TILE, A.D.ny / LBM_TILE, tile_kernel ? (unsigned)ni : 0u);
    const bool les = A.P.use_les != 0;
    // the column cache is set on both bed views or on neither
    const bool cg = A.bed_s.cg != nullptr && A.bed_c.cg != nullptr;
    // pipelined interior kernel: FP32 populations, 32-bit population indices
    const bool pipe = tile_kernel && S == LBM_STORE_F32 && !(A.flags & F_TILE_CLASSIC) &&
                      19.0 * (double)A.D.n < 2147483647.0 && pipe_smem_ready();
    // pipelined 16-bit interior kernel: staged pairs need an even nx (tiles of 16) and a 32-bit cell count
    bool pipe16 = false;
    if constexpr (S != LBM_STORE_F32)
        pipe16 = tile_kernel && !(A.flags & F_TILE_CLASSIC) && (double)A.D.n < 2147483647.0 &&
                 pipe16_smem_ready<S>();
    switch (which) {
        case KER_PREPASS_CANON:
            if (cg) k_prepass<S, 0, true><<<g, kBlock3, 0, st>>>(A);
            else k_prepass<S, 0, false><<<g, kBlock3, 0, st>>>(A);
            LAUNCHED(1);
            break;
        case KER_PREPASS_FUSED:
            if (cg) k_prepass<S, 1, true><<<g, kBlock3, 0, st>>>(A);
            else k_prepass<S, 1, false><<<g, kBlock3, 0, st>>>(A);
            LAUNCHED(1);
            break;
        case KER_COLLIDE_CANON:
            if (cg) k_collide<S, 0, true><<<g, kBlock3, 0, st>>>(A);
            else k_collide<S, 0, false><<<g, kBlock3, 0, st>>>(A);
            LAUNCHED(1);
            break;
        case KER_COLLIDE_FUSED:
            if (cg) k_collide<S, 1, true><<<g, kBlock3, 0, st>>>(A);
            else k_collide<S, 1, false><<<g, kBlock3, 0, st>>>(A);
            LAUNCHED(1);
            break;
        case KER_STREAM:
            if (cg) k_stream<S, true><<<g, kBlock3, 0, st>>>(A);
            else k_stream<S, false><<<g, kBlock3, 0, st>>>(A);
            LAUNCHED(1);
            break;


        case KER_TILE_CANON:
            if constexpr (S != LBM_STORE_F32) {
                if (pipe16) {
                    if (les) k_tile_pipe16<S, 0, true><<<gt, 256, P16_SMEM_BYTES, st>>>(A);
                    else k_tile_pipe16<S, 0, false><<<gt, 256, P16_SMEM_BYTES, st>>>(A);
                    LAUNCHED(1);
                    break;
                }
            }
            if (pipe) {
                if (les) k_tile_pipe<0, true><<<gt, 256, PIPE_SMEM_BYTES, st>>>(A);
                else k_tile_pipe<0, false><<<gt, 256, PIPE_SMEM_BYTES, st>>>(A);
            } else {
                if (les) k_tile<S, 0, true><<<gt, 256, 0, st>>>(A);
                else k_tile<S, 0, false><<<gt, 256, 0, st>>>(A);
            }
            LAUNCHED(1);
            break;
        case KER_TILE_FUSED:
            if constexpr (S != LBM_STORE_F32) {
                if (pipe16) {
                    if (les) k_tile_pipe16<S, 1, true><<<gt, 256, P16_SMEM_BYTES, st>>>(A);
                    else k_tile_pipe16<S, 1, false><<<gt, 256, P16_SMEM_BYTES, st>>>(A);
                    LAUNCHED(1);
                    break;
                }
            }
            if (pipe) {
                if (les) k_tile_pipe<1, true><<<gt, 256, PIPE_SMEM_BYTES, st>>>(A);
                else k_tile_pipe<1, false><<<gt, 256, PIPE_SMEM_BYTES, st>>>(A);
            } else {
                if (les) k_tile<S, 1, true><<<gt, 256, 0, st>>>(A);
                else k_tile<S, 1, false><<<gt, 256, 0, st>>>(A);
            }
            LAUNCHED(1);
            break;
        case KER_STREAM_INTERIOR: { k_stream_interior<S><<<gs, 256, 0, st>>>(A); LAUNCHED(1); } break;
        default: break;
    }
}
void launch_step_kernel(int which, const StepArgs &A, cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: launch_step_kernel_s<LBM_STORE_F16S>(which, A, st); break;
        case LBM_STORE_BF16S: launch_step_kernel_s<LBM_STORE_BF16S>(which, A, st); break;
        default: launch_step_kernel_s<LBM_STORE_F32>(which, A, st); break;
    }
}
template <int S>
static void launch_water_collide_s(const StepArgs &A, int *list, int *count, cudaStream_t st) {
    const dim3 g = grid3(A);
    if (g.z == 0) return;
    cudaMemsetAsync(count, 0, sizeof(int), st);
    if (A.P.collision == LBM_COLLIDE_KBC) k_collide_water<S, LBM_COLLIDE_KBC><<<g, kBlock3, 0, st>>>(A, list, count);
    else k_collide_water<S, LBM_COLLIDE_REGULARIZED><<<g, kBlock3, 0, st>>>(A, list, count);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_collide_list<S><<<(unsigned)(sms * 2), 256, 0, st>>>(A, list, count);
    LAUNCHED(2);
}
void launch_water_collide(const StepArgs &A, int *list, int *count, cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: launch_water_collide_s<LBM_STORE_F16S>(A, list, count, st); break;
        case LBM_STORE_BF16S: launch_water_collide_s<LBM_STORE_BF16S>(A, list, count, st); break;
        default: launch_water_collide_s<LBM_STORE_F32>(A, list, count, st); break;
    }
}
template <int S>
static void launch_water_stream_s(const StepArgs &A, int *list, int *count, cudaStream_t st) {
    const dim3 g = grid3(A);
    if (g.z == 0) return;
    cudaMemsetAsync(count, 0, sizeof(int), st);
    k_stream_water<S><<<g, kBlock3, 0, st>>>(A, list, count);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_stream_list<S><<<(unsigned)(sms * 2), 256, 0, st>>>(A, list, count);
    LAUNCHED(2);
}
void launch_water_stream(const StepArgs &A, int *list, int *count, cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: launch_water_stream_s<LBM_STORE_F16S>(A, list, count, st); break;
        case LBM_STORE_BF16S: launch_water_stream_s<LBM_STORE_BF16S>(A, list, count, st); break;
        default: launch_water_stream_s<LBM_STORE_F32>(A, list, count, st); break;
    }
}
void launch_column_flux(const StepArgs &A, float *qx, float *qy, cudaStream_t st) {
    const unsigned g = (unsigned)(((A.D.nx + 31) / 32) * A.D.ny);
    k_column_flux<<<g, dim3(32, 8, 1), 0, st>>>(A, qx, qy); LAUNCHED(1);
}
void launch_advect(const lbm_params &P, const Dom &D, const float *bed_h, const float *qx, const float *qy,
                   const float *h_in, float *h_out, float *h_last, float t, cudaStream_t st) {
    k_advect<<<blocks_for(D.a, 256), 256, 0, st>>>(P, D, bed_h, qx, qy, h_in, h_out, h_last, t); LAUNCHED(1);
}
void launch_refill(const StepArgs &A, const int8_t *type_prev, int *count, cudaStream_t st) {
    if (!(A.flags & F_VOF_STATE)) {
        const unsigned gh = blocks_for(A.D.a, 256);
        switch (A.P.pop_storage) {
            case LBM_STORE_F16S: k_refill_height<LBM_STORE_F16S><<<gh, 256, 0, st>>>(A, count); break;
            case LBM_STORE_BF16S: k_refill_height<LBM_STORE_BF16S><<<gh, 256, 0, st>>>(A, count); break;
            default: k_refill_height<LBM_STORE_F32><<<gh, 256, 0, st>>>(A, count); break;
        }
        LAUNCHED(1);
        return;
    }
    unsigned g = blocks_for(A.D.n, 256);
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: { k_refill<LBM_STORE_F16S><<<g, 256, 0, st>>>(A, type_prev, count); LAUNCHED(1); } break;
        case LBM_STORE_BF16S: { k_refill<LBM_STORE_BF16S><<<g, 256, 0, st>>>(A, type_prev, count); LAUNCHED(1); } break;
        default: k_refill<LBM_STORE_F32><<<g, 256, 0, st>>>(A, type_prev, count); LAUNCHED(1); break;
    }
}
template <int S>
static void launch_refill_vof_s(const StepArgs &A, const VofArgs &V, const int8_t *type_prev, int *list, int *count,
                                cudaStream_t st) {
    int *lcount = list + A.D.n;
    cudaMemsetAsync(lcount, 0, sizeof(int), st);
    cudaMemsetAsync(V.near, 0, vof_near_bytes(V.D), st);
    k_refill_vof_mark<<<blocks_for(A.D.n, 256), 256, 0, st>>>(A, V, type_prev, list, lcount);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_refill_vof_list<S><<<(unsigned)sms, 256, 0, st>>>(A, type_prev, list, lcount, count);
    LAUNCHED(2);
}
void launch_refill_vof(const StepArgs &A, const VofArgs &V, const int8_t *type_prev, int *list, int *count,
                       cudaStream_t st) {
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: launch_refill_vof_s<LBM_STORE_F16S>(A, V, type_prev, list, count, st); break;
        case LBM_STORE_BF16S: launch_refill_vof_s<LBM_STORE_BF16S>(A, V, type_prev, list, count, st); break;
        default: launch_refill_vof_s<LBM_STORE_F32>(A, V, type_prev, list, count, st); break;
    }
}
void launch_height_types(const StepArgs &A, float *fill, int8_t *type, int8_t *type_prev, cudaStream_t st) {
    k_height_types<<<blocks_for(A.D.n, 256), 256, 0, st>>>(A, fill, type, type_prev); LAUNCHED(1);
}

void launch_init_constants(const InitArgs &I, cudaStream_t st) {
    size_t n = I.D.n > I.D.a ? I.D.n : I.D.a;
    k_init_constants<<<blocks_for(n, 256), 256, 0, st>>>(I); LAUNCHED(1);
}
void launch_fs_height_init(const InitArgs &I, cudaStream_t st) {
    k_fs_height_init<<<blocks_for(I.D.a, 256), 256, 0, st>>>(I); LAUNCHED(1);
}
void launch_classify_store(const InitArgs &I, cudaStream_t st) {
    k_classify_store<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I); LAUNCHED(1);
}
void launch_vof_block(const InitArgs &I, cudaStream_t st) {
    k_vof_block<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I); LAUNCHED(1);
}
void launch_init_fields(const InitArgs &I, cudaStream_t st) {
    k_profile<<<1, 1, 0, st>>>(I); LAUNCHED(1);
    unsigned g = blocks_for(I.D.n, 256);
    switch (I.P.pop_storage) {
        case LBM_STORE_F16S:
            k_init_fields<LBM_STORE_F16S><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            k_fs_boundary_pop<LBM_STORE_F16S><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            break;
        case LBM_STORE_BF16S:
            k_init_fields<LBM_STORE_BF16S><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            k_fs_boundary_pop<LBM_STORE_BF16S><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            break;
        default:
            k_init_fields<LBM_STORE_F32><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            k_fs_boundary_pop<LBM_STORE_F32><<<g, 256, 0, st>>>(I); LAUNCHED(1);
            break;
    }
}
void launch_vof_mass_init(const InitArgs &I, cudaStream_t st) {
    k_vof_mass_init<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I); LAUNCHED(1);
}
void launch_export(const InitArgs &I, const ExportArgs &E, cudaStream_t st) {
    k_export<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I, E); LAUNCHED(1);
}

}  // namespace lbm

// ------------------------------------------------------------ VOF launchers
namespace lbm {

static inline unsigned vblocks(const VofArgs &V) { return blocks_for(V.D.n, 256); }

void launch_vof_open(const VofArgs &V, const BedView &B, cudaStream_t st) {
    k_vof_open<<<vblocks(V), 256, 0, st>>>(V, B); LAUNCHED(1);
}

// FP64 tree over len values: returns the device address of the sum
static const double *tree_reduce(const double *in, long long len, double *ping, double *pong, cudaStream_t st) {
    const double *cur = in;
    double *bufs[2] = {ping, pong};
    int b = 0;
    while (len > 1) {
        const long long nb = (len + 255) / 256;
        k_tree_level<<<(unsigned)nb, 256, 0, st>>>(cur, len, bufs[b]); LAUNCHED(1);
        cur = bufs[b];
        b ^= 1;
        len = nb;
    }
    return cur;
}

static cudaError_t vof_snapshot(const VofArgs &V, const float *a, float *a0, const float *b, float *b0, bool types,
                                cudaStream_t st) {
    const size_t n = V.D.n;
    cudaError_t e = cudaSuccess;
    if (a && e == cudaSuccess) e = cudaMemcpyAsync(a0, a, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (b && e == cudaSuccess) e = cudaMemcpyAsync(b0, b, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (types && e == cudaSuccess) e = cudaMemcpyAsync(V.t0, V.type, n, cudaMemcpyDeviceToDevice, st);
    return e;
}

static cudaError_t vof_redistribute(const VofArgs &V, cudaStream_t st) {
    cudaError_t e = vof_snapshot(V, V.mass, V.m0, V.mass_excess, V.x0, false, st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(V.near, 0, vof_near_bytes(V.D), st)) != cudaSuccess) return e;
    k_vof_redist_donor<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
    k_vof_redist_recv<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
    return cudaGetLastError();
}
static void vof_finalize(const VofArgs &V, int *cnt, cudaStream_t st) {
    k_vof_finalize<<<vblocks(V), 256, 0, st>>>(V, cnt); LAUNCHED(1);
}
cudaError_t vof_interface_layer(const VofArgs &V, cudaStream_t st) {
    // type snapshot with the coarse marks of open gas cells, dilated by one
    // block into V.near, which the layer kernel tests before its 18 neighbours
    const size_t nb = vof_near_bytes(V.D);
    cudaError_t e = cudaMemsetAsync(V.near + nb, 0, nb, st);
    if (e != cudaSuccess) return e;
    k_vof_types_gas_mark<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
    k_vof_gas_dilate<<<blocks_for(nb, 256), 256, 0, st>>>(V); LAUNCHED(1);
    k_vof_interface_layer<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
    return cudaGetLastError();
}
void launch_vof_height(const VofArgs &V, cudaStream_t st) {
    k_vof_height<<<blocks_for(V.D.a, 128), 128, 0, st>>>(V); LAUNCHED(1);
}

// the VOF part of one step after the stream and its macro step
// (CODEX.py:3898-3917), up to the column height; refill and coalescence
// repair follow in the caller
cudaError_t vof_sequence(const VofArgs &V, bool collapse_due, double *tree, cudaStream_t st) {
    cudaError_t e;
    const size_t n = V.D.n;
    int *cnt = V.count;
    // counters of this step (the reference resets them in these kernels)
    if ((e = cudaMemsetAsync(cnt + CNT_VOF_EXCESS, 0, 5 * sizeof(int), st)) != cudaSuccess) return e;  // excess..cmp
    if ((e = cudaMemsetAsync(V.fcount, 0, 7 * sizeof(float), st)) != cudaSuccess) return e;
    switch (V.P.pop_storage) {
        case LBM_STORE_F16S: k_vof_exchange<LBM_STORE_F16S><<<vblocks(V), 256, 0, st>>>(V); break;
        case LBM_STORE_BF16S: k_vof_exchange<LBM_STORE_BF16S><<<vblocks(V), 256, 0, st>>>(V); break;
        default: k_vof_exchange<LBM_STORE_F32><<<vblocks(V), 256, 0, st>>>(V); break;
    }
    LAUNCHED(1);
    k_vof_apply<<<vblocks(V), 256, 0, st>>>(V, cnt + CNT_VOF_EXCESS); LAUNCHED(1);
    for (int r = 0; r < 3; ++r) {
        if ((e = vof_redistribute(V, st)) != cudaSuccess) return e;
        vof_finalize(V, cnt + CNT_VOF_EXCESS, st);
    }
    if ((e = vof_interface_layer(V, st)) != cudaSuccess) return e;
    // orphans: snapshots of mass, fill and type
    if ((e = vof_snapshot(V, V.mass, V.m0, V.fill, V.x0, true, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(V.near, 0, vof_near_bytes(V.D), st)) != cudaSuccess) return e;
    k_vof_orphan_donor<<<vblocks(V), 256, 0, st>>>(V, cnt + CNT_ORPHAN); LAUNCHED(1);
    k_vof_orphan_recv<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
    double *ping = tree, *pong = tree + (n / 256 + 2);
    if (V.P.vof_detached_advection) {
        k_vof_detached_donor<<<vblocks(V), 256, 0, st>>>(V, 0, cnt + CNT_DET); LAUNCHED(1);
        k_vof_detached_apply<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
        k_store_sum<<<1, 1, 0, st>>>(tree_reduce(V.dd, (long long)n, ping, pong, st), V.fcount + 5); LAUNCHED(1);
    }
    vof_finalize(V, cnt + CNT_VOF_EXCESS, st);
    if (V.P.vof_detached_advection && V.P.vof_detached_residual_fill_threshold > 0.0f) {
        k_vof_detached_donor<<<vblocks(V), 256, 0, st>>>(V, 1, cnt + CNT_CMP); LAUNCHED(1);
        k_vof_detached_apply<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
        k_store_sum<<<1, 1, 0, st>>>(tree_reduce(V.dd, (long long)n, ping, pong, st), V.fcount + 6); LAUNCHED(1);
    }
    vof_finalize(V, cnt + CNT_VOF_EXCESS, st);
    if ((e = vof_redistribute(V, st)) != cudaSuccess) return e;
    vof_finalize(V, cnt + CNT_VOF_EXCESS, st);
    if ((e = vof_interface_layer(V, st)) != cudaSuccess) return e;
    if (collapse_due) {
        // exterior marks: capped 6-connected flood from the top row
        if ((e = cudaMemsetAsync(cnt + CNT_SWEEPS, 0, sizeof(int), st)) != cudaSuccess) return e;
        k_vof_flood_seed<<<vblocks(V), 256, 0, st>>>(V); LAUNCHED(1);
        const int S = V.P.vof_collapse_flood_sweeps;
        const int batch = 16;
        for (int s0 = 0; s0 < S; s0 += batch) {
            const int s1 = s0 + batch < S ? s0 + batch : S;
            for (int s = s0; s < s1; ++s) {
                k_vof_flood_level<<<vblocks(V), 256, 0, st>>>(V, s, cnt + CNT_SWEEPS); LAUNCHED(1);
            }
            int reached = 0;
            if ((e = cudaMemcpyAsync(&reached, cnt + CNT_SWEEPS, sizeof(int), cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess)
                return e;
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
            if (reached < s1) break;   // a level of this batch added nothing: the flood is complete
        }
        // FP64 sums of trapped mass, trapped volume and exterior capacity
        const long long nb = (long long)((n + 255) / 256);
        double *lm = tree + 2 * (n / 256 + 2), *lv = tree + 3 * (n / 256 + 2), *lc = tree + 4 * (n / 256 + 2);
        double *tp = tree + 5 * (n / 256 + 2);
        k_vof_collapse_sums<<<(unsigned)nb, 256, 0, st>>>(V, lm, lv, lc); LAUNCHED(1);
        // reduce each partial array; results are copied to three fixed slots
        double *res = tp;   // tp[0..2]
        const double *rm = tree_reduce(lm, nb, ping, pong, st);
        if ((e = cudaMemcpyAsync(res + 0, rm, sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
        const double *rv = tree_reduce(lv, nb, ping, pong, st);
        if ((e = cudaMemcpyAsync(res + 1, rv, sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
        const double *rc = tree_reduce(lc, nb, ping, pong, st);
        if ((e = cudaMemcpyAsync(res + 2, rc, sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
        k_vof_collapse_decide<<<1, 1, 0, st>>>(res + 0, res + 1, res + 2, V.P.vof_collapse_max_volume_m3, V.fcount);
        LAUNCHED(1);
        k_vof_collapse_apply<<<vblocks(V), 256, 0, st>>>(V, cnt + CNT_COLLAPSE); LAUNCHED(1);
    }
    if ((e = vof_interface_layer(V, st)) != cudaSuccess) return e;
    launch_vof_height(V, st);
    return cudaGetLastError();
}

void launch_vof_coalesce(const VofArgs &V, cudaStream_t st) {
    switch (V.P.pop_storage) {
        case LBM_STORE_F16S: k_vof_coalesce<LBM_STORE_F16S><<<vblocks(V), 256, 0, st>>>(V, V.count + CNT_COALESCE); break;
        case LBM_STORE_BF16S: k_vof_coalesce<LBM_STORE_BF16S><<<vblocks(V), 256, 0, st>>>(V, V.count + CNT_COALESCE); break;
        default: k_vof_coalesce<LBM_STORE_F32><<<vblocks(V), 256, 0, st>>>(V, V.count + CNT_COALESCE); break;
    }
    LAUNCHED(1);
}
// ------------------------------------------------------ ensemble launchers
void launch_batch_bed(const BatchLaunch &L, long long m, cudaStream_t st) {
    const int par = (int)(m & 1);
    const unsigned g = blocks_for((size_t)L.ncols, 256);
    kb_bed<<<g, 256, 0, st>>>(L, m, par); LAUNCHED(1);
    kb_hmax<<<g, 256, 0, st>>>(L, par); LAUNCHED(1);
    kb_colgeo<<<blocks_for((size_t)L.ncols, 128), 128, 0, st>>>(L, par); LAUNCHED(1);
}

int batch_tile_blocks(int storage, bool les, int collision, int arith, bool tma) {
    if (arith == LBM_ARITH_FAST) return batch_tile_blocks_fast(storage, les, collision, tma);
    return batch_tile_blocks_any<ArExact>(storage, les, tma);
}

template <int S>
static void launch_batch_group_s(int which, const BatchGroup &G, cudaStream_t st) {
    if (!G.nmap) return;
    const dim3 b3(32, 8, 1);
    switch (which) {
        case KER_PREPASS_CANON: kb_general<S, 0, 0><<<G.nmap, b3, 0, st>>>(G); break;
        case KER_PREPASS_FUSED: kb_general<S, 1, 0><<<G.nmap, b3, 0, st>>>(G); break;
        case KER_COLLIDE_CANON: kb_general<S, 0, 1><<<G.nmap, b3, 0, st>>>(G); break;
        case KER_COLLIDE_FUSED: kb_general<S, 1, 1><<<G.nmap, b3, 0, st>>>(G); break;
        case KER_STREAM: kb_general<S, 0, 2><<<G.nmap, b3, 0, st>>>(G); break;
        case KER_STREAM_INTERIOR: kb_stream_interior<S><<<G.nmap, 256, 0, st>>>(G); break;
        default: return;
    }
    LAUNCHED(1);
}
void launch_batch_group(int which, int storage, const BatchGroup &G, bool les, int collision, int arith,
                        int tile_blocks, cudaStream_t st) {
    if (which == KER_TILE_CANON || which == KER_TILE_FUSED || which == KER_TILE_TMA) {
        if (arith == LBM_ARITH_FAST) launch_batch_tile_fast(which, storage, G, les, collision, tile_blocks, st);
        else launch_batch_tile_any<ArExact>(which, storage, G, les, tile_blocks, st);
        return;
    }
    switch (storage) {
        case LBM_STORE_F16S: launch_batch_group_s<LBM_STORE_F16S>(which, G, st); break;
        case LBM_STORE_BF16S: launch_batch_group_s<LBM_STORE_BF16S>(which, G, st); break;
        default: launch_batch_group_s<LBM_STORE_F32>(which, G, st); break;
    }
}

void launch_diagnostics(const DiagArgs &G, cudaStream_t st) {
    k_diag_cells<<<G.ncellp, DIAG_THREADS, 0, st>>>(G); LAUNCHED(1);
    if (G.fs) {
        k_diag_columns<<<blocks_for(G.D.nx, 128), 128, 0, st>>>(G); LAUNCHED(1);
    }
    k_diag_slice<<<blocks_for((size_t)G.D.nz * G.D.nx, 256), 256, 0, st>>>(G); LAUNCHED(1);
    k_diag_slice_sum<<<G.nslp, DIAG_SLICE_THREADS, 0, st>>>(G, 0); LAUNCHED(1);
    k_diag_slice_mean<<<1, 32, 0, st>>>(G); LAUNCHED(1);
    k_diag_slice_sum<<<G.nslp, DIAG_SLICE_THREADS, 0, st>>>(G, 1); LAUNCHED(1);
    k_diag_final<<<1, 32, 0, st>>>(G); LAUNCHED(1);
}

void launch_vof_exterior(const Dom &D, const int *dist, int32_t *out, cudaStream_t st) {
    k_vof_exterior<<<blocks_for(D.n, 256), 256, 0, st>>>((int)D.n, dist, out); LAUNCHED(1);
}

}  // namespace lbm

// ------------------------------------------- allocation-free link geometry
// lbm_link_geometry_noalloc: the link geometry that lbm_export_diagnostics
// writes (phi, obstacle, near_obstacle, lattice_open, lattice_open_frac,
// lattice_wall_type), for a bed height field the caller passes, without any
// context or allocation.  The bed heights at the nine link-endpoint (x, y)
// positions of each column are sampled once into a fixed device array, and
// the per-cell pass reads them from there (the bed-only path of the step
// kernels, same arithmetic as the per-link path of k_export).
namespace lbm {

#define LBM_MAX_DEVICES 64

// [9][columns]: bed height at endpoint e of each column, stride nx*ny.
// Every call overwrites the entries it reads, so nothing needs clearing.
static __device__ __align__(256) float g_noalloc_endpoints[9 * LBM_NOALLOC_MAX_COLUMNS];

__global__ void k_noalloc_endpoints(lbm_params P, Dom D, const float *__restrict__ bed_h, float *cache) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (int)D.a) return;
    const int j = a / D.nx, i = a - j * D.nx;
    const float dx = P.dx, hdx = 0.5f * dx;
    float xc = ((float)i + 0.5f) * dx, yc = ((float)j + 0.5f) * dx;
    int xi0[3], xi1[3], yj0[3], yj1[3];
    float xf[3], yf[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        bl_axis(xc + hdx * (float)(s - 1), dx, D.nx, xi0[s], xi1[s], xf[s]);
        bl_axis(yc + hdx * (float)(s - 1), dx, D.ny, yj0[s], yj1[s], yf[s]);
    }
#pragma unroll
    for (int xa = 0; xa < 3; ++xa)
#pragma unroll
        for (int yb = 0; yb < 3; ++yb)
            cache[(size_t)(CG_ETA + 3 * xa + yb) * D.a + a] =
                bl_sample(bed_h, D, xi0[xa], yj0[yb], xi1[xa], yj1[yb], xf[xa], yf[yb]);
}

__global__ void k_noalloc_links(lbm_params P, Dom D, const float *__restrict__ bed_h, const float *cache,
                                ExportArgs E) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)D.n) return;
    int k, j, i;
    cell_of(D, c, k, j, i);
    BedView B;
    B.h = bed_h;
    B.hmax = nullptr;
    B.uw = B.vw = B.ww = nullptr;
    B.cg = cache;
    GeoLinks L;
    Geo g = geo_cached(P, D, B, k, j, i, L);
    bool open = (g.lo & 1u) != 0u;
    if (E.phi) E.phi[c] = phi_cell(P, D, bed_h, k, j, i);
    if (E.obstacle) E.obstacle[c] = open ? 0 : 1;
    if (E.near_obstacle) E.near_obstacle[c] = g.near ? 1 : 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (E.lattice_open) E.lattice_open[(size_t)q * D.n + c] = (int8_t)((g.lo >> q) & 1u);
        if (E.lattice_open_frac) E.lattice_open_frac[(size_t)q * D.n + c] = L.lf[q];
        if (E.lattice_wall_type) E.lattice_wall_type[(size_t)q * D.n + c] = (int8_t)L.wt[q];
    }
}

// Device address of g_noalloc_endpoints on the current device.  In host
// code the array's name is only a host-side stand-in, so the address is
// looked up with the device current.  Outside stream capture it is looked
// up on every call (a device reset or another driver context loads the
// module again, at a new address) and remembered per device; while the
// stream is being captured the remembered address is used, since a lookup
// may have to load the module, which capture does not allow.
static std::mutex g_noalloc_mutex;
static float *g_noalloc_address[LBM_MAX_DEVICES] = {};

static cudaError_t noalloc_endpoints_address(cudaStream_t st, float **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= LBM_MAX_DEVICES) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_endpoints);
        if (e != cudaSuccess) return e;
        g_noalloc_address[dev] = (float *)p;
    } else if (!g_noalloc_address[dev]) {
        return cudaErrorStreamCaptureUnsupported;   // no call outside capture on this device yet
    }
    *out = g_noalloc_address[dev];
    return cudaSuccess;
}

static int noalloc_fail(char *err, size_t err_len, int code, const char *msg) {
    if (err && err_len) snprintf(err, err_len, "%s", msg);
    return code;
}

}  // namespace lbm

extern "C" int lbm_link_geometry_noalloc(const lbm_params *params, const float *bed_h, float *phi, int32_t *obstacle,
                                         int32_t *near_obstacle, int8_t *lattice_open, float *lattice_open_frac,
                                         int8_t *lattice_wall_type, void *stream, char *err, size_t err_len) {
    using namespace lbm;
    if (err && err_len) err[0] = '\0';
    if (!params || !bed_h)
        return noalloc_fail(err, err_len, LBM_ERR_BAD_ARG, "lbm_link_geometry_noalloc: params and bed_h are required");
    const lbm_params &P = *params;
    if (P.abi_version != LBM_ABI_VERSION || P.magic_end != LBM_PARAMS_MAGIC)
        return noalloc_fail(err, err_len, LBM_ERR_BAD_ARG,
                            "lbm_link_geometry_noalloc: lbm_params layout or ABI version mismatch");
    if (P.nx < 1 || P.ny < 1 || P.nz < 2)
        return noalloc_fail(err, err_len, LBM_ERR_BAD_ARG, "lbm_link_geometry_noalloc: grid must be nx, ny >= 1, nz >= 2");
    const size_t cols = (size_t)P.nx * (size_t)P.ny;
    if (cols > (size_t)LBM_NOALLOC_MAX_COLUMNS) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "lbm_link_geometry_noalloc: nx*ny = %zu columns exceeds the fixed maximum of %d; "
                 "use lbm_export_diagnostics on a context instead",
                 cols, (int)LBM_NOALLOC_MAX_COLUMNS);
        return noalloc_fail(err, err_len, LBM_ERR_BAD_ARG, msg);
    }
    if (cols * (size_t)P.nz > 0x7fffffffULL)
        return noalloc_fail(err, err_len, LBM_ERR_BAD_ARG, "lbm_link_geometry_noalloc: more than 2^31-1 cells");
    if (P.include_cube || P.use_phi_open_fraction || P.use_phi_open_flags || P.x_solid)
        return noalloc_fail(err, err_len, LBM_ERR_UNSUPPORTED,
                            "lbm_link_geometry_noalloc: only bed geometry with periodic x is supported "
                            "(no cube, no phi geometry, no solid x walls)");
    float *cache = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = noalloc_endpoints_address(st, &cache);
    if (e != cudaSuccess) {
        char msg[200];
        snprintf(msg, sizeof msg, "lbm_link_geometry_noalloc: device address of the fixed array: %s",
                 cudaGetErrorString(e));
        return noalloc_fail(err, err_len, LBM_ERR_CUDA, msg);
    }
    Dom D;
    D.nx = P.nx;
    D.ny = P.ny;
    D.nz = P.nz;
    D.a = cols;
    D.n = cols * (size_t)P.nz;
    ExportArgs E;
    memset(&E, 0, sizeof E);
    E.phi = phi;
    E.obstacle = obstacle;
    E.near_obstacle = near_obstacle;
    E.lattice_open = lattice_open;
    E.lattice_open_frac = lattice_open_frac;
    E.lattice_wall_type = lattice_wall_type;
    k_noalloc_endpoints<<<blocks_for(D.a, 128), 128, 0, st>>>(P, D, bed_h, cache); LAUNCHED(1);
    k_noalloc_links<<<blocks_for(D.n, 256), 256, 0, st>>>(P, D, bed_h, cache, E); LAUNCHED(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        char msg[200];
        snprintf(msg, sizeof msg, "lbm_link_geometry_noalloc: launch: %s", cudaGetErrorString(e));
        return noalloc_fail(err, err_len, LBM_ERR_CUDA, msg);
    }
    return LBM_OK;
}
