// lbm_kernels.cu - kernels of the D3Q19 step (air and height-function
// free-surface paths) and their launchers.
//
// Kernel map (reference kernel -> here):
//   update_wave_bed_and_velocities           k_bed + k_hmax (2-D)
//   compute_phi / build_lattice_open         recomputed per cell (lbm_geom.cuh)
//   update_bed_populations + macro_step +
//   compute_LES + collide_*                  k_collide (from the post-stream state)
//   stream + x walls + open BCs +
//   (next step) condition + macro + LES +
//   collide                                  k_fused (air path, one pass per step)
//   stream + x walls + open BCs (+ water
//   post-stream macro_step)                  k_stream
//   velocity stencil of compute_LES          k_prepass (u of every cell)
//   compute_free_surface_column_flux         k_column_flux
//   advect_free_surface_height               k_advect
//   refill_new_free_surface_cells            k_refill
#include <cuda_runtime.h>

#include "lbm_launch.h"
#include "lbm_step.cuh"

namespace lbm {

static __device__ __forceinline__ void cell_of(const Dom &D, size_t c, int &k, int &j, int &i) {
    k = (int)(c / D.a);
    size_t r = c - (size_t)k * D.a;
    j = (int)(r / D.nx);
    i = (int)(r - (size_t)j * D.nx);
}

// ------------------------------------------------------------- bed (2-D)
// update_wave_bed_and_velocities, CODEX.py:1082-1162, harmonics generalised
__global__ void k_bed(const __grid_constant__ lbm_params P, Dom D, const float *__restrict__ h_prev, float *h, float *uw, float *vw,
                      float *ww, const float *__restrict__ piecewise, float t) {
    size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (a >= D.a) return;
    int j = (int)(a / D.nx), i = (int)(a - (size_t)j * D.nx);
    (void)j;
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

// max of the bed over the 3x3 column neighbourhood (periodic), the support
// of every link-endpoint sample of the column
__global__ void k_hmax(Dom D, const float *__restrict__ h, float *hmax) {
    size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (a >= D.a) return;
    int j = (int)(a / D.nx), i = (int)(a - (size_t)j * D.nx);
    float m = -3.4e38f;
    for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
            int jj = (j + dj + D.ny) % D.ny, ii = (i + di + D.nx) % D.nx;
            m = fmaxf(m, h[D.col(jj, ii)]);
        }
    hmax[a] = m;
}

// ------------------------------------------------------- step kernels
template <int S>
__device__ __forceinline__ void load_cell(const StepArgs &A, size_t c, float f[19]) {
    const typename Store<S>::T *src = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = Store<S>::ld(src, (size_t)q * A.D.n + c, q, A.P.rho0);
}
template <int S>
__device__ __forceinline__ void store_cell(const StepArgs &A, size_t c, const float f[19]) {
    typename Store<S>::T *dst = (typename Store<S>::T *)A.fdst;
#pragma unroll
    for (int q = 0; q < 19; ++q) Store<S>::st(dst, (size_t)q * A.D.n + c, f[q], q, A.P.rho0);
}

// Front half shared by the pre-pass and the collide kernels: populations
// entering the collide step (IN = 0: the stored post-stream state; IN = 1:
// stream + BC of the previous step from its post-collision state), then the
// condition and macro stages on the collide step's geometry.
template <int S, int IN>
__device__ __forceinline__ void front(const StepArgs &A, size_t c, int k, int j, int i, float f[19], Geo &gc,
                                      GeoLinks &Lc, int &type, float &fill, float &gbf, float &r, float &vx, float &vy,
                                      float &vz) {
    if (IN == 0) {
        load_cell<S>(A, c, f);
    } else {
        GeoLinks Ls;
        Geo gs = geo_cell(A.P, A.D, A.bed_s, k, j, i, Ls);
        int cut = 0, fscut = 0, bridge = 0;
        stream_bc<S>(A, (const typename Store<S>::T *)A.fsrc, gs, Ls, k, j, i, c, f, cut, fscut, bridge);
    }
    gc = geo_cell(A.P, A.D, A.bed_c, k, j, i, Lc);
    const bool water = A.P.fs_mode != LBM_FS_NONE;
    type = LBM_FS_LIQUID;
    fill = 1.0f;
    gbf = 0.0f;
    bool open = (gc.lo & 1u) != 0u;
    if (water) {
        fs_state(A, c, k, j, open, type, fill);
        gbf = gbf_of(A.P, k, open, type);
    }
    condition(A.P, A.D, A.bed_c, gc, Lc, k, j, i, f);
    macro(A.P, A.D, f, k, water, type, gbf, r, vx, vy, vz);
}

template <int S, int IN>
__global__ void __launch_bounds__(256) k_prepass(const __grid_constant__ StepArgs A) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= A.D.n) return;
    int k, j, i;
    cell_of(A.D, c, k, j, i);
    float f[19], r, vx, vy, vz, fill, gbf;
    int type;
    Geo gc;
    GeoLinks Lc;
    front<S, IN>(A, c, k, j, i, f, gc, Lc, type, fill, gbf, r, vx, vy, vz);
    A.u_out[c] = vx;
    A.u_out[A.D.n + c] = vy;
    A.u_out[2 * A.D.n + c] = vz;
}

template <int S, int IN>
__global__ void __launch_bounds__(256) k_collide(const __grid_constant__ StepArgs A) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= A.D.n) return;
    int k, j, i;
    cell_of(A.D, c, k, j, i);
    float f[19], r, vx, vy, vz, fill, gbf;
    int type;
    Geo gc;
    GeoLinks Lc;
    front<S, IN>(A, c, k, j, i, f, gc, Lc, type, fill, gbf, r, vx, vy, vz);
    const lbm_params &P = A.P;
    const bool water = P.fs_mode != LBM_FS_NONE;
    const bool open = (gc.lo & 1u) != 0u;
    const bool gas = water && type == LBM_FS_GAS;
    if (A.flags & F_WRITE_MACRO) {
        A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
    }
    if (!(r == r) || fabsf(r) > 3.0e38f) atomicOr(A.status, 1u);
    float om;
    if (P.use_les) {
        bool active = open && !gas;
        if (active) {
            om = les_omega(A, k, j, i, c, vx, vy, vz);
            if ((A.flags & F_WRITE_ALL_OMEGA) || !gc.fast) A.omega[c] = om;
        } else {
            om = A.omega[c];
        }
    } else {
        om = P.omega0;
    }
    collide(A, c, k, !open, water, gas, gbf, r, vx, vy, vz, om, f);
    store_cell<S>(A, c, f);
}

template <int S>
__global__ void __launch_bounds__(256) k_stream(const __grid_constant__ StepArgs A) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int cut = 0, fscut = 0, bridge = 0;
    if (c < A.D.n) {
        int k, j, i;
        cell_of(A.D, c, k, j, i);
        GeoLinks Ls;
        Geo gs = geo_cell(A.P, A.D, A.bed_s, k, j, i, Ls);
        float f[19];
        stream_bc<S>(A, (const typename Store<S>::T *)A.fsrc, gs, Ls, k, j, i, c, f, cut, fscut, bridge);
        store_cell<S>(A, c, f);
        if (A.P.fs_mode != LBM_FS_NONE) {
            // post-stream macro_step of the water path, CODEX.py:3897
            int type;
            float fill;
            bool open = (gs.lo & 1u) != 0u;
            fs_state(A, c, k, j, open, type, fill);
            float gbf = gbf_of(A.P, k, open, type);
            float r, vx, vy, vz;
            macro(A.P, A.D, f, k, true, type, gbf, r, vx, vy, vz);
            A.rho[c] = r; A.ux[c] = vx; A.uy[c] = vy; A.uz[c] = vz;
        }
    }
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

// -------------------------------------------- height-function free surface
// compute_free_surface_column_flux, CODEX.py:2376-2388 (sequential in k)
__global__ void k_column_flux(const __grid_constant__ StepArgs A, float *qx_out, float *qy_out) {
    size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (a >= A.D.a) return;
    const Dom &D = A.D;
    int j = (int)(a / D.nx), i = (int)(a - (size_t)j * D.nx);
    float h = A.fs_h[a];
    float qx = 0.0f, qy = 0.0f;
    for (int k = 0; k < D.nz; ++k) {
        size_t c = D.cell(k, j, i);
        int type;
        float fill;
        classify_height(A.P, h, k, true, type, fill);
        if (type == LBM_FS_GAS) continue;
        if (!cell_open(A.P, D, A.bed_s, k, j, i)) continue;
        qx += fill * A.ux[c] * A.P.vel_scale * A.P.dx;
        qy += fill * A.uy[c] * A.P.vel_scale * A.P.dx;
    }
    qx_out[a] = qx;
    qy_out[a] = qy;
}

// advect_free_surface_height, CODEX.py:2391-2429
__global__ void k_advect(const __grid_constant__ lbm_params P, Dom D, const float *__restrict__ bed_h, const float *__restrict__ qx,
                         const float *__restrict__ qy, const float *__restrict__ h_in, float *h_out, float *h_last,
                         float t) {
    size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (a >= D.a) return;
    int j = (int)(a / D.nx), i = (int)(a - (size_t)j * D.nx);
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
// type_prev/type (F_VOF_STATE).
template <int S>
__global__ void __launch_bounds__(256) k_refill(const __grid_constant__ StepArgs A, const int8_t *type_prev_v, int *count) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    int did = 0;
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const bool vofm = (A.flags & F_VOF_STATE) != 0;
    if (c < D.n) {
        int k, j, i;
        cell_of(D, c, k, j, i);
        int tp, tn;
        float fl;
        bool cand;
        if (vofm) {
            tp = type_prev_v[c];
            tn = A.fs_type[c];
            cand = tp == LBM_FS_GAS && tn != LBM_FS_GAS;
        } else {
            classify_height(P, A.fs_h_last[D.col(j, i)], k, true, tp, fl);
            classify_height(P, A.fs_h[D.col(j, i)], k, true, tn, fl);
            cand = tp == LBM_FS_GAS && tn != LBM_FS_GAS;
        }
        if (cand && cell_open(P, D, A.bed_s, k, j, i)) {
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
                size_t nb = D.cell(nk, nj, ni);
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
                if (!cell_open(P, D, A.bed_s, nk, nj, ni)) continue;
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
                // stale gravity fraction: the state at the start of the step
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
                        size_t s = D.cell(sk, sj, si);
                        int stp, stn;
                        float sfl;
                        if (vofm) {
                            stp = type_prev_v[s];
                            stn = A.fs_type[s];
                        } else {
                            classify_height(P, A.fs_h_last[D.col(sj, si)], sk, true, stp, sfl);
                            classify_height(P, A.fs_h[D.col(sj, si)], sk, true, stn, sfl);
                        }
                        if (stp != LBM_FS_GAS && stn != LBM_FS_GAS && cell_open(P, D, A.bed_s, sk, sj, si))
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
            // the refilled cell is never a source for another refilled cell
            // (sources need type_prev != GAS), so writing in place is safe
            store_cell<S>(A, c, fr);
            did = 1;
        }
    }
    unsigned m = __activemask();
    int s = __reduce_add_sync(m, did);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(count, s);
}

// free-surface fields of the height path after a call: fill and type from
// the new height, type_prev from the height before advection
__global__ void k_height_types(const __grid_constant__ StepArgs A, float *fill, int8_t *type, int8_t *type_prev) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= A.D.n) return;
    int k, j, i;
    cell_of(A.D, c, k, j, i);
    bool open = cell_open(A.P, A.D, A.bed_s, k, j, i);
    int tp, tn;
    float fp, fn;
    classify_height(A.P, A.fs_h_last[A.D.col(j, i)], k, open, tp, fp);
    classify_height(A.P, A.fs_h[A.D.col(j, i)], k, open, tn, fn);
    fill[c] = fn;
    type[c] = (int8_t)tn;
    type_prev[c] = (int8_t)tp;
}

// ---------------------------------------------------------- launchers
static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

void launch_bed(const lbm_params &P, const Dom &D, const float *h_prev, float *h, float *hmax, float *uw, float *vw,
                float *ww, const float *piecewise, float t, cudaStream_t st) {
    k_bed<<<blocks_for(D.a, 256), 256, 0, st>>>(P, D, h_prev, h, uw, vw, ww, piecewise, t);
    k_hmax<<<blocks_for(D.a, 256), 256, 0, st>>>(D, h, hmax);
}
void launch_hmax(const Dom &D, const float *h, float *hmax, cudaStream_t st) {
    k_hmax<<<blocks_for(D.a, 256), 256, 0, st>>>(D, h, hmax);
}

template <int S>
static void launch_step_kernel_s(int which, const StepArgs &A, cudaStream_t st) {
    unsigned g = blocks_for(A.D.n, 256);
    switch (which) {
        case KER_PREPASS_CANON: k_prepass<S, 0><<<g, 256, 0, st>>>(A); break;
        case KER_PREPASS_FUSED: k_prepass<S, 1><<<g, 256, 0, st>>>(A); break;
        case KER_COLLIDE_CANON: k_collide<S, 0><<<g, 256, 0, st>>>(A); break;
        case KER_COLLIDE_FUSED: k_collide<S, 1><<<g, 256, 0, st>>>(A); break;
        case KER_STREAM: k_stream<S><<<g, 256, 0, st>>>(A); break;
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
void launch_column_flux(const StepArgs &A, float *qx, float *qy, cudaStream_t st) {
    k_column_flux<<<blocks_for(A.D.a, 128), 128, 0, st>>>(A, qx, qy);
}
void launch_advect(const lbm_params &P, const Dom &D, const float *bed_h, const float *qx, const float *qy,
                   const float *h_in, float *h_out, float *h_last, float t, cudaStream_t st) {
    k_advect<<<blocks_for(D.a, 256), 256, 0, st>>>(P, D, bed_h, qx, qy, h_in, h_out, h_last, t);
}
void launch_refill(const StepArgs &A, const int8_t *type_prev, int *count, cudaStream_t st) {
    unsigned g = blocks_for(A.D.n, 256);
    switch (A.P.pop_storage) {
        case LBM_STORE_F16S: k_refill<LBM_STORE_F16S><<<g, 256, 0, st>>>(A, type_prev, count); break;
        case LBM_STORE_BF16S: k_refill<LBM_STORE_BF16S><<<g, 256, 0, st>>>(A, type_prev, count); break;
        default: k_refill<LBM_STORE_F32><<<g, 256, 0, st>>>(A, type_prev, count); break;
    }
}
void launch_height_types(const StepArgs &A, float *fill, int8_t *type, int8_t *type_prev, cudaStream_t st) {
    k_height_types<<<blocks_for(A.D.n, 256), 256, 0, st>>>(A, fill, type, type_prev);
}

}  // namespace lbm
