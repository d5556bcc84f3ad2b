// lbm_init.cu - initialisation kernels (CODEX.py:992-1080, 1165-1302,
// 2688-2875) and the on-demand export of the per-cell fields the
// reference keeps resident (phi, obstacle, lattice_open*, pressure
// reference).  Setup only; none of these run inside the step loop.
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
static inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// init_constants, CODEX.py:1022-1080
__global__ void k_init_constants(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const Dom &D = I.D;
    const lbm_params &P = I.P;
    if (c < D.n) {
        I.rho[c] = P.rho0; I.ux[c] = 0.0f; I.uy[c] = 0.0f; I.uz[c] = 0.0f;
        I.omega[c] = P.omega0;
        if (I.fs_fill) I.fs_fill[c] = 1.0f;
        if (I.fs_type) I.fs_type[c] = LBM_FS_LIQUID;
        if (I.fs_type_prev) I.fs_type_prev[c] = LBM_FS_LIQUID;
        if (I.fs_mass) I.fs_mass[c] = P.rho0;
        if (I.fs_mass_excess) I.fs_mass_excess[c] = 0.0f;
        if (I.fs_excess_dir) I.fs_excess_dir[c] = 0;
    }
    if (c < D.a) {
        int i = (int)(c % D.nx);
        float bh = P.bed_offset_m;
        if (P.bed_profile == LBM_BED_PIECEWISE) bh = I.piecewise[i];
        I.water_h[c] = bh;
        I.water_h_last[c] = bh;
        I.u_wave[c] = 0.0f; I.v_wave[c] = 0.0f; I.w_wave[c] = 0.0f;
        I.fs_h[c] = P.fs_base_m;
        I.fs_h_last[c] = P.fs_base_m;
        if (I.fs_flux_x) I.fs_flux_x[c] = 0.0f;
        if (I.fs_flux_y) I.fs_flux_y[c] = 0.0f;
    }
}

// initialize_free_surface_height, CODEX.py:1197-1207
__global__ void k_fs_height_init(const __grid_constant__ InitArgs I) {
    size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (a >= I.D.a) return;
    const lbm_params &P = I.P;
    int i = (int)(a % I.D.nx);
    float x = ((float)i + 0.5f) * P.dx;
    float h = P.fs_base_m;
    if (P.fs_initial == LBM_FSINIT_SOLITARY || P.fs_mode == LBM_FS_PRESCRIBED_SOLITARY) h = solitary_h(P, I.D, x, 0.0f);
    else if (P.fs_initial == LBM_FSINIT_GAUSSIAN) h = gaussian_h(P, I.D, x);
    I.fs_h[a] = h;
    I.fs_h_last[a] = h;
}

// classify_free_surface_cells, CODEX.py:1210-1235 (stored form)
__global__ void k_classify_store(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    int8_t old = I.fs_type[c];
    float fl = 1.0f;
    int ct = LBM_FS_LIQUID;
    if (I.P.fs_mode != LBM_FS_NONE) {
        bool open = cell_open(I.P, I.D, I.bed, k, j, i);
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
__global__ void k_vof_block(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
    const lbm_params &P = I.P;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    if (!cell_open(P, I.D, I.bed, k, j, i)) return;
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
__global__ void k_profile(const __grid_constant__ InitArgs I) {
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
__global__ void k_init_fields(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
    const lbm_params &P = I.P;
    const Dom &D = I.D;
    int k, j, i;
    cell_of(D, c, k, j, i);
    GeoLinks L;
    Geo g = geo_cell(P, D, I.bed, k, j, i, L);
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
            size_t a = D.col(j, i);
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
__global__ void k_fs_boundary_pop(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
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
        bool open = cell_open(P, D, I.bed, k, j, i);
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
                    size_t s = D.cell(sk, sj, si);
                    if (I.fs_type[s] == LBM_FS_GAS && cell_open(P, D, I.bed, sk, sj, si)) src_gas = true;
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
__global__ void k_vof_mass_init(const __grid_constant__ InitArgs I) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
    int k, j, i;
    cell_of(I.D, c, k, j, i);
    bool open = cell_open(I.P, I.D, I.bed, k, j, i);
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
__global__ void k_export(const __grid_constant__ InitArgs I, const __grid_constant__ ExportArgs E) {
    size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (c >= I.D.n) return;
    const lbm_params &P = I.P;
    const Dom &D = I.D;
    int k, j, i;
    cell_of(D, c, k, j, i);
    GeoLinks L;
    Geo g = geo_cell(P, D, I.bed, k, j, i, L, false);
    bool open = (g.lo & 1u) != 0u;
    if (E.phi) E.phi[c] = phi_cell(P, D, I.bed.h, k, j, i);
    if (E.obstacle) E.obstacle[c] = open ? 0 : 1;
    if (E.near_obstacle) E.near_obstacle[c] = g.near ? 1 : 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (E.lattice_open) E.lattice_open[(size_t)q * D.n + c] = (int8_t)((g.lo >> q) & 1u);
        if (E.lattice_open_frac) E.lattice_open_frac[(size_t)q * D.n + c] = L.lf[q];
        if (E.lattice_wall_type) E.lattice_wall_type[(size_t)q * D.n + c] = (int8_t)L.wt[q];
    }
    int tp = I.fs_type_prev ? I.fs_type_prev[c] : LBM_FS_LIQUID;
    if (E.prh) E.prh[c] = prh_of(P, k, open, tp);
    if (E.gbf) E.gbf[c] = gbf_of(P, k, open, tp);
}

// ---------------------------------------------------------------- launchers
void launch_init_constants(const InitArgs &I, cudaStream_t st) {
    size_t n = I.D.n > I.D.a ? I.D.n : I.D.a;
    k_init_constants<<<blocks_for(n, 256), 256, 0, st>>>(I);
}
void launch_fs_height_init(const InitArgs &I, cudaStream_t st) {
    k_fs_height_init<<<blocks_for(I.D.a, 256), 256, 0, st>>>(I);
}
void launch_classify_store(const InitArgs &I, cudaStream_t st) {
    k_classify_store<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I);
}
void launch_vof_block(const InitArgs &I, cudaStream_t st) {
    k_vof_block<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I);
}
void launch_init_fields(const InitArgs &I, cudaStream_t st) {
    k_profile<<<1, 1, 0, st>>>(I);
    unsigned g = blocks_for(I.D.n, 256);
    switch (I.P.pop_storage) {
        case LBM_STORE_F16S:
            k_init_fields<LBM_STORE_F16S><<<g, 256, 0, st>>>(I);
            k_fs_boundary_pop<LBM_STORE_F16S><<<g, 256, 0, st>>>(I);
            break;
        case LBM_STORE_BF16S:
            k_init_fields<LBM_STORE_BF16S><<<g, 256, 0, st>>>(I);
            k_fs_boundary_pop<LBM_STORE_BF16S><<<g, 256, 0, st>>>(I);
            break;
        default:
            k_init_fields<LBM_STORE_F32><<<g, 256, 0, st>>>(I);
            k_fs_boundary_pop<LBM_STORE_F32><<<g, 256, 0, st>>>(I);
            break;
    }
}
void launch_vof_mass_init(const InitArgs &I, cudaStream_t st) {
    k_vof_mass_init<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I);
}
void launch_export(const InitArgs &I, const ExportArgs &E, cudaStream_t st) {
    k_export<<<blocks_for(I.D.n, 256), 256, 0, st>>>(I, E);
}

}  // namespace lbm
