// lbm_launch.h - argument structs and launchers shared by the kernel files
// and the host API of the B200 D3Q19 step engine.
#pragma once

#include <cuda_runtime.h>

#include "lbm_dev.cuh"

namespace lbm {

struct StepArgs;

enum { KER_PREPASS_CANON = 0, KER_PREPASS_FUSED = 1, KER_COLLIDE_CANON = 2, KER_COLLIDE_FUSED = 3, KER_STREAM = 4 };

struct InitArgs {
    lbm_params P;
    Dom D;
    BedView bed;
    void *f_cur, *f_other;
    float *rho, *ux, *uy, *uz, *omega;
    float *water_h, *water_h_last, *u_wave, *v_wave, *w_wave;
    float *fs_h, *fs_h_last, *fs_flux_x, *fs_flux_y;
    const float *piecewise;
    float *u_inlet_profile;
    const float *rho_initial, *noise;
    float *fs_fill, *fs_mass, *fs_mass_excess;
    int8_t *fs_type, *fs_type_prev, *fs_excess_dir;
};

struct ExportArgs {
    float *phi;
    int32_t *obstacle, *near_obstacle;
    int8_t *lattice_open;
    float *lattice_open_frac;
    int8_t *lattice_wall_type;
    float *prh, *gbf;
};

// solitary_surface_height_at_x, CODEX.py:1165-1181
LBM_DEV float solitary_h(const lbm_params &P, const Dom &D, float xp, float t) {
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
LBM_DEV float gaussian_h(const lbm_params &P, const Dom &D, float xp) {
    float Lx = (float)D.nx * P.dx;
    float xrel = xp - P.gaussian_center_x_m;
    if (!P.x_solid) {
        if (xrel > 0.5f * Lx) xrel -= Lx;
        if (xrel < -0.5f * Lx) xrel += Lx;
    }
    float arg = xrel / P.gaussian_sigma_m;
    return P.fs_base_m + P.gaussian_amp_m * lbm_expf(-0.5f * arg * arg);
}

void launch_bed(const lbm_params &P, const Dom &D, const float *h_prev, float *h, float *hmax, float *uw, float *vw,
                float *ww, const float *piecewise, float t, cudaStream_t st);
void launch_hmax(const Dom &D, const float *h, float *hmax, cudaStream_t st);
void launch_step_kernel(int which, const StepArgs &A, cudaStream_t st);
void launch_column_flux(const StepArgs &A, float *qx, float *qy, cudaStream_t st);
void launch_advect(const lbm_params &P, const Dom &D, const float *bed_h, const float *qx, const float *qy,
                   const float *h_in, float *h_out, float *h_last, float t, cudaStream_t st);
void launch_refill(const StepArgs &A, const int8_t *type_prev, int *count, cudaStream_t st);
void launch_height_types(const StepArgs &A, float *fill, int8_t *type, int8_t *type_prev, cudaStream_t st);

void launch_init_constants(const InitArgs &I, cudaStream_t st);
void launch_fs_height_init(const InitArgs &I, cudaStream_t st);
void launch_classify_store(const InitArgs &I, cudaStream_t st);
void launch_vof_block(const InitArgs &I, cudaStream_t st);
void launch_init_fields(const InitArgs &I, cudaStream_t st);
void launch_vof_mass_init(const InitArgs &I, cudaStream_t st);
void launch_export(const InitArgs &I, const ExportArgs &E, cudaStream_t st);

}  // namespace lbm
