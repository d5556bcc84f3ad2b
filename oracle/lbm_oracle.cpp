/*
 * lbm_oracle.cpp - CPU restatement of the reference D3Q19 step.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  This file is the oracle against
 * which the CUDA library is checked.  Only the tests, the smoke check and
 * the benchmark's CPU-baseline leg may load it.
 *
 * It restates, kernel by kernel and in the reference's own multi-pass
 * order, the Taichi kernels of LBM_3D_LES_air_over_waves_CODEX.py (cited
 * per function as CODEX.py:line).  It exports the same C ABI as the CUDA
 * library (include/lbm_b200.h) over HOST pointers, so the Python tests can
 * run both backends on identical inputs.
 *
 * Semantics pinned here (the reference leaves them to Taichi):
 *   - Arithmetic is IEEE f32 in source order; compile with
 *     -ffp-contract=off (no FMA contraction).  Python constants are rounded
 *     to f32 where Taichi captures them (the host layer pre-folds them into
 *     lbm_params).  The template parameter T = double gives the FP64
 *     reference run used for the storage-precision error budgets.
 *   - sin/cos/log/exp come from include/lbm_mathfn.h (double evaluation,
 *     one rounding), shared with the GPU so both round the same double.
 *   - Integer '%' on negative operands follows Python (floored).
 *   - Reference kernels with intra-kernel races get deterministic
 *     snapshot-read / ordered-apply semantics:
 *       redistribute_vof_mass_excess (CODEX.py:1417-1574),
 *       remove_orphan_vof_interface_cells (1659-1776): decisions read the
 *         pre-kernel state; a receiver adds its incoming shares in
 *         increasing (q, distance) order of the donor direction;
 *       advect_detached_vof_cells / compress_detached_vof_residuals
 *         (1861-1993): receivers sum incoming moves in +x,-x,+y,-y,+z,-z
 *         donor order;
 *       propagate_vof_exterior_gas_marks (2032-2054): Jacobi sweeps,
 *         i.e. a gas cell is exterior iff its 6-connected distance to a
 *         top-row seed is <= the sweep cap;
 *       f32 atomic sums (2070-2075, 1909, 1988) are FP64 sums in the fixed
 *         256-wide pairwise tree of lbm_tree_sum();
 *       repair_vof_coalescence_links (2319-2373) reads donor populations
 *         from the pre-kernel state.
 *   - Backscatter's ti.random (CODEX.py:3280) is the SplitMix64 counter
 *     RNG of lbm_mathfn.h keyed by (seed, step, cell); the initial kick of
 *     init_fields (2747) comes from the caller's init_noise buffer.
 *
 * Parity status: pinned against golden vectors produced by running the
 * reference's own kernel source through a numpy stand-in for Taichi
 * (tests/golden/gen_golden.py); see the golden tests for the tolerances.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lbm_b200.h"
#include "lbm_mathfn.h"

namespace {

const int CX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
const int CY[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1};
const int CZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16};

inline int pymod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

template <typename T> struct Fn;
template <> struct Fn<float> {
    static float sin(float x) { return lbm_sinf(x); }
    static float cos(float x) { return lbm_cosf(x); }
    static float log(float x) { return lbm_logf(x); }
    static float exp(float x) { return lbm_expf(x); }
    static float sqrt(float x) { return std::sqrt(x); }
    static float floor(float x) { return std::floor(x); }
};
template <> struct Fn<double> {
    static double sin(double x) { return lbm_sin_d(x); }
    static double cos(double x) { return lbm_cos_d(x); }
    static double log(double x) { return lbm_log_d(x); }
    static double exp(double x) { return lbm_exp_d(x); }
    static double sqrt(double x) { return std::sqrt(x); }
    static double floor(double x) { return std::floor(x); }
};

/* Deterministic FP64 sum: repeated 256-wide pairwise trees (stride
   halving) over consecutive chunks, until one value remains.  The CUDA
   library implements the identical tree. */
double tree_sum(std::vector<double> v) {
    if (v.empty()) return 0.0;
    while (v.size() > 1) {
        size_t nchunk = (v.size() + 255) / 256;
        std::vector<double> out(nchunk);
        for (size_t c = 0; c < nchunk; ++c) {
            double a[256];
            for (int t = 0; t < 256; ++t) {
                size_t idx = c * 256 + t;
                a[t] = idx < v.size() ? v[idx] : 0.0;
            }
            for (int s = 128; s >= 1; s >>= 1)
                for (int t = 0; t < s; ++t) a[t] = a[t] + a[t + s];
            out[c] = a[0];
        }
        v.swap(out);
    }
    return v[0];
}

struct CtxBase {
    virtual ~CtxBase() {}
    lbm_params p{};
    lbm_buffers b{};
    bool bound = false;
    std::string err;
    lbm_counters ctr{};
    virtual int init_geometry() = 0;
    virtual int init_fields() = 0;
    virtual int step(int n) = 0;
    virtual int export_diag() = 0;
};

template <typename T>
struct Sim : CtxBase {
    using F = Fn<T>;
    int Nx = 0, Ny = 0, Nz = 0;
    long N = 0, A = 0;
    int cur = 0;
    int64_t nstep = 0;
    /* internal state */
    std::vector<T> f[2];
    std::vector<T> rho, ux, uy, uz, omega, phi, prh, gbf, rho_initial;
    std::vector<int8_t> lo, wt;
    std::vector<T> lf;
    std::vector<int32_t> near_obs, obstacle, obstacle_prev, exterior;
    std::vector<T> water_h, water_h_last, u_wave, v_wave, w_wave, fs_h, fs_h_last, flux_x, flux_y, piecewise, prof;
    std::vector<T> fill, mass, mass_delta, mass_excess, detached_delta;
    std::vector<int8_t> type, type_prev, excess_dir;
    std::vector<float> noise;
    /* counters (reference scalar fields) */
    int32_t c_boundary_refill = 0, c_fs_refill = 0, c_coalesce = 0, c_bridge = 0, c_fs_cut = 0, c_vof_excess = 0,
            c_orphan = 0, c_collapse_cells = 0, c_det_count = 0, c_cmp_count = 0, c_cut = 0;
    T c_cand_vol = 0, c_applied_vol = 0, c_scale = 0, c_cand_mass = 0, c_capacity = 0, c_det_mass = 0, c_cmp_mass = 0;
    int32_t sweeps_used = 0;

    /* constants as the kernels use them */
    T dx, rho0, tau0, nu0;
    T w[19];

    long cell(int k, int j, int i) const { return ((long)k * Ny + j) * Nx + i; }
    long col(int j, int i) const { return (long)j * Nx + i; }
    long li(int q, long c) const { return (long)q * N + c; }

    bool water() const { return p.fs_mode != LBM_FS_NONE; }
    bool vof() const { return water() && p.fs_tracking == LBM_TRACK_VOF; }

    void setup() {
        Nx = p.nx; Ny = p.ny; Nz = p.nz;
        N = (long)Nx * Ny * Nz;
        A = (long)Nx * Ny;
        for (int s = 0; s < 2; ++s) f[s].assign(19 * N, T(0));
        rho.assign(N, 0); ux.assign(N, 0); uy.assign(N, 0); uz.assign(N, 0); omega.assign(N, 0);
        phi.assign(N, 0); prh.assign(N, 0); gbf.assign(N, 0); rho_initial.assign(N, 0);
        lo.assign(19 * N, 0); wt.assign(19 * N, 0); lf.assign(19 * N, 0);
        near_obs.assign(N, 0); obstacle.assign(N, 0); obstacle_prev.assign(N, 0); exterior.assign(N, 0);
        water_h.assign(A, 0); water_h_last.assign(A, 0); u_wave.assign(A, 0); v_wave.assign(A, 0);
        w_wave.assign(A, 0); fs_h.assign(A, 0); fs_h_last.assign(A, 0); flux_x.assign(A, 0); flux_y.assign(A, 0);
        piecewise.assign(Nx, 0); prof.assign(Nz, 0);
        fill.assign(N, 0); mass.assign(N, 0); mass_delta.assign(N, 0); mass_excess.assign(N, 0);
        detached_delta.assign(N, 0);
        type.assign(N, 0); type_prev.assign(N, 0); excess_dir.assign(N, 0);
        noise.assign(3 * N, 0.0f);
        dx = (T)p.dx; rho0 = (T)p.rho0; tau0 = (T)p.tau0; nu0 = (T)p.nu0;
        const T w0 = (T)(float)(1.0 / 3.0), w1 = (T)(float)(1.0 / 18.0), w2 = (T)(float)(1.0 / 36.0);
        for (int q = 0; q < 19; ++q) w[q] = q == 0 ? w0 : (q <= 6 ? w1 : w2);
    }

    /* ------------------------------------------------------------------
       buffer sync: the bound buffers are the state of record between calls
       ------------------------------------------------------------------ */
    template <typename S> static void load(std::vector<T> &dst, const S *src, long n) {
        if (src) for (long i = 0; i < n; ++i) dst[i] = (T)src[i];
    }
    template <typename S> static void store(const std::vector<T> &src, S *dst, long n) {
        if (dst) for (long i = 0; i < n; ++i) dst[i] = (S)src[i];
    }
    static void load8(std::vector<int8_t> &dst, const int8_t *src, long n) { if (src) memcpy(dst.data(), src, n); }
    static void store8(const std::vector<int8_t> &src, int8_t *dst, long n) { if (dst) memcpy(dst, src.data(), n); }

    void load_all() {
        for (int s = 0; s < 2; ++s) load(f[s], (const float *)b.f[s], 19 * N);
        load(rho, b.rho, N); load(ux, b.ux, N); load(uy, b.uy, N); load(uz, b.uz, N); load(omega, b.omega, N);
        load(water_h, b.water_h, A); load(water_h_last, b.water_h_last, A);
        load(u_wave, b.u_wave, A); load(v_wave, b.v_wave, A); load(w_wave, b.w_wave, A);
        load(fs_h, b.fs_h, A); load(fs_h_last, b.fs_h_last, A); load(flux_x, b.fs_flux_x, A); load(flux_y, b.fs_flux_y, A);
        load(piecewise, b.piecewise_bed_z, Nx); load(prof, b.u_inlet_profile, Nz);
        load(rho_initial, b.rho_initial, N);
        if (b.init_noise) memcpy(noise.data(), b.init_noise, sizeof(float) * 3 * N);
        load(fill, b.fs_fill, N); load8(type, b.fs_type, N); load8(type_prev, b.fs_type_prev, N);
        load(mass, b.fs_mass, N); load(mass_excess, b.fs_mass_excess, N); load8(excess_dir, b.fs_excess_dir, N);
    }
    void store_all() {
        for (int s = 0; s < 2; ++s) store(f[s], (float *)b.f[s], 19 * N);
        store(rho, b.rho, N); store(ux, b.ux, N); store(uy, b.uy, N); store(uz, b.uz, N); store(omega, b.omega, N);
        store(water_h, b.water_h, A); store(water_h_last, b.water_h_last, A);
        store(u_wave, b.u_wave, A); store(v_wave, b.v_wave, A); store(w_wave, b.w_wave, A);
        store(fs_h, b.fs_h, A); store(fs_h_last, b.fs_h_last, A); store(flux_x, b.fs_flux_x, A); store(flux_y, b.fs_flux_y, A);
        store(prof, b.u_inlet_profile, Nz);
        store(fill, b.fs_fill, N); store8(type, b.fs_type, N); store8(type_prev, b.fs_type_prev, N);
        store(mass, b.fs_mass, N); store(mass_excess, b.fs_mass_excess, N); store8(excess_dir, b.fs_excess_dir, N);
        fill_counters();
    }
    void fill_counters() {
        ctr.boundary_refill_count = c_boundary_refill;
        ctr.free_surface_refill_count = c_fs_refill;
        ctr.free_surface_coalescence_repair_count = c_coalesce;
        ctr.free_surface_thin_gap_bridge_count = c_bridge;
        ctr.free_surface_cut_link_count = c_fs_cut;
        ctr.free_surface_vof_excess_count = c_vof_excess;
        ctr.free_surface_vof_orphan_count = c_orphan;
        ctr.free_surface_vof_collapse_cell_count = c_collapse_cells;
        ctr.free_surface_vof_detached_advect_count = c_det_count;
        ctr.free_surface_vof_detached_compress_count = c_cmp_count;
        ctr.boundary_cut_link_count = c_cut;
        ctr.free_surface_vof_collapse_candidate_volume_m3 = (float)c_cand_vol;
        ctr.free_surface_vof_collapse_applied_volume_m3 = (float)c_applied_vol;
        ctr.free_surface_vof_collapse_removal_scale = (float)c_scale;
        ctr.free_surface_vof_collapse_candidate_mass = (float)c_cand_mass;
        ctr.free_surface_vof_collapse_exterior_capacity = (float)c_capacity;
        ctr.free_surface_vof_detached_advect_mass = (float)c_det_mass;
        ctr.free_surface_vof_detached_compress_mass = (float)c_cmp_mass;
        ctr.step = nstep;
        ctr.current_f = cur;
        ctr.flood_sweeps_used = sweeps_used;
    }

    /* ------------------------------------------------------------------
       helpers (CODEX.py:623-707, 821-988)
       ------------------------------------------------------------------ */
    /* calculate_feq, CODEX.py:623-643 */
    T feq(T r, T vx, T vy, T vz, int q) const {
        T u2 = vx * vx + vy * vy + vz * vz;
        T cu = T(3.0) * ((T)CX[q] * vx + (T)CY[q] * vy + (T)CZ[q] * vz);
        return r * w[q] * (T(1.0) + cu + T(0.5) * cu * cu - T(1.5) * u2);
    }
    /* local_g_body_lb, CODEX.py:646-651 */
    T g_local(long c) const {
        T g = (T)p.g_body_lb;
        if (p.use_component_balanced_pressure) g = (T)p.g_lb * gbf[c];
        return g;
    }
    static T smooth01(T x) { return x * x * (T(3.0) - T(2.0) * x); }

    /* periodic bilinear sampling weights of a centre-sampled 2-D field
       (CODEX.py:665-683, 2570-2588, 941-957) */
    void bilinear_setup(T xp, T yp, int &i0, int &j0, int &i1, int &j1, T &fx, T &fy) const {
        T Lx = (T)Nx * dx, Ly = (T)Ny * dx, Nxf = (T)Nx, Nyf = (T)Ny;
        T xw = xp - F::floor(xp / Lx) * Lx;
        T yw = yp - F::floor(yp / Ly) * Ly;
        T u = xw / dx - T(0.5);
        T v = yw / dx - T(0.5);
        u = u - F::floor(u / Nxf) * Nxf;
        v = v - F::floor(v / Nyf) * Nyf;
        i0 = (int)F::floor(u);
        j0 = (int)F::floor(v);
        fx = u - (T)i0;
        fy = v - (T)j0;
        /* a wrapped coordinate that rounds up to N would index out of range
           in the reference; wrap it */
        if (i0 >= Nx) i0 -= Nx;
        if (j0 >= Ny) j0 -= Ny;
        if (i0 < 0) i0 += Nx;
        if (j0 < 0) j0 += Ny;
        i1 = (i0 + 1) % Nx;
        j1 = (j0 + 1) % Ny;
    }
    T sample_h(const std::vector<T> &h, T xp, T yp) const {
        int i0, j0, i1, j1; T fx, fy;
        bilinear_setup(xp, yp, i0, j0, i1, j1, fx, fy);
        T h00 = h[col(j0, i0)], h10 = h[col(j0, i1)], h01 = h[col(j1, i0)], h11 = h[col(j1, i1)];
        T hx0 = h00 * (T(1.0) - fx) + h10 * fx;
        T hx1 = h01 * (T(1.0) - fx) + h11 * fx;
        return hx0 * (T(1.0) - fy) + hx1 * fy;
    }
    /* sample_wall_velocity_lb, CODEX.py:937-988 */
    void sample_wall_u(T xp, T yp, T &wx, T &wy, T &wz) const {
        int i0, j0, i1, j1; T fx, fy;
        bilinear_setup(xp, yp, i0, j0, i1, j1, fx, fy);
        auto bl = [&](const std::vector<T> &a) {
            T v00 = a[col(j0, i0)], v10 = a[col(j0, i1)], v01 = a[col(j1, i0)], v11 = a[col(j1, i1)];
            T x0 = v00 * (T(1.0) - fx) + v10 * fx;
            T x1 = v01 * (T(1.0) - fx) + v11 * fx;
            return x0 * (T(1.0) - fy) + x1 * fy;
        };
        wx = bl(u_wave); wy = bl(v_wave); wz = bl(w_wave);
    }
    /* sample_phi_periodic, CODEX.py:661-707 */
    T sample_phi(T xp, T yp, T zp) const {
        int i0, j0, i1, j1; T fx, fy;
        bilinear_setup(xp, yp, i0, j0, i1, j1, fx, fy);
        T r = zp / dx - T(0.5);
        int k0 = (int)F::floor(r);
        T fz = r - (T)k0;
        int k1 = k0 + 1;
        if (k0 < 0) { k0 = 0; k1 = 0; fz = T(0.0); }
        if (k1 >= Nz) { k0 = Nz - 1; k1 = Nz - 1; fz = T(0.0); }
        T p00_0 = phi[cell(k0, j0, i0)] * (T(1.0) - fx) + phi[cell(k0, j0, i1)] * fx;
        T p01_0 = phi[cell(k0, j1, i0)] * (T(1.0) - fx) + phi[cell(k0, j1, i1)] * fx;
        T pxy_0 = p00_0 * (T(1.0) - fy) + p01_0 * fy;
        T p00_1 = phi[cell(k1, j0, i0)] * (T(1.0) - fx) + phi[cell(k1, j0, i1)] * fx;
        T p01_1 = phi[cell(k1, j1, i0)] * (T(1.0) - fx) + phi[cell(k1, j1, i1)] * fx;
        T pxy_1 = p00_1 * (T(1.0) - fy) + p01_1 * fy;
        return pxy_0 * (T(1.0) - fz) + pxy_1 * fz;
    }
    /* cube_sdf_at_point, CODEX.py:897-934 */
    T cube_sdf(T xp, T yp, T zp) const {
        T Lx = (T)Nx * dx, Ly = (T)Ny * dx;
        T dxp = xp - (T)p.cube_cx;
        T dyp = yp - (T)p.cube_cy;
        if (!p.x_solid) {
            if (dxp > T(0.5) * Lx) dxp -= Lx;
            if (dxp < -T(0.5) * Lx) dxp += Lx;
        }
        if (dyp > T(0.5) * Ly) dyp -= Ly;
        if (dyp < -T(0.5) * Ly) dyp += Ly;
        T xl = (T)p.cube_yaw_cos * dxp + (T)p.cube_yaw_sin * dyp;
        T yl = -(T)p.cube_yaw_sin * dxp + (T)p.cube_yaw_cos * dyp;
        T z1 = zp - (T)p.cube_cz;
        T xpitch = (T)p.cube_pitch_cos * xl - (T)p.cube_pitch_sin * z1;
        T zl = (T)p.cube_pitch_sin * xl + (T)p.cube_pitch_cos * z1;
        T qx = std::fabs(xpitch) - (T)p.cube_hx;
        T qy = std::fabs(yl) - (T)p.cube_hy;
        T qz = std::fabs(zl) - (T)p.cube_hz;
        T ox = std::max(qx, T(0.0)), oy = std::max(qy, T(0.0)), oz = std::max(qz, T(0.0));
        T outside = F::sqrt(ox * ox + oy * oy + oz * oz);
        T inside = std::min(std::max(qx, std::max(qy, qz)), T(0.0));
        return outside + inside;
    }
    /* free_surface_hydrostatic_density_at_cell, CODEX.py:821-845; gravity
       fraction taken from the given array (stale fraction semantics) */
    T fs_density_cell(int k, int j, int i, T gbf_c) const {
        T head = T(0.0);
        if (p.use_component_balanced_pressure) {
            T zc = ((T)k + T(0.5)) * dx;
            head = gbf_c < T(0.5) ? zc - (T)p.fs_base_m : T(0.0);
        } else if (p.use_hydrostatic_balanced_pressure) {
            head = fs_h[col(j, i)] - (T)p.fs_base_m;
        } else {
            T zc = ((T)k + T(0.5)) * dx;
            head = fs_h[col(j, i)] - zc;
        }
        if (head < T(0.0) && !p.use_hydrostatic_balanced_pressure) head = T(0.0);
        return rho0 + (T)p.g_lb * (head / dx) / (T)p.one_third;
    }
    /* free_surface_pressure_density_at_link, CODEX.py:848-867 */
    T fs_density_link(int k, int j, int i, int q) const {
        long c = cell(k, j, i);
        if (p.use_component_balanced_pressure) {
            T zi = ((T)k + T(0.5)) * dx - T(0.5) * (T)CZ[q] * dx;
            T head = T(0.0);
            if (gbf[c] < T(0.5)) head += zi - (T)p.fs_base_m;
            return rho0 + (T)p.g_lb * (head / dx) / (T)p.one_third;
        } else if (p.use_hydrostatic_balanced_pressure && vof()) {
            T zi = ((T)k + T(0.5)) * dx - T(0.5) * (T)CZ[q] * dx;
            T head = zi - (T)p.fs_base_m;
            return rho0 + (T)p.g_lb * (head / dx) / (T)p.one_third;
        }
        return fs_density_cell(k, j, i, gbf[c]);
    }
    /* vof_cell_liquid_fraction, CODEX.py:870-885 */
    T vof_alpha(long c) const {
        T a = T(1.0);
        if (vof() && lo[li(0, c)] == 1) {
            if (type[c] == LBM_FS_GAS) a = T(0.0);
            else if (type[c] == LBM_FS_INTERFACE) {
                a = fill[c];
                if (a < T(0.0)) a = T(0.0);
                if (a > T(1.0)) a = T(1.0);
            }
        }
        return a;
    }

    /* ------------------------------------------------------------------
       geometry producers
       ------------------------------------------------------------------ */
    /* update_wave_bed_and_velocities, CODEX.py:1082-1162 (two harmonics
       generalised to (amp_h, k_h, c_h); the reference's are
       (amp, k/2, c) and (amp, k, c/2)) */
    void update_bed(T t) {
        const bool moving = p.bed_profile == LBM_BED_MOVING_SINE;
        T ramp = (T)p.bed_ramp_time;
        T a1 = T(0.0), a2 = T(0.0);
        if (moving) {
            if (t < ramp) {
                T s = smooth01(t / ramp);
                a1 = (T)p.bed_amp1 * s;
                a2 = (T)p.bed_amp2 * s;
            } else {
                a1 = (T)p.bed_amp1;
                a2 = (T)p.bed_amp2;
            }
        }
        const T k1 = (T)p.bed_k1, k2 = (T)p.bed_k2, c1 = (T)p.bed_c1, c2 = (T)p.bed_c2;
        const T h0 = (T)p.bed_h0, dtp = (T)p.dt_phys_f, vs = (T)p.vel_scale;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                long a = col(j, i);
                T x0 = (T)i * dx;
                water_h_last[a] = water_h[a];
                T eta1 = 0, eta2 = 0, eta = 0, ph1 = 0, ph2 = 0;
                if (moving) {
                    T xph1 = x0 - c1 * t;
                    T xph2 = x0 - c2 * t;
                    ph1 = k1 * xph1;
                    ph2 = k2 * xph2;
                    eta1 = a1 * F::sin(ph1);
                    eta2 = a2 * F::sin(ph2);
                    eta = eta1 + eta2;
                }
                T bed_h = (T)p.bed_offset_m + eta;
                if (p.bed_profile == LBM_BED_PIECEWISE) bed_h = piecewise[i];
                water_h[a] = bed_h;
                T us = 0, vsv = 0, ws = 0;
                if (moving) {
                    T ex1 = a1 * k1 * F::cos(ph1);
                    T ex2 = a2 * k2 * F::cos(ph2);
                    T eta_x = ex1 + ex2;
                    T eta_y = T(0.0);
                    T eta_t = (water_h[a] - water_h_last[a]) / dtp;
                    if (p.bed_orbital_velocity) us = c1 * eta1 / (h0 + eta1) + c2 * eta2 / (h0 + eta2);
                    ws = eta_t + us * eta_x + vsv * eta_y;
                }
                u_wave[a] = us / vs;
                v_wave[a] = vsv / vs;
                w_wave[a] = ws / vs;
            }
    }

    /* compute_phi_slope_corrected, CODEX.py:2432-2490 */
    void compute_phi() {
        const T hid = (T)p.half_inv_dx;
#pragma omp parallel for collapse(2)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int ip = (i + 1) % Nx, im = (i - 1 + Nx) % Nx, jp = (j + 1) % Ny, jm = (j - 1 + Ny) % Ny;
                T dhdx = (water_h[col(j, ip)] - water_h[col(j, im)]) * hid;
                if (p.x_solid) {
                    if (i == 0) dhdx = (water_h[col(j, i + 1)] - water_h[col(j, i)]) / dx;
                    else if (i == Nx - 1) dhdx = (water_h[col(j, i)] - water_h[col(j, i - 1)]) / dx;
                }
                T dhdy = (water_h[col(jp, i)] - water_h[col(jm, i)]) * hid;
                T denom = F::sqrt(T(1.0) + dhdx * dhdx + dhdy * dhdy);
                if (denom < T(1e-6)) denom = T(1.0);
                T hl = water_h[col(j, i)];
                for (int k = 0; k < Nz; ++k) {
                    T zc = ((T)k + T(0.5)) * dx;
                    T xc = ((T)i + T(0.5)) * dx;
                    T yc = ((T)j + T(0.5)) * dx;
                    T v = T(1.0e6);
                    if (p.include_bed) v = (zc - hl) / denom;
                    if (p.include_cube) {
                        T cp = cube_sdf(xc, yc, zc);
                        if (cp < v) v = cp;
                    }
                    if (p.x_solid) {
                        T xw = std::min(xc, (T)Nx * dx - xc);
                        if (xw < v) v = xw;
                    }
                    phi[cell(k, j, i)] = v;
                }
            }
    }

    /* build_lattice_open_from_free_surface_periodic, CODEX.py:2492-2686 */
    void build_lattice_open() {
        const T hdx = T(0.5) * dx;
#pragma omp parallel for collapse(2)
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < Nx; ++i) {
                    long c = cell(k, j, i);
                    T xc = ((T)i + T(0.5)) * dx, yc = ((T)j + T(0.5)) * dx, zc = ((T)k + T(0.5)) * dx;
                    int8_t lov[19] = {0};
                    T lfv[19] = {0};
                    int8_t wtv[19] = {0};
                    T eta_c = sample_h(water_h, xc, yc);
                    T gap_c = zc - eta_c;
                    T ggc = T(1.0e6);
                    int wtc = LBM_WALL_NONE;
                    if (p.include_bed) { ggc = gap_c; wtc = LBM_WALL_BED; }
                    if (p.include_cube) {
                        T cg = cube_sdf(xc, yc, zc);
                        if (cg < ggc) { ggc = cg; wtc = LBM_WALL_CUBE; }
                    }
                    T sgc = ggc;
                    if (p.use_phi_open_fraction) sgc = phi[c];
                    T frc = T(0.5) + sgc / dx;
                    if (frc < T(0.0)) frc = T(0.0);
                    if (frc > T(1.0)) frc = T(1.0);
                    lfv[0] = frc;
                    wtv[0] = (int8_t)wtc;
                    for (int q = 1; q < 19; ++q) {
                        T xq = xc + hdx * (T)CX[q];
                        T yq = yc + hdx * (T)CY[q];
                        T zq = zc + hdx * (T)CZ[q];
                        T eta = sample_h(water_h, xq, yq);
                        T gap = zq - eta;
                        T gg = T(1.0e6);
                        int wq = LBM_WALL_NONE;
                        if (p.include_bed) { gg = gap; wq = LBM_WALL_BED; }
                        if (p.include_cube) {
                            T cg = cube_sdf(xq, yq, zq);
                            if (cg < gg) { gg = cg; wq = LBM_WALL_CUBE; }
                        }
                        T sg = gg;
                        if (p.use_phi_open_fraction) sg = sample_phi(xq, yq, zq);
                        T fr = T(0.5) + sg / dx;
                        if (fr < T(0.0)) fr = T(0.0);
                        if (fr > T(1.0)) fr = T(1.0);
                        lfv[q] = fr;
                        wtv[q] = (int8_t)wq;
                        T og = gg;
                        if (p.use_phi_open_flags) og = sg;
                        lov[q] = og < T(0.0) ? 0 : 1;
                        if (p.x_solid) {
                            if (i == 0 && CX[q] > 0) { lov[q] = 0; lfv[q] = T(0.0); wtv[q] = LBM_WALL_XMIN; }
                            else if (i == Nx - 1 && CX[q] < 0) { lov[q] = 0; lfv[q] = T(0.0); wtv[q] = LBM_WALL_XMAX; }
                        }
                    }
                    lov[0] = 0;
                    for (int q = 1; q < 19; ++q) if (lov[q] == 1) lov[0] = 1;
                    int nb = 0;
                    for (int q = 1; q < 19; ++q) if (lov[q] == 0) nb = 1;
                    near_obs[c] = nb;
                    if (lov[0] == 0) for (int q = 1; q < 19; ++q) lfv[q] = T(0.0);
                    for (int q = 0; q < 19; ++q) {
                        lo[li(q, c)] = lov[q];
                        lf[li(q, c)] = lfv[q];
                        wt[li(q, c)] = wtv[q];
                    }
                }
    }

    /* ------------------------------------------------------------------
       free-surface initial height and classification
       ------------------------------------------------------------------ */
    /* solitary_surface_height_at_x, CODEX.py:1165-1181 */
    T solitary_h(T xp, T t) const {
        T Lx = (T)Nx * dx;
        T h0 = (T)p.fs_depth_m;
        T ks = F::sqrt((T)(float)(3.0 * (double)p.solitary_amp_m) / (T(4.0) * h0 * h0 * h0));
        T center = (T)p.solitary_x0_m + (T)p.solitary_dir_cel * t;
        T xrel = xp - center;
        if (!p.x_solid) {
            if (xrel > T(0.5) * Lx) xrel -= Lx;
            if (xrel < -T(0.5) * Lx) xrel += Lx;
        }
        T arg = ks * xrel;
        T ep = F::exp(arg), em = F::exp(-arg);
        T sech = T(2.0) / (ep + em);
        return (T)p.fs_base_m + (T)p.solitary_amp_m * sech * sech;
    }
    /* gaussian_surface_height_at_x, CODEX.py:1184-1194 */
    T gaussian_h(T xp) const {
        T Lx = (T)Nx * dx;
        T xrel = xp - (T)p.gaussian_center_x_m;
        if (!p.x_solid) {
            if (xrel > T(0.5) * Lx) xrel -= Lx;
            if (xrel < -T(0.5) * Lx) xrel += Lx;
        }
        T arg = xrel / (T)p.gaussian_sigma_m;
        return (T)p.fs_base_m + (T)p.gaussian_amp_m * F::exp(-T(0.5) * arg * arg);
    }
    /* initialize_free_surface_height, CODEX.py:1197-1207 */
    void init_fs_height(T t) {
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                T x = ((T)i + T(0.5)) * dx;
                T h = (T)p.fs_base_m;
                if (p.fs_initial == LBM_FSINIT_SOLITARY || p.fs_mode == LBM_FS_PRESCRIBED_SOLITARY) h = solitary_h(x, t);
                else if (p.fs_initial == LBM_FSINIT_GAUSSIAN) h = gaussian_h(x);
                fs_h[col(j, i)] = h;
                fs_h_last[col(j, i)] = h;
            }
    }
    /* classify_free_surface_cells, CODEX.py:1210-1235 */
    void classify() {
#pragma omp parallel for
        for (long c = 0; c < N; ++c) {
            int k = (int)(c / A);
            long a = c % A;
            int8_t old = type[c];
            T fl = T(1.0);
            int8_t ct = LBM_FS_LIQUID;
            if (water()) {
                T zb = (T)k * dx;
                T h = fs_h[a];
                fl = (h - zb) / dx;
                if (fl < T(0.0)) fl = T(0.0);
                if (fl > T(1.0)) fl = T(1.0);
                if (fl <= T(FILL_LO)) ct = LBM_FS_GAS;
                else if (fl >= T(FILL_HI)) ct = LBM_FS_LIQUID;
                else ct = LBM_FS_INTERFACE;
                if (lo[li(0, c)] == 0) { fl = T(0.0); ct = LBM_FS_GAS; }
            }
            fill[c] = fl;
            type_prev[c] = old;
            type[c] = ct;
        }
    }
    static T overlap(T cmin, T cmax, T bmin, T bmax) {
        T lo_ = cmin;
        if (bmin > lo_) lo_ = bmin;
        T hi = cmax;
        if (bmax < hi) hi = bmax;
        T ov = hi - lo_;
        if (ov < T(0.0)) ov = T(0.0);
        return ov / (cmax - cmin);
    }
    /* apply_vof_initial_disconnected_shape, CODEX.py:1253-1286 */
    void vof_initial_block() {
        if (!(vof() && p.vof_initial_block)) return;
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < Nx; ++i) {
                    long c = cell(k, j, i);
                    if (lo[li(0, c)] != 1) continue;
                    T x0 = (T)i * dx, x1 = x0 + dx, y0 = (T)j * dx, y1 = y0 + dx, z0 = (T)k * dx, z1 = z0 + dx;
                    T fx = overlap(x0, x1, (T)p.vof_block_xmin, (T)p.vof_block_xmax);
                    T fy = overlap(y0, y1, (T)p.vof_block_ymin, (T)p.vof_block_ymax);
                    T fz = overlap(z0, z1, (T)p.vof_block_zmin, (T)p.vof_block_zmax);
                    T bf = fx * fy * fz;
                    if (bf > T(FILL_LO)) {
                        int8_t old = type[c];
                        T fl = fill[c];
                        if (bf > fl) fl = bf;
                        int8_t ct = LBM_FS_INTERFACE;
                        if (fl >= T(FILL_HI)) { fl = T(1.0); ct = LBM_FS_LIQUID; }
                        fill[c] = fl;
                        type_prev[c] = old;
                        type[c] = ct;
                    }
                }
    }
    /* update_pressure_reference_fields, CODEX.py:710-740 */
    void update_pressure_reference() {
#pragma omp parallel for
        for (long c = 0; c < N; ++c) {
            int k = (int)(c / A);
            prh[c] = T(0.0);
            gbf[c] = T(0.0);
            if (water() && lo[li(0, c)] == 1 && type[c] != LBM_FS_GAS) {
                T zc = ((T)k + T(0.5)) * dx;
                if (p.pressure_formulation == LBM_PRESSURE_HYDROSTATIC_BALANCED) {
                    prh[c] = (T)p.fs_base_m - zc;
                    gbf[c] = T(0.0);
                } else if (p.pressure_formulation == LBM_PRESSURE_VOF_COMPONENT_BALANCED) {
                    if (zc < (T)p.fs_base_m) { prh[c] = (T)p.fs_base_m - zc; gbf[c] = T(0.0); }
                    else { prh[c] = T(0.0); gbf[c] = T(1.0); }
                } else {
                    gbf[c] = T(1.0);
                }
            }
        }
    }

#include "lbm_oracle_step.inc"
#include "lbm_oracle_vof.inc"
};

}  // namespace

/* ======================================================================
   C ABI (include/lbm_b200.h), host pointers
   ====================================================================== */
struct lbm_ctx {
    CtxBase *impl;
};

static int make_ctx(const lbm_params *params, lbm_ctx **out, bool fp64) {
    if (!params || !out) return LBM_ERR_BAD_ARG;
    if (params->abi_version != LBM_ABI_VERSION || params->magic_end != LBM_PARAMS_MAGIC) return LBM_ERR_BAD_ARG;
    if (params->nx < 1 || params->ny < 1 || params->nz < 2) return LBM_ERR_BAD_ARG;
    if (params->x_solid && params->nx < 2) return LBM_ERR_BAD_ARG;
    lbm_ctx *c = new lbm_ctx;
    if (fp64) {
        auto *s = new Sim<double>();
        s->p = *params;
        s->setup();
        c->impl = s;
    } else {
        auto *s = new Sim<float>();
        s->p = *params;
        s->setup();
        c->impl = s;
    }
    *out = c;
    return LBM_OK;
}

extern "C" {

const char *lbm_backend_name(void) { return "cpu-oracle"; }
int lbm_abi_version(void) { return LBM_ABI_VERSION; }
int64_t lbm_struct_size(int32_t which) {
    switch (which) {
        case 0: return (int64_t)sizeof(lbm_params);
        case 1: return (int64_t)sizeof(lbm_buffers);
        case 2: return (int64_t)sizeof(lbm_counters);
        case 3: return (int64_t)sizeof(lbm_diag);
        case 4: return (int64_t)sizeof(lbm_diag_inputs);
        default: return -1;
    }
}
int lbm_create(const lbm_params *params, lbm_ctx **out) { return make_ctx(params, out, false); }
/* oracle only: the FP64 reference run */
int lbm_oracle_create_fp64(const lbm_params *params, lbm_ctx **out) { return make_ctx(params, out, true); }

int lbm_bind(lbm_ctx *ctx, const lbm_buffers *bufs) {
    if (!ctx || !bufs) return LBM_ERR_BAD_ARG;
    if (!bufs->f[0] || !bufs->f[1]) { ctx->impl->err = "f buffers are required"; return LBM_ERR_BAD_ARG; }
    ctx->impl->b = *bufs;
    ctx->impl->bound = true;
    return LBM_OK;
}
int lbm_init_geometry(lbm_ctx *ctx, void *) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->impl->bound) return LBM_ERR_NOT_BOUND;
    return ctx->impl->init_geometry();
}
int lbm_init_fields(lbm_ctx *ctx, void *) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->impl->bound) return LBM_ERR_NOT_BOUND;
    return ctx->impl->init_fields();
}
int lbm_step(lbm_ctx *ctx, int32_t nsteps, void *) {
    if (!ctx || nsteps < 0) return LBM_ERR_BAD_ARG;
    if (!ctx->impl->bound) return LBM_ERR_NOT_BOUND;
    return ctx->impl->step(nsteps);
}
int lbm_export_diagnostics(lbm_ctx *ctx, void *) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->impl->bound) return LBM_ERR_NOT_BOUND;
    return ctx->impl->export_diag();
}
int lbm_read_counters(lbm_ctx *ctx, lbm_counters *out) {
    if (!ctx || !out) return LBM_ERR_BAD_ARG;
    *out = ctx->impl->ctr;
    return LBM_OK;
}
int lbm_link_geometry_noalloc(const lbm_params *, const float *, float *, int32_t *, int32_t *, int8_t *, float *,
                              int8_t *, void *, char *err, size_t err_len) {
    if (err && err_len) snprintf(err, err_len, "%s", "the CPU oracle has no allocation-free variant");
    return LBM_ERR_UNSUPPORTED;
}
int lbm_set_tile_chunk(lbm_ctx *ctx, int32_t planes) {
    return (ctx && planes >= 0) ? LBM_OK : LBM_ERR_BAD_ARG;
}
int lbm_set_step_graphs(lbm_ctx *ctx, int32_t) { return ctx ? LBM_OK : LBM_ERR_BAD_ARG; }
int lbm_batch_create(lbm_ctx *const *, int32_t, lbm_batch **out) {
    if (out) *out = nullptr;
    return LBM_ERR_UNSUPPORTED;   // ensembles are a device-side feature
}
int lbm_batch_step(lbm_batch *, int32_t, void *) { return LBM_ERR_UNSUPPORTED; }
int lbm_batch_destroy(lbm_batch *) { return LBM_ERR_BAD_ARG; }
const char *lbm_batch_last_error(lbm_batch *) { return "the CPU oracle has no ensembles"; }
int lbm_diagnostics(lbm_ctx *ctx, const lbm_diag_inputs *in, lbm_diag *out, void *) {
    if (!ctx || !in || !out) return LBM_ERR_BAD_ARG;
    return LBM_ERR_UNSUPPORTED;   // device reductions only; the oracle's fields are on the host
}
int lbm_set_arithmetic(lbm_ctx *ctx, int32_t mode) {
    return (ctx && (mode == LBM_ARITH_EXACT || mode == LBM_ARITH_FAST)) ? LBM_OK : LBM_ERR_BAD_ARG;
}
int lbm_get_arithmetic(lbm_ctx *ctx, int32_t *mode) {
    if (!ctx || !mode) return LBM_ERR_BAD_ARG;
    *mode = LBM_ARITH_EXACT;   // the oracle computes in the reference's order only
    return LBM_OK;
}
int lbm_launch_count(int64_t *count) {
    if (!count) return LBM_ERR_BAD_ARG;
    *count = 0;
    return LBM_OK;
}
int lbm_set_kernel_timing(lbm_ctx *ctx, int32_t) { return ctx ? LBM_OK : LBM_ERR_BAD_ARG; }
int lbm_kernel_timing(lbm_ctx *ctx, double *total_ms, int64_t *launches, int64_t *cells) {
    if (!ctx || !total_ms || !launches || !cells) return LBM_ERR_BAD_ARG;
    *total_ms = 0.0;
    *launches = 0;
    *cells = 0;
    return LBM_OK;
}
int lbm_destroy(lbm_ctx *ctx) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    delete ctx->impl;
    delete ctx;
    return LBM_OK;
}
const char *lbm_last_error(lbm_ctx *ctx) { return ctx ? ctx->impl->err.c_str() : "null context"; }

/* oracle only: the deterministic FP64 tree sum, exposed for tests */
double lbm_oracle_tree_sum(const double *v, int64_t n) {
    if (!v || n <= 0) return 0.0;
    std::vector<double> x(v, v + n);
    return tree_sum(x);
}

}  // extern "C"
