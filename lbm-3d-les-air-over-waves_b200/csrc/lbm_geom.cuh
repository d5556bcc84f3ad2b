// lbm_geom.cuh - per-link solid geometry recomputed in registers.
//
// The reference stores four per-link fields every step
// (build_lattice_open_from_free_surface_periodic, CODEX.py:2492-2686:
// lattice_open, lattice_open_frac, lattice_wall_type, near_obstacle, 232 B
// per cell).  Here they are recomputed where they are needed from the 2-D
// bed height, the cube and the x walls; nothing is stored.  A cell whose
// every link endpoint is more than half a cell above the bed and outside
// the cube takes a fast path (all links open, fraction 1): the test is
// conservative, so the fast and full paths give identical results.
//
// Link endpoints x_c + c_q dx/2 take only three x and three y positions per
// cell, so the full path sets up the periodic bilinear interpolation once
// per axis position and evaluates the bed (and, when needed, the wall
// velocity) once per (x, y) endpoint: the same arithmetic as sampling link
// by link, with a ninth of the divisions.
#pragma once

#include "lbm_dev.cuh"

namespace lbm {

struct Geo {
    uint32_t lo;     // bit q set: lattice_open[q] == 1 (bit 0: the cell is open)
    uint32_t part;   // bit q set: lattice_open_frac[q] < 1
    bool near;       // near_obstacle
    bool fast;       // all links open with fraction 1 (links below not written)
};
// per-link fractions and wall sources, and the wall velocity at the nine
// link endpoints; written only for cells off the fast path (the fast path
// reads none of it)
struct GeoLinks {
    float lf[19];
    uint8_t wt[19];
    float uw[9][3];   // [3*(cx+1) + (cy+1)][component], valid when has_uw
    bool has_uw;
};
__host__ __device__ constexpr int endpoint_index(int q) { return 3 * (cxq(q) + 1) + (cyq(q) + 1); }

// one axis of the periodic bilinear sampling setup (CODEX.py:665-683,
// 2570-2588, 941-957): position -> (i0, i1, fraction)
LBM_DEV void bl_axis(float p, float dx, int n, int &i0, int &i1, float &f) {
    float L = (float)n * dx, Nf = (float)n;
    float w = p - floorf(p / L) * L;
    float u = w / dx - 0.5f;
    u = u - floorf(u / Nf) * Nf;
    i0 = (int)floorf(u);
    f = u - (float)i0;
    if (i0 >= n) i0 -= n;
    if (i0 < 0) i0 += n;
    i1 = (i0 + 1) % n;
}
LBM_DEV void bl_setup(const lbm_params &P, const Dom &D, float xp, float yp, int &i0, int &j0, int &i1, int &j1,
                      float &fx, float &fy) {
    bl_axis(xp, P.dx, D.nx, i0, i1, fx);
    bl_axis(yp, P.dx, D.ny, j0, j1, fy);
}
LBM_DEV float bl_sample(const float *a, const Dom &D, int i0, int j0, int i1, int j1, float fx, float fy) {
    float v00 = __ldg(a + D.col(j0, i0)), v10 = __ldg(a + D.col(j0, i1));
    float v01 = __ldg(a + D.col(j1, i0)), v11 = __ldg(a + D.col(j1, i1));
    float x0 = v00 * (1.0f - fx) + v10 * fx;
    float x1 = v01 * (1.0f - fx) + v11 * fx;
    return x0 * (1.0f - fy) + x1 * fy;
}
LBM_DEV float sample_h(const lbm_params &P, const Dom &D, const float *h, float xp, float yp) {
    int i0, j0, i1, j1;
    float fx, fy;
    bl_setup(P, D, xp, yp, i0, j0, i1, j1, fx, fy);
    return bl_sample(h, D, i0, j0, i1, j1, fx, fy);
}
// sample_wall_velocity_lb, CODEX.py:937-988
LBM_DEV void sample_wall(const lbm_params &P, const Dom &D, const BedView &B, float xp, float yp, float &wx,
                         float &wy, float &wz) {
    int i0, j0, i1, j1;
    float fx, fy;
    bl_setup(P, D, xp, yp, i0, j0, i1, j1, fx, fy);
    wx = bl_sample(B.uw, D, i0, j0, i1, j1, fx, fy);
    wy = bl_sample(B.vw, D, i0, j0, i1, j1, fx, fy);
    wz = bl_sample(B.ww, D, i0, j0, i1, j1, fx, fy);
}

// cube_sdf_at_point, CODEX.py:897-934
LBM_DEV float cube_sdf(const lbm_params &P, const Dom &D, float xp, float yp, float zp) {
    float Lx = (float)D.nx * P.dx, Ly = (float)D.ny * P.dx;
    float dxp = xp - P.cube_cx;
    float dyp = yp - P.cube_cy;
    if (!P.x_solid) {
        if (dxp > 0.5f * Lx) dxp -= Lx;
        if (dxp < -0.5f * Lx) dxp += Lx;
    }
    if (dyp > 0.5f * Ly) dyp -= Ly;
    if (dyp < -0.5f * Ly) dyp += Ly;
    float xl = P.cube_yaw_cos * dxp + P.cube_yaw_sin * dyp;
    float yl = -P.cube_yaw_sin * dxp + P.cube_yaw_cos * dyp;
    float z1 = zp - P.cube_cz;
    float xpitch = P.cube_pitch_cos * xl - P.cube_pitch_sin * z1;
    float zl = P.cube_pitch_sin * xl + P.cube_pitch_cos * z1;
    float qx = fabsf(xpitch) - P.cube_hx;
    float qy = fabsf(yl) - P.cube_hy;
    float qz = fabsf(zl) - P.cube_hz;
    float ox = fmaxf(qx, 0.0f), oy = fmaxf(qy, 0.0f), oz = fmaxf(qz, 0.0f);
    float outside = sqrtf(ox * ox + oy * oy + oz * oz);
    float inside = fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
    return outside + inside;
}

// compute_phi_slope_corrected for one cell, CODEX.py:2432-2490
LBM_DEV float phi_cell(const lbm_params &P, const Dom &D, const float *h, int k, int j, int i) {
    const float dx = P.dx;
    int ip = (i + 1) % D.nx, im = (i - 1 + D.nx) % D.nx, jp = (j + 1) % D.ny, jm = (j - 1 + D.ny) % D.ny;
    float dhdx = (__ldg(h + D.col(j, ip)) - __ldg(h + D.col(j, im))) * P.half_inv_dx;
    if (P.x_solid) {
        if (i == 0) dhdx = (__ldg(h + D.col(j, i + 1)) - __ldg(h + D.col(j, i))) / dx;
        else if (i == D.nx - 1) dhdx = (__ldg(h + D.col(j, i)) - __ldg(h + D.col(j, i - 1))) / dx;
    }
    float dhdy = (__ldg(h + D.col(jp, i)) - __ldg(h + D.col(jm, i))) * P.half_inv_dx;
    float denom = sqrtf(1.0f + dhdx * dhdx + dhdy * dhdy);
    if (denom < 1e-6f) denom = 1.0f;
    float hl = __ldg(h + D.col(j, i));
    float zc = ((float)k + 0.5f) * dx;
    float xc = ((float)i + 0.5f) * dx;
    float yc = ((float)j + 0.5f) * dx;
    float v = 1.0e6f;
    if (P.include_bed) v = (zc - hl) / denom;
    if (P.include_cube) {
        float cp = cube_sdf(P, D, xc, yc, zc);
        if (cp < v) v = cp;
    }
    if (P.x_solid) {
        float xw = fminf(xc, (float)D.nx * dx - xc);
        if (xw < v) v = xw;
    }
    return v;
}

// sample_phi_periodic, CODEX.py:661-707 (phi evaluated on the fly)
static __device__ __noinline__ float sample_phi(int slot, Dom D, const float *h, float xp, float yp, float zp) {
    const lbm_params &P = c_params[slot];
    int i0, j0, i1, j1;
    float fx, fy;
    bl_setup(P, D, xp, yp, i0, j0, i1, j1, fx, fy);
    float r = zp / P.dx - 0.5f;
    int k0 = (int)floorf(r);
    float fz = r - (float)k0;
    int k1 = k0 + 1;
    if (k0 < 0) { k0 = 0; k1 = 0; fz = 0.0f; }
    if (k1 >= D.nz) { k0 = D.nz - 1; k1 = D.nz - 1; fz = 0.0f; }
    float p00_0 = phi_cell(P, D, h, k0, j0, i0) * (1.0f - fx) + phi_cell(P, D, h, k0, j0, i1) * fx;
    float p01_0 = phi_cell(P, D, h, k0, j1, i0) * (1.0f - fx) + phi_cell(P, D, h, k0, j1, i1) * fx;
    float pxy_0 = p00_0 * (1.0f - fy) + p01_0 * fy;
    float p00_1 = phi_cell(P, D, h, k1, j0, i0) * (1.0f - fx) + phi_cell(P, D, h, k1, j0, i1) * fx;
    float p01_1 = phi_cell(P, D, h, k1, j1, i0) * (1.0f - fx) + phi_cell(P, D, h, k1, j1, i1) * fx;
    float pxy_1 = p00_1 * (1.0f - fy) + p01_1 * fy;
    return pxy_0 * (1.0f - fz) + pxy_1 * fz;
}

LBM_DEV bool geo_far_except_x(const lbm_params &P, const Dom &D, const BedView &B, int k, int j, int i);
// conservative "far from every wall" test
LBM_DEV bool geo_far(const lbm_params &P, const Dom &D, const BedView &B, int k, int j, int i) {
    if (P.x_solid && (i == 0 || i == D.nx - 1)) return false;
    return geo_far_except_x(P, D, B, k, j, i);
}
// the same test without the solid x walls: the cell may have links closed
// by an x wall, but none that meets the bed, the cube or phi geometry
LBM_DEV bool geo_far_except_x(const lbm_params &P, const Dom &D, const BedView &B, int k, int j, int i) {
    if (P.use_phi_open_fraction || P.use_phi_open_flags) return false;
    const float dx = P.dx, hdx = 0.5f * dx;
    float zc = ((float)k + 0.5f) * dx;
    if (P.include_bed) {
        float hm = __ldg(B.hmax + D.col(j, i));
        float margin = 1e-4f * dx + 1e-6f * (fabsf(zc) + fabsf(hm));
        if (!((zc - hdx) - hm >= hdx + margin)) return false;
    }
    if (P.include_cube) {
        float xc = ((float)i + 0.5f) * dx, yc = ((float)j + 0.5f) * dx;
        float Lx = (float)D.nx * dx, Ly = (float)D.ny * dx;
        float dxp = xc - P.cube_cx, dyp = yc - P.cube_cy;
        if (!P.x_solid) {
            if (dxp > 0.5f * Lx) dxp -= Lx;
            if (dxp < -0.5f * Lx) dxp += Lx;
            if (fabsf(dxp) > 0.5f * Lx - dx) return false;  // near the periodic seam
        }
        if (dyp > 0.5f * Ly) dyp -= Ly;
        if (dyp < -0.5f * Ly) dyp += Ly;
        if (fabsf(dyp) > 0.5f * Ly - dx) return false;
        float d = cube_sdf(P, D, xc, yc, zc);
        float margin = 1e-3f * dx + 1e-6f * (fabsf(xc) + fabsf(yc) + fabsf(zc));
        if (!(d >= 1.2072f * dx + margin)) return false;
    }
    return true;
}

// build_lattice_open_from_free_surface_periodic for one cell (full path);
// with want_uw, also the wall velocity at the nine link endpoints
static __device__ __noinline__ Geo geo_slow(int slot, Dom D, BedView B, int k, int j, int i, GeoLinks *L,
                                            bool want_uw) {
    const lbm_params &P = c_params[slot];
    Geo g;
    g.fast = false;
    const float dx = P.dx, hdx = 0.5f * dx;
    float xc = ((float)i + 0.5f) * dx, yc = ((float)j + 0.5f) * dx, zc = ((float)k + 0.5f) * dx;
    // bilinear setups of the three endpoint positions per axis
    int xi0[3], xi1[3], yj0[3], yj1[3];
    float xf[3], yf[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        bl_axis(xc + hdx * (float)(s - 1), dx, D.nx, xi0[s], xi1[s], xf[s]);
        bl_axis(yc + hdx * (float)(s - 1), dx, D.ny, yj0[s], yj1[s], yf[s]);
    }
    float eta9[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            eta9[3 * a + b] = bl_sample(B.h, D, xi0[a], yj0[b], xi1[a], yj1[b], xf[a], yf[b]);
    L->has_uw = want_uw;
    if (want_uw) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                L->uw[3 * a + b][0] = bl_sample(B.uw, D, xi0[a], yj0[b], xi1[a], yj1[b], xf[a], yf[b]);
                L->uw[3 * a + b][1] = bl_sample(B.vw, D, xi0[a], yj0[b], xi1[a], yj1[b], xf[a], yf[b]);
                L->uw[3 * a + b][2] = bl_sample(B.ww, D, xi0[a], yj0[b], xi1[a], yj1[b], xf[a], yf[b]);
            }
    }
    float eta_c = eta9[4];
    float gap_c = zc - eta_c;
    float ggc = 1.0e6f;
    int wtc = LBM_WALL_NONE;
    if (P.include_bed) { ggc = gap_c; wtc = LBM_WALL_BED; }
    if (P.include_cube) {
        float cg = cube_sdf(P, D, xc, yc, zc);
        if (cg < ggc) { ggc = cg; wtc = LBM_WALL_CUBE; }
    }
    float sgc = ggc;
    if (P.use_phi_open_fraction) sgc = phi_cell(P, D, B.h, k, j, i);
    float frc = 0.5f + sgc / dx;
    if (frc < 0.0f) frc = 0.0f;
    if (frc > 1.0f) frc = 1.0f;
    L->lf[0] = frc;
    L->wt[0] = (uint8_t)wtc;
    uint32_t lo = 0u;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        float xq = xc + hdx * (float)cxq(q);
        float yq = yc + hdx * (float)cyq(q);
        float zq = zc + hdx * (float)czq(q);
        float eta = eta9[endpoint_index(q)];
        float gap = zq - eta;
        float gg = 1.0e6f;
        int wq_ = LBM_WALL_NONE;
        if (P.include_bed) { gg = gap; wq_ = LBM_WALL_BED; }
        if (P.include_cube) {
            float cg = cube_sdf(P, D, xq, yq, zq);
            if (cg < gg) { gg = cg; wq_ = LBM_WALL_CUBE; }
        }
        float sg = gg;
        if (P.use_phi_open_fraction) sg = sample_phi(slot, D, B.h, xq, yq, zq);
        float fr = 0.5f + sg / dx;
        if (fr < 0.0f) fr = 0.0f;
        if (fr > 1.0f) fr = 1.0f;
        float og = P.use_phi_open_flags ? sg : gg;
        bool open = !(og < 0.0f);
        if (P.x_solid) {
            if (i == 0 && cxq(q) > 0) { open = false; fr = 0.0f; wq_ = LBM_WALL_XMIN; }
            else if (i == D.nx - 1 && cxq(q) < 0) { open = false; fr = 0.0f; wq_ = LBM_WALL_XMAX; }
        }
        L->lf[q] = fr;
        L->wt[q] = (uint8_t)wq_;
        if (open) lo |= (1u << q);
    }
    if (lo) lo |= 1u;
    g.near = (lo & 0x7FFFEu) != 0x7FFFEu;
    if (!(lo & 1u)) {
        for (int q = 1; q < 19; ++q) L->lf[q] = 0.0f;
    }
    uint32_t part = 0u;
    for (int q = 0; q < 19; ++q)
        if (L->lf[q] < 1.0f) part |= (1u << q);
    g.part = part;
    g.lo = lo;
    return g;
}

// Per-column cache of the bed at the link endpoints.  With bed-only
// geometry (no cube, no phi geometry, periodic x) a cell's link endpoints
// sit at nine (x, y) positions that do not depend on k, so the bed height
// and wall velocity there are sampled once per column per bed state, with
// the arithmetic of the per-link path.  Layout [component][column]:
// 0..8 bed height at endpoint e = endpoint_index(q), 9..35 wall velocity
// (e, component), 36 slope denominator of compute_phi_slope_corrected.
LBM_DEV void colgeo_column(const lbm_params &P, const Dom &D, const BedView &B, int j, int i, float *cg) {
    const float dx = P.dx, hdx = 0.5f * dx;
    const size_t A = D.a;
    const int a = D.col(j, i);
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
        for (int yb = 0; yb < 3; ++yb) {
            const int e = 3 * xa + yb;
            cg[(size_t)(CG_ETA + e) * A + a] = bl_sample(B.h, D, xi0[xa], yj0[yb], xi1[xa], yj1[yb], xf[xa], yf[yb]);
            cg[(size_t)(CG_UW + 3 * e) * A + a] = bl_sample(B.uw, D, xi0[xa], yj0[yb], xi1[xa], yj1[yb], xf[xa], yf[yb]);
            cg[(size_t)(CG_UW + 3 * e + 1) * A + a] =
                bl_sample(B.vw, D, xi0[xa], yj0[yb], xi1[xa], yj1[yb], xf[xa], yf[yb]);
            cg[(size_t)(CG_UW + 3 * e + 2) * A + a] =
                bl_sample(B.ww, D, xi0[xa], yj0[yb], xi1[xa], yj1[yb], xf[xa], yf[yb]);
        }
    // slope denominator of phi_cell (periodic x)
    int ip = (i + 1) % D.nx, im = (i - 1 + D.nx) % D.nx, jp = (j + 1) % D.ny, jm = (j - 1 + D.ny) % D.ny;
    float dhdx = (__ldg(B.h + D.col(j, ip)) - __ldg(B.h + D.col(j, im))) * P.half_inv_dx;
    float dhdy = (__ldg(B.h + D.col(jp, i)) - __ldg(B.h + D.col(jm, i))) * P.half_inv_dx;
    float denom = sqrtf(1.0f + dhdx * dhdx + dhdy * dhdy);
    if (denom < 1e-6f) denom = 1.0f;
    cg[(size_t)CG_DEN * A + a] = denom;
}

// geo_slow for bed-only geometry from the column cache (same arithmetic)
LBM_DEV Geo geo_cached(const lbm_params &P, const Dom &D, const BedView &B, int k, int j, int i, GeoLinks &L) {
    const size_t A = D.a;
    const int a = D.col(j, i);
    const float dx = P.dx, hdx = 0.5f * dx;
    float zc = ((float)k + 0.5f) * dx;
    float eta9[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) eta9[e] = __ldg(B.cg + (size_t)(CG_ETA + e) * A + a);
    Geo g;
    g.fast = false;
    const int wtb = P.include_bed ? LBM_WALL_BED : LBM_WALL_NONE;
    float ggc = P.include_bed ? zc - eta9[4] : 1.0e6f;
    float frc = 0.5f + ggc / dx;
    if (frc < 0.0f) frc = 0.0f;
    if (frc > 1.0f) frc = 1.0f;
    L.lf[0] = frc;
    L.wt[0] = (uint8_t)wtb;
    uint32_t lo = 0u;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        float zq = zc + hdx * (float)czq(q);
        float gg = P.include_bed ? zq - eta9[endpoint_index(q)] : 1.0e6f;
        float fr = 0.5f + gg / dx;
        if (fr < 0.0f) fr = 0.0f;
        if (fr > 1.0f) fr = 1.0f;
        L.lf[q] = fr;
        L.wt[q] = (uint8_t)wtb;
        if (!(gg < 0.0f)) lo |= (1u << q);
    }
    if (lo) lo |= 1u;
    g.near = (lo & 0x7FFFEu) != 0x7FFFEu;
    uint32_t part = 0u;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (q > 0 && !(lo & 1u)) L.lf[q] = 0.0f;
        if (L.lf[q] < 1.0f) part |= (1u << q);
    }
    g.part = part;
    g.lo = lo;
    L.has_uw = false;
    return g;
}
// wall velocity at endpoint e from the column cache
LBM_DEV void cached_wall(const Dom &D, const BedView &B, int j, int i, int e, float &wx, float &wy, float &wz) {
    const size_t A = D.a;
    const int a = D.col(j, i);
    wx = __ldg(B.cg + (size_t)(CG_UW + 3 * e) * A + a);
    wy = __ldg(B.cg + (size_t)(CG_UW + 3 * e + 1) * A + a);
    wz = __ldg(B.cg + (size_t)(CG_UW + 3 * e + 2) * A + a);
}

// CG: the bed view carries the column cache (bed-only geometry); the link
// data then never goes through an out-of-line call
template <bool CG = false>
LBM_DEV Geo geo_cell(const lbm_params &P, int slot, const Dom &D, const BedView &B, int k, int j, int i, GeoLinks &L,
                     bool allow_fast = true, bool want_uw = false) {
    if (allow_fast && geo_far(P, D, B, k, j, i)) {
        Geo g;
        g.lo = 0x7FFFFu;
        g.part = 0u;
        g.near = false;
        g.fast = true;
        return g;
    }
    if (CG) return geo_cached(P, D, B, k, j, i, L);
    return geo_slow(slot, D, B, k, j, i, &L, want_uw);
}

static __device__ __noinline__ bool cell_open_slow(int slot, Dom D, BedView B, int k, int j, int i) {
    GeoLinks L;
    if (B.cg) return (geo_cached(c_params[slot], D, B, k, j, i, L).lo & 1u) != 0u;
    return (geo_slow(slot, D, B, k, j, i, &L, false).lo & 1u) != 0u;
}
// lattice_open[0] only (cheap when far from walls)
LBM_DEV bool cell_open(const lbm_params &P, int slot, const Dom &D, const BedView &B, int k, int j, int i) {
    // a solid x wall closes links of the cells next to it, not the cells
    if (geo_far_except_x(P, D, B, k, j, i)) return true;
    return cell_open_slow(slot, D, B, k, j, i);
}

}  // namespace lbm
