// lbm_stages.cuh - per-cell stages of the D3Q19 step, shared by the kernels.
//
//   stream_fast   pull gather of an interior cell far from every wall
//   stream_bc     stream() + apply_x_solid_wall_bounceback() +
//                 apply_open_boundary_conditions()      CODEX.py:3418-3712
//   condition     update_bed_populations_and_reinit()   CODEX.py:2878-2940
//   macro         macro_step()                          CODEX.py:2943-3008
//   les_omega     compute_LES()                         CODEX.py:3011-3141
//   collide       collide_KBC() / collide_regularized() CODEX.py:3143-3416
//
// Inlined stages read the solver constants from the kernel argument copy
// (A.P: constant-bank operands); out-of-line near-wall helpers read the
// same constants from c_params[A.slot].
#pragma once

#include "lbm_geom.cuh"
#include "lbm_launch.h"

namespace lbm {

// --------------------------------------------------------- free surface
LBM_DEV void classify_height(const lbm_params &P, float h, int k, bool open, int &type, float &fill) {
    float zb = (float)k * P.dx;
    float fl = (h - zb) / P.dx;
    if (fl < 0.0f) fl = 0.0f;
    if (fl > 1.0f) fl = 1.0f;
    int ct;
    if (fl <= 1e-4f) ct = LBM_FS_GAS;
    else if (fl >= (float)(1.0 - 1e-4)) ct = LBM_FS_LIQUID;
    else ct = LBM_FS_INTERFACE;
    if (!open) { fl = 0.0f; ct = LBM_FS_GAS; }
    type = ct;
    fill = fl;
}

// free-surface state of a cell at the start of the step
LBM_DEV void fs_state(const StepArgs &A, int c, int k, int j, int i, bool open, int &type, float &fill) {
    if (A.flags & F_VOF_STATE) {
        type = A.fs_type[c];
        fill = A.fs_fill[c];
    } else {
        classify_height(A.P, __ldg(A.fs_h + A.D.col(j, i)), k, open, type, fill);
    }
}

// gravity_body_fraction (update_pressure_reference_fields, CODEX.py:710-740)
LBM_DEV float gbf_of(const lbm_params &P, int k, bool open, int type) {
    if (!(P.fs_mode != LBM_FS_NONE && open && type != LBM_FS_GAS)) return 0.0f;
    if (P.pressure_formulation == LBM_PRESSURE_HYDROSTATIC_BALANCED) return 0.0f;
    if (P.pressure_formulation == LBM_PRESSURE_VOF_COMPONENT_BALANCED) {
        float zc = ((float)k + 0.5f) * P.dx;
        return zc < P.fs_base_m ? 0.0f : 1.0f;
    }
    return 1.0f;
}
LBM_DEV float prh_of(const lbm_params &P, int k, bool open, int type) {
    if (!(P.fs_mode != LBM_FS_NONE && open && type != LBM_FS_GAS)) return 0.0f;
    float zc = ((float)k + 0.5f) * P.dx;
    if (P.pressure_formulation == LBM_PRESSURE_HYDROSTATIC_BALANCED) return P.fs_base_m - zc;
    if (P.pressure_formulation == LBM_PRESSURE_VOF_COMPONENT_BALANCED) return zc < P.fs_base_m ? P.fs_base_m - zc : 0.0f;
    return 0.0f;
}
// local_g_body_lb, CODEX.py:646-651
LBM_DEV float g_local(const lbm_params &P, float gbf) {
    return P.use_component_balanced_pressure ? P.g_lb * gbf : P.g_body_lb;
}
// free_surface_hydrostatic_density_at_cell, CODEX.py:821-845
LBM_DEV float fs_density_cell(const lbm_params &P, float h_col, int k, float gbf) {
    float head = 0.0f;
    if (P.use_component_balanced_pressure) {
        float zc = ((float)k + 0.5f) * P.dx;
        head = gbf < 0.5f ? zc - P.fs_base_m : 0.0f;
    } else if (P.use_hydrostatic_balanced_pressure) {
        head = h_col - P.fs_base_m;
    } else {
        float zc = ((float)k + 0.5f) * P.dx;
        head = h_col - zc;
    }
    if (head < 0.0f && !P.use_hydrostatic_balanced_pressure) head = 0.0f;
    return P.rho0 + P.g_lb * (head / P.dx) / P.one_third;
}
// free_surface_pressure_density_at_link, CODEX.py:848-867
LBM_DEV float fs_density_link(const lbm_params &P, float h_col, int k, int cz, float gbf) {
    if (P.use_component_balanced_pressure) {
        float zi = ((float)k + 0.5f) * P.dx - 0.5f * (float)cz * P.dx;
        float head = 0.0f;
        if (gbf < 0.5f) head += zi - P.fs_base_m;
        return P.rho0 + P.g_lb * (head / P.dx) / P.one_third;
    }
    if (P.use_hydrostatic_balanced_pressure && P.fs_tracking == LBM_TRACK_VOF) {
        float zi = ((float)k + 0.5f) * P.dx - 0.5f * (float)cz * P.dx;
        float head = zi - P.fs_base_m;
        return P.rho0 + P.g_lb * (head / P.dx) / P.one_third;
    }
    return fs_density_cell(P, h_col, k, gbf);
}

LBM_DEV float smooth01(float x) { return x * x * (3.0f - 2.0f * x); }

// ------------------------------------------------------------ fast path
// A cell takes the fast path when every stage is the plain interior one:
// all links open with fraction 1 (far from the bed and the cube, for both
// geometries the pass spans), no out-of-domain source, no x wall, no x
// fringe, no top drive, no free surface.
LBM_DEV bool cell_fast(const StepArgs &A, bool check_s, bool check_c, int k, int j, int i) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    if (P.fs_mode != LBM_FS_NONE) return false;
    if (k < 1 || k > D.nz - 2) return false;
    if (P.x_solid && (i == 0 || i == D.nx - 1)) return false;
    if (P.enable_x_fringe && i < 5 && k > D.nz / 2) return false;
    if (check_s && !geo_far(P, D, A.bed_s, k, j, i)) return false;
    if (check_c && !geo_far(P, D, A.bed_c, k, j, i)) return false;
    return true;
}

// pull gather of an interior cell: f(x - c_q)[q], periodic in x and y
template <int S>
LBM_DEV void stream_fast(const StepArgs &A, const typename Store<S>::T *__restrict__ fs, int k, int j, int i,
                         int c, float out[19]) {
    const Dom &D = A.D;
    const size_t n = D.n;
    const int nxy = D.nx * D.ny;
    const int xp = (i + 1 == D.nx) ? 1 - D.nx : 1;   // offset to the +x neighbour
    const int xm = (i == 0) ? D.nx - 1 : -1;
    const int yp = (j + 1 == D.ny) ? (1 - D.ny) * D.nx : D.nx;
    const int ym = (j == 0) ? (D.ny - 1) * D.nx : -D.nx;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        // source = x - c_q
        int s = c;
        if (cxq(q) > 0) s += xm; else if (cxq(q) < 0) s += xp;
        if (cyq(q) > 0) s += ym; else if (cyq(q) < 0) s += yp;
        if (czq(q) > 0) s -= nxy; else if (czq(q) < 0) s += nxy;
        out[q] = Store<S>::ld(fs, (size_t)q * n + (size_t)s, q, A.P.rho0);
    }
}

// ------------------------------------------------------------ stream + BC
// post-stream populations of cell (k,j,i) from post-collision fs[]
// AIR: compiled for air mode only (no free-surface code in the kernel)
template <int S, bool AIR = false>
LBM_DEV void stream_bc(const StepArgs &A, const typename Store<S>::T *__restrict__ fs, const Geo &g,
                       const GeoLinks &L, int k, int j, int i, int c, float out[19], int &cut, int &fscut,
                       int &bridge) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const size_t n = D.n;
    const bool water = !AIR && P.fs_mode != LBM_FS_NONE;
    const bool vof = water && P.fs_tracking == LBM_TRACK_VOF;
    const float rho0 = P.rho0;
    const bool open_c = (g.lo & 1u) != 0u;
    int type_c = LBM_FS_LIQUID;
    float fill_c = 1.0f;
    bool dest_gas = false;
    float gbf_c = 0.0f, hcol = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
    if (water) {
        fs_state(A, c, k, j, i, open_c, type_c, fill_c);
        dest_gas = type_c == LBM_FS_GAS && open_c;
        gbf_c = gbf_of(P, k, open_c, type_c);
        hcol = __ldg(A.fs_h + D.col(j, i));
        vx = A.ux[c]; vy = A.uy[c]; vz = A.uz[c];
    }
#define LDS(q, cell) Store<S>::ld(fs, (size_t)(q) * n + (size_t)(cell), (q), rho0)
    out[0] = dest_gas ? feq<0>(rho0, 0.0f, 0.0f, 0.0f, 0.0f) : LDS(0, c);
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const int cx = cxq(q), cy = cyq(q), cz = czq(q), qb = oppq(q);
        int sir = i - cx;
        int si = sir;
        bool sf = true;
        if (!P.x_solid) si = sir < 0 ? sir + D.nx : (sir >= D.nx ? sir - D.nx : sir);
        else if (sir < 0) { si = 0; sf = false; }
        else if (sir >= D.nx) { si = D.nx - 1; sf = false; }
        int sj = j - cy;
        sj = sj < 0 ? sj + D.ny : (sj >= D.ny ? sj - D.ny : sj);
        int sk = k - cz;
        const float fr = (g.part & (1u << q)) ? L.lf[q] : 1.0f;
        float v;
        if (water) {
            bool src_gas = false;
            int s = 0;
            if (sf && sk >= 0 && sk < D.nz) {
                s = D.cell(sk, sj, si);
                int ts;
                float fls;
                if (A.flags & F_VOF_STATE) {
                    ts = A.fs_type[s];
                    if (ts == LBM_FS_GAS) src_gas = cell_open(P, A.slot, D, A.bed_s, sk, sj, si);
                } else {
                    classify_height(P, __ldg(A.fs_h + D.col(sj, si)), sk, true, ts, fls);
                    if (ts == LBM_FS_GAS) src_gas = cell_open(P, A.slot, D, A.bed_s, sk, sj, si);
                }
            } else if (sk >= D.nz) {
                src_gas = true;
            }
            if (dest_gas) {
                // calculate_feq(rho0, 0, 0, 0, q) = (rho0 * w_q) * 1
                v = rho0 * wq(q) * 1.0f;
            } else if (!sf) {
                v = LDS(qb, c);
                cut++;
            } else if (sk >= 0 && sk < D.nz && !src_gas) {
                float fst;
                if (fr < 1.0f) fst = fr * LDS(q, s) + (1.0f - fr) * LDS(qb, c);
                else fst = LDS(q, s);
                float o = fst;
                if (vof && P.vof_link_aperture) {
                    // vof_link_liquid_aperture of the source, CODEX.py:870-894
                    float la = 1.0f;
                    int ts = A.fs_type[s];
                    if (ts != LBM_FS_LIQUID && cell_open(P, A.slot, D, A.bed_s, sk, sj, si)) {
                        if (ts == LBM_FS_GAS) la = 0.0f;
                        else if (ts == LBM_FS_INTERFACE) {
                            la = A.fs_fill[s];
                            if (la < 0.0f) la = 0.0f;
                            if (la > 1.0f) la = 1.0f;
                        }
                    }
                    if (la < 1.0f) {
                        float rfs = rho0;
                        if (P.use_hydrostatic_balanced_pressure || P.fs_boundary == LBM_FSB_HYDROSTATIC)
                            rfs = fs_density_link(P, hcol, k, cz, gbf_c);
                        float u2 = usq(vx, vy, vz);
                        float ffs = 0.0f;
                        switch (q) {
#define FQ(Q) case Q: ffs = feq<Q>(rfs, vx, vy, vz, u2) + feq<oppq(Q)>(rfs, vx, vy, vz, u2) - LDS(oppq(Q), c); break;
                            FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                            FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                        }
                        o = la * fst + (1.0f - la) * ffs;
                        fscut++;
                    }
                }
                v = o;
                if (fr < 1.0f) cut++;
            } else if (sk < 0) {
                v = LDS(qb, c);
                cut++;
            } else {
                float rfs = rho0;
                if (P.use_hydrostatic_balanced_pressure || P.fs_boundary == LBM_FSB_HYDROSTATIC)
                    rfs = fs_density_link(P, hcol, k, cz, gbf_c);
                float u2 = usq(vx, vy, vz);
                float ffs = 0.0f;
                switch (q) {
#define FQ(Q) case Q: ffs = feq<Q>(rfs, vx, vy, vz, u2) + feq<oppq(Q)>(rfs, vx, vy, vz, u2) - LDS(oppq(Q), c); break;
                    FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                    FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                }
                float o = ffs;
                if (vof && P.vof_thin_gap_bridge && sk >= 0 && sk < D.nz && src_gas) {
                    int bir = si - cx;
                    int bi = bir;
                    int bj = pymod(sj - cy + D.ny, D.ny);
                    int bk = sk - cz;
                    bool bv = true;
                    if (!P.x_solid) bi = pymod(bir + D.nx, D.nx);
                    else if (bir < 0 || bir >= D.nx) bv = false;
                    if (bk < 0 || bk >= D.nz) bv = false;
                    if (bv) {
                        int bc = D.cell(bk, bj, bi);
                        if (A.fs_type[bc] != LBM_FS_GAS && cell_open(P, A.slot, D, A.bed_s, bk, bj, bi)) {
                            float bw = fill_c;
                            float fb = A.fs_fill[bc];
                            if (fb < bw) bw = fb;
                            bw *= P.vof_thin_gap_bridge_strength;
                            if (bw > 0.0f) {
                                if (bw > 1.0f) bw = 1.0f;
                                o = (1.0f - bw) * ffs + bw * LDS(q, bc);
                                bridge++;
                            }
                        }
                    }
                }
                v = o;
                fscut++;
            }
        } else {
            if (!sf) {
                v = LDS(qb, c);
                cut++;
            } else if (sk >= 0 && sk < D.nz) {
                int s = D.cell(sk, sj, si);
                if (fr < 1.0f) {
                    v = fr * LDS(q, s) + (1.0f - fr) * LDS(qb, c);
                    cut++;
                } else {
                    v = LDS(q, s);
                }
            } else if (P.top_free_slip && sk >= D.nz) {
                // specular wall above the top row (extension)
                v = LDS(mirzq(q), D.cell(D.nz - 1, sj, si));
            } else {
                v = LDS(q, c);
            }
        }
        out[q] = v;
    }
    // apply_x_solid_wall_bounceback, CODEX.py:3554-3580
    if (P.x_solid && (i == 0 || i == D.nx - 1)) {
        bool active = !(water && dest_gas);
        if (active) {
#pragma unroll
            for (int q = 1; q < 19; ++q) {
                if ((i == 0 && cxq(q) > 0) || (i == D.nx - 1 && cxq(q) < 0)) out[q] = LDS(oppq(q), c);
            }
        }
    }
    // (A) x-fringe, CODEX.py:3616-3645
    if (P.enable_x_fringe && i < 5 && open_c && k > D.nz / 2) {
        float s_ = 1.0f - (float)i / 4.0f;
        float kr = (float)k / (float)(D.nz - 1);
        float strength = 0.05f * (kr * kr - 0.25f);
        float sigma = strength * smooth01(s_);
        float uxt = __ldg(A.u_inlet_profile + k) + 0.0f;
        float u2 = usq(uxt, 0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float ft = 0.0f;
            switch (q) {
#define FQ(Q) case Q: ft = feq<Q>(rho0, uxt, 0.0f, 0.0f, u2); break;
                FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
            }
            out[q] = (1.0f - sigma) * out[q] + sigma * ft;
        }
    }
    // (B) top drive, CODEX.py:3651-3663
    if (P.enable_top_drive && k == D.nz - 1 && open_c) {
        float ut = P.u_top_lb;
        float u2 = usq(ut, 0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            switch (q) {
#define FQ(Q) case Q: out[q] = feq<Q>(rho0, ut, 0.0f, 0.0f, u2); break;
                FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
            }
        }
    }
    // (C) moving-wall IBB on near-obstacle cells, CODEX.py:3674-3712
    if (g.near) {
        const float hdx = 0.5f * P.dx;
        float xc = ((float)i + 0.5f) * P.dx, yc = ((float)j + 0.5f) * P.dx;
        const BedView &B = A.bed_s;
#pragma unroll
        for (int q = 1; q < 19; ++q) {
            if (!(g.part & (1u << q))) continue;   // fraction 1: identity
            const int qb = oppq(q);
            float fo = L.lf[q];
            float wx = 0.0f, wy = 0.0f, wz = 0.0f;
            if (L.wt[q] == LBM_WALL_BED) {
                int a = D.col(j, i);
                wx = __ldg(B.uw + a); wy = __ldg(B.vw + a); wz = __ldg(B.ww + a);
                if (P.use_link_wall_velocity) {
                    if (L.has_uw) {
                        const int e = endpoint_index(q);
                        wx = L.uw[e][0]; wy = L.uw[e][1]; wz = L.uw[e][2];
                    } else if (B.cg) {
                        cached_wall(D, B, j, i, endpoint_index(q), wx, wy, wz);
                    } else {
                        sample_wall(P, D, B, xc + hdx * (float)cxq(q), yc + hdx * (float)cyq(q), wx, wy, wz);
                    }
                }
            }
            float cuw = (float)cxq(qb) * wx + (float)cyq(qb) * wy + (float)czq(qb) * wz;
            float fwall = LDS(qb, c) - 6.0f * wq(qb) * rho0 * cuw;
            out[q] = out[q] * fo + fwall * (1.0f - fo);
        }
    }
#undef LDS
}

// ---------------------------------------------------- pre-collision stages
// update_bed_populations_and_reinit for one cell (geometry of the collide step)
LBM_DEV void condition(const lbm_params &P, const Dom &D, const BedView &B, const Geo &g, const GeoLinks &L, int k,
                       int j, int i, float f[19]) {
    if (g.fast || (g.lo == 0x7FFFFu)) return;   // no closed link
    const bool moving = P.bed_profile == LBM_BED_MOVING_SINE;
    const float hdx = 0.5f * P.dx;
    int a = D.col(j, i);
    float ux_ = __ldg(B.uw + a), uy_ = __ldg(B.vw + a), uz_ = __ldg(B.ww + a);
    float xc = ((float)i + 0.5f) * P.dx, yc = ((float)j + 0.5f) * P.dx;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (g.lo & (1u << q)) continue;
        float fr = L.lf[q];
        int wt = L.wt[q];
        bool apply = false;
        float vx = 0.0f, vy = 0.0f, vz = 0.0f;
        if (wt == LBM_WALL_BED && moving) {
            apply = true;
            vx = ux_; vy = uy_; vz = uz_;
        } else if (!P.physics_water) {
            apply = true;
            if (wt == LBM_WALL_BED) { vx = ux_; vy = uy_; vz = uz_; }
        }
        if (!apply) continue;
        if (wt == LBM_WALL_BED && P.use_link_wall_velocity) {
            if (L.has_uw) {
                const int e = endpoint_index(q);
                vx = L.uw[e][0]; vy = L.uw[e][1]; vz = L.uw[e][2];
            } else if (B.cg) {
                cached_wall(D, B, j, i, endpoint_index(q), vx, vy, vz);
            } else {
                sample_wall(P, D, B, xc + hdx * (float)cxq(q), yc + hdx * (float)cyq(q), vx, vy, vz);
            }
        }
        float u2 = usq(vx, vy, vz);
        float fe = 0.0f;
        switch (q) {
#define FQ(Q) case Q: fe = feq<Q>(P.rho0, vx, vy, vz, u2); break;
            FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
            FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
        }
        f[q] = fr * f[q] + (1.0f - fr) * fe;
    }
}

// macro_step for one cell; returns rho, u (gas/Guo/top-drive rules)
LBM_DEV void macro(const lbm_params &P, const Dom &D, const float f[19], int k, bool water, int type, float gbf,
                   float &r, float &vx, float &vy, float &vz) {
    float rr = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) rr += f[q];
    float jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (cxq(q) > 0) jx += f[q]; else if (cxq(q) < 0) jx += -f[q];
        if (cyq(q) > 0) jy += f[q]; else if (cyq(q) < 0) jy += -f[q];
        if (czq(q) > 0) jz += f[q]; else if (czq(q) < 0) jz += -f[q];
    }
    r = rr;
    if (water) {
        if (type == LBM_FS_GAS) {
            r = P.rho0; vx = 0.0f; vy = 0.0f; vz = 0.0f;
        } else {
            float fz = -rr * g_local(P, gbf);
            float inv = 1.0f / rr;
            vx = jx * inv;
            vy = jy * inv;
            vz = (jz + 0.5f * fz) * inv;
        }
    } else {
        float inv = 1.0f / rr;
        vx = jx * inv;
        vy = jy * inv;
        vz = jz * inv;
    }
    if (P.enable_top_drive && k == D.nz - 1) {
        vx = P.u_top_lb; vy = 0.0f; vz = 0.0f;
    }
}

// log-law wall model of compute_LES (CODEX.py:3097-3129), applied when the
// cell below is solid; out of line because it runs only next to the bed
static __device__ __noinline__ float wall_model_nu(int slot, Dom D, BedView bed, int k, int j, int i, float vx,
                                                   float vy, float nu_t) {
    const lbm_params &P = c_params[slot];
    GeoLinks Lb;
    float phi;
    if (bed.cg) {
        Geo gb = geo_cached(P, D, bed, k - 1, j, i, Lb);
        if (gb.lo & 1u) return nu_t;
        // phi_cell with bed-only geometry
        phi = 1.0e6f;
        if (P.include_bed)
            phi = (((float)k + 0.5f) * P.dx - __ldg(bed.h + D.col(j, i))) /
                  __ldg(bed.cg + (size_t)CG_DEN * D.a + D.col(j, i));
    } else {
        Geo gb = geo_slow(slot, D, bed, k - 1, j, i, &Lb, false);
        if (gb.lo & 1u) return nu_t;
        phi = phi_cell(P, D, bed.h, k, j, i);
    }
    float dist = fmaxf(phi, P.wall_dist_floor);
    float lv = lbm_logf(dist / P.z0_phys);
    if (lv < 2.0f) lv = 2.0f;
    float uwx = 0.0f, uwy = 0.0f;
    if (Lb.wt[0] == LBM_WALL_BED) {
        uwx = __ldg(bed.uw + D.col(j, i));
        uwy = __ldg(bed.vw + D.col(j, i));
    }
    float rx = vx - uwx, ry = vy - uwy;
    float sp = sqrtf(rx * rx + ry * ry);
    if (sp > 1e-6f) {
        float ut = sp * P.kappa / lv;
        float tw = ut * ut;
        float sa = sp / 0.5f;
        float nwm = tw / sa;
        float ntw = nwm - P.nu0;
        if (ntw < 0.0f) ntw = 0.0f;
        nu_t = fmaxf(nu_t, ntw);
    }
    return nu_t;
}

// Smagorinsky relaxation rate from the strain of a velocity stencil
// (compute_LES, CODEX.py:3038-3140); u_* are the 6 face neighbours
LBM_DEV float les_from_stencil(const StepArgs &A, int k, int j, int i, float vx, float vy, float uxp, float uxm,
                               float uyp, float uym, float uzp, float uzm, float vxp, float vxm, float vyp, float vym,
                               float vzp, float vzm, float wxp, float wxm, float wyp, float wym, float wzp,
                               float wzm) {
    const lbm_params &P = A.P;
    float du_dx = 0.5f * (uxp - uxm);
    float du_dy = 0.5f * (uyp - uym);
    float du_dz = 0.5f * (uzp - uzm);
    float dv_dx = 0.5f * (vxp - vxm);
    float dv_dy = 0.5f * (vyp - vym);
    float dv_dz = 0.5f * (vzp - vzm);
    float dw_dx = 0.5f * (wxp - wxm);
    float dw_dy = 0.5f * (wyp - wym);
    float dw_dz = 0.5f * (wzp - wzm);
    float Sxx = du_dx, Syy = dv_dy, Szz = dw_dz;
    float Sxy = 0.5f * (du_dy + dv_dx);
    float Sxz = 0.5f * (du_dz + dw_dx);
    float Syz = 0.5f * (dv_dz + dw_dy);
    float Sc = (Sxx * Sxx + Syy * Syy + Szz * Szz + 2.0f * (Sxy * Sxy + Sxz * Sxz + Syz * Syz));
    float Smag = sqrtf(2.0f * Sc + 1e-6f);
    float nu_t = P.cs_delta_sq * Smag;
    if (nu_t > P.nu_t_max) nu_t = P.nu_t_max;
    if (k > 0 && !geo_far(P, A.D, A.bed_c, k - 1, j, i)) nu_t = wall_model_nu(A.slot, A.D, A.bed_c, k, j, i, vx, vy, nu_t);
    float nu_eff = P.nu0 + nu_t;
    float tau_eff = 0.5f + 3.0f * nu_eff;
    if (tau_eff > 2.0f) tau_eff = 2.0f;
    return 1.0f / tau_eff;
}

// compute_LES for one active cell from the pre-pass velocity buffer
LBM_DEV float les_omega(const StepArgs &A, int k, int j, int i, int c, float vx, float vy, float vz) {
    const Dom &D = A.D;
    const size_t n = D.n;
    int ip = i + 1 == D.nx ? 0 : i + 1, im = i == 0 ? D.nx - 1 : i - 1;
    int jp = j + 1 == D.ny ? 0 : j + 1, jm = j == 0 ? D.ny - 1 : j - 1;
    int kp = k + 1 >= D.nz ? D.nz - 1 : k + 1, km = k - 1 < 0 ? 0 : k - 1;
    const float *U = A.u_les, *V = A.u_les + n, *W = A.u_les + 2 * n;
    int cxp = D.cell(k, j, ip), cxm = D.cell(k, j, im), cyp = D.cell(k, jp, i), cym = D.cell(k, jm, i);
    int czp = D.cell(kp, j, i), czm = D.cell(km, j, i);
    return les_from_stencil(A, k, j, i, vx, vy, __ldg(U + cxp), __ldg(U + cxm), __ldg(U + cyp), __ldg(U + cym),
                            __ldg(U + czp), __ldg(U + czm), __ldg(V + cxp), __ldg(V + cxm), __ldg(V + cyp),
                            __ldg(V + cym), __ldg(V + czp), __ldg(V + czm), __ldg(W + cxp), __ldg(W + cxm),
                            __ldg(W + cyp), __ldg(W + cym), __ldg(W + czp), __ldg(W + czm));
}

// Guo forcing term (CODEX.py:3223-3232, 3389-3396)
template <int Q>
LBM_DEV float guo(float om, float vx, float vy, float vz, float fz) {
    const float cs2 = LBM_CS2;
    float czi = (float)czq(Q);
    float cdu = cdot<Q>(vx, vy, vz);
    return wq(Q) * (1.0f - 0.5f * om) * (((czi - vz) / cs2) + (cdu * czi / (cs2 * cs2))) * fz;
}

// second-moment tensor of a population deviation, terms with a zero
// lattice component skipped (each adds +-0 in the reference's order)
LBM_DEV void second_moments(const float d[19], float &Pxx, float &Pyy, float &Pzz, float &Pxy, float &Pxz,
                            float &Pyz) {
    Pxx = 0.0f; Pyy = 0.0f; Pzz = 0.0f; Pxy = 0.0f; Pxz = 0.0f; Pyz = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const int a = cxq(q), b = cyq(q), e = czq(q);
        float fn = d[q];
        if (a != 0) Pxx += fn;
        if (b != 0) Pyy += fn;
        if (e != 0) Pzz += fn;
        if (a * b != 0) Pxy += a * b > 0 ? fn : -fn;
        if (a * e != 0) Pxz += a * e > 0 ? fn : -fn;
        if (b * e != 0) Pyz += b * e > 0 ? fn : -fn;
    }
}

// Hermite projection sum_ab Q_ab P_ab of direction q (D3Q19 has at most one
// nonzero off-diagonal Q); sc multiplies each P first when given
template <int Q>
LBM_DEV float hermite2(float Pxx, float Pyy, float Pzz, float Pxy, float Pxz, float Pyz) {
    constexpr int a = cxq(Q), b = cyq(Q), e = czq(Q);
    const float cs2 = LBM_CS2;
    const float Qxx = (float)(a * a) - cs2, Qyy = (float)(b * b) - cs2, Qzz = (float)(e * e) - cs2;
    float t = Qxx * Pxx + Qyy * Pyy + Qzz * Pzz;
    float s2 = 0.0f;
    if (a * b != 0) s2 = a * b > 0 ? Pxy : -Pxy;
    if (a * e != 0) s2 = a * e > 0 ? Pxz : -Pxz;
    if (b * e != 0) s2 = b * e > 0 ? Pyz : -Pyz;
    return t + 2.0f * s2;
}

// collide_KBC / collide_regularized for one cell (in place on f[])
// COLL: the collision model when the caller knows it at compile time (-1:
// from P.collision)
template <int COLL = -1>
LBM_DEV void collide(const StepArgs &A, int c, int k, bool solid, bool water, bool gas, float gbf, float r,
                     float vx, float vy, float vz, float om, float f[19]) {
    const lbm_params &P = A.P;
    const float eps = 1e-6f;
    if (gas) { r = P.rho0; vx = 0.0f; vy = 0.0f; vz = 0.0f; }
    float u2 = usq(vx, vy, vz);
    float fe[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        switch (q) {
#define FQ(Q) case Q: fe[q] = feq<Q>(r, vx, vy, vz, u2); break;
            FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
            FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
        }
    }
    const bool force = water && !gas;
    const float fz = force ? -r * g_local(P, gbf) : 0.0f;
    if (COLL == LBM_COLLIDE_REGULARIZED || (COLL < 0 && P.collision == LBM_COLLIDE_REGULARIZED)) {
        if (gas) {
#pragma unroll
            for (int q = 0; q < 19; ++q) f[q] = fe[q];
            return;
        }
        float d[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) d[q] = f[q] - fe[q];
        float Pxx, Pyy, Pzz, Pxy, Pxz, Pyz;
        second_moments(d, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz);
        const float omc = 1.0f - om;
        float fsv[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float h2 = 0.0f;
            switch (q) {
#define FQ(Q) case Q: h2 = hermite2<Q>(Pxx, Pyy, Pzz, Pxy, Pxz, Pyz); break;
                FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
            }
            float fnr = wq(q) * LBM_INV_2CS4 * h2;
            float v = fe[q] + omc * fnr;
            if (force) {
                float fi = 0.0f;
                switch (q) {
#define FQ(Q) case Q: fi = guo<Q>(om, vx, vy, vz, fz); break;
                    FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                    FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
                }
                v = v + fi;
            }
            fsv[q] = v;
        }
        float alpha = 1.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (fsv[q] < eps) {
                float den = fsv[q] - fe[q];
                if (den < 0.0f) {
                    float cand = (eps - fe[q]) / den;
                    if (cand < alpha) alpha = cand;
                }
            }
        }
        if (alpha < 0.0f) alpha = 0.0f;
        if (alpha > 1.0f) alpha = 1.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = fe[q] + alpha * (fsv[q] - fe[q]);
        return;
    }
    // KBC-style BGK with positivity limiter, top sponge and backscatter
    if (P.enable_top_sponge && k > A.D.nz - 3) {
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = f[q] - LBM_OM_SPONGE * (f[q] - fe[q]);
        return;
    }
    float fsv[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float v = f[q] - om * (f[q] - fe[q]);
        if (force) {
            float fi = 0.0f;
            switch (q) {
#define FQ(Q) case Q: fi = guo<Q>(om, vx, vy, vz, fz); break;
                FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
            }
            v = v + fi;
        }
        fsv[q] = v;
    }
    float alpha = 1.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (fsv[q] < eps) {
            float den = fsv[q] - fe[q];
            if (den < 0.0f) {
                float cand = (eps - fe[q]) / den;
                if (cand < alpha) alpha = cand;
            }
        }
    }
    if (alpha < 0.0f) alpha = 0.0f;
    if (alpha > 1.0f) alpha = 1.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = fe[q] + alpha * (fsv[q] - fe[q]);
    if (P.c_backscatter > 0.0f && !solid) {
        float d[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) d[q] = f[q] - fe[q];
        float Pxx, Pyy, Pzz, Pxy, Pxz, Pyz;
        second_moments(d, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz);
        float tr = (Pxx + Pyy + Pzz) / 3.0f;
        Pxx -= tr; Pyy -= tr; Pzz -= tr;
        const uint64_t key = A.clock ? (uint64_t)(*A.clock + (long long)A.step) : A.step;
        float xi = 2.0f * lbm_uniform01(P.seed, key, (uint64_t)c) - 1.0f;
        float scale = P.c_backscatter * xi;
        float sPxx = scale * Pxx, sPyy = scale * Pyy, sPzz = scale * Pzz;
        float sPxy = scale * Pxy, sPxz = scale * Pxz, sPyz = scale * Pyz;
        float dl[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float h2 = 0.0f;
            switch (q) {
#define FQ(Q) case Q: h2 = hermite2<Q>(sPxx, sPyy, sPzz, sPxy, sPxz, sPyz); break;
                FQ(0) FQ(1) FQ(2) FQ(3) FQ(4) FQ(5) FQ(6) FQ(7) FQ(8) FQ(9) FQ(10) FQ(11) FQ(12) FQ(13) FQ(14)
                FQ(15) FQ(16) FQ(17) FQ(18)
#undef FQ
            }
            dl[q] = wq(q) * LBM_INV_2CS4 * h2;
        }
        float gamma = 1.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (dl[q] < 0.0f) {
                float cand = (eps - f[q]) / dl[q];
                if (cand < gamma) gamma = cand;
            }
        }
        if (gamma < 0.0f) gamma = 0.0f;
        if (gamma > 1.0f) gamma = 1.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = f[q] + gamma * dl[q];
    }
}

}  // namespace lbm
