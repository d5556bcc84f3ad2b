// lbm_diag.cuh - device reductions of the reference harness's metrics.
//
// run_ab_case.py computes its per-plot metric row (make_visualize,
// run_ab_case.py:283-679) and main() its health line (CODEX.py:3930-3937)
// on the host from whole fields.  Here the same quantities are reduced on
// the device and only a small record is copied back:
//   k_diag_cells     one pass over every cell: the maximum speed over active
//                    cells (first maximum in C order), the volume and VOF
//                    sums and counts; per-block partials
//   k_diag_columns   per x: the surface elevation summed over y, min and max
//   k_diag_slice     the xz slice at slice_j: pressure, total pressure,
//                    vorticity, obstacle and band masks
//   k_diag_slice_sum the slice's high-pass values and masked sums, in two
//                    passes (band means, then squared deviations); per-block
//                    partials
//   k_diag_slice_mean the band means between the two passes
//   k_diag_final     one block: the partials in a fixed order, the surface
//                    line statistics, the neighbourhood of the maximum
// Sums are FP64 and reduced in a fixed order, so a result does not depend on
// scheduling.
#pragma once

#include "lbm_stages.cuh"

namespace lbm {

LBM_DEV bool diag_open(const DiagArgs &G, int k, int j, int i) {
    return cell_open(G.P, G.slot, G.D, G.bed, k, j, i);
}
// inactive in the reference's sense: obstacle, or gas with a free surface
LBM_DEV bool diag_inactive(const DiagArgs &G, int c, int k, int j, int i) {
    if (!diag_open(G, k, j, i)) return true;
    return G.fs && G.type[c] == LBM_FS_GAS;
}
// speed of a cell in m/s as the reference's float32 numpy evaluates it
LBM_DEV float diag_speed_phys(const DiagArgs &G, int c) {
    const float a = G.ux[c], b = G.uy[c], d = G.uz[c];
    const float s = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(d, d)));
    return __fmul_rn(s, G.P.vel_scale);
}

__global__ void __launch_bounds__(DIAG_THREADS) k_diag_cells(DiagArgs G) {
    const Dom &D = G.D;
    DiagCellPart my;
    my.max_key = 0ull;
    my.active = my.tiny = my.excess_count = 0;
    my.fill_sum = my.mass_sum = my.excess_sum = 0.0;
    my.min_iface = 3.4e38f;
    my.pad = 0;
    const float empty = G.P.vof_empty_fill_threshold;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < (long long)D.n;
         c += (long long)gridDim.x * blockDim.x) {
        const int ci = (int)c;
        const int k = ci / (int)D.a, r = ci - k * (int)D.a, j = r / D.nx, i = r - j * D.nx;
        const bool open = diag_open(G, k, j, i);
        const bool inactive = !open || (G.fs && G.type[ci] == LBM_FS_GAS);
        if (!inactive) {
            const float sp = diag_speed_phys(G, ci);
            const unsigned long long key =
                ((unsigned long long)__float_as_uint(sp) << 32) | (unsigned long long)(0xffffffffu - (unsigned)ci);
            if (key > my.max_key) my.max_key = key;
            my.active++;
        }
        if (open && G.fs) {
            const float fl = G.fill[ci];
            my.fill_sum += (double)fl;
            if (G.vof) {
                my.mass_sum += (double)G.mass[ci];
                const float ex = G.excess[ci];
                my.excess_sum += (double)ex;
                if (fabsf(ex) > 1.0e-12f) my.excess_count++;
                if (G.type[ci] == LBM_FS_INTERFACE) {
                    my.min_iface = fminf(my.min_iface, fl);
                    if (fl > 0.0f && fl < empty) my.tiny++;
                }
            }
        }
    }
    // block reduction in a fixed order
    __shared__ DiagCellPart sh[DIAG_THREADS];
    sh[threadIdx.x] = my;
    __syncthreads();
    for (int w = DIAG_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            DiagCellPart &a = sh[threadIdx.x];
            const DiagCellPart &b = sh[threadIdx.x + w];
            a.max_key = a.max_key > b.max_key ? a.max_key : b.max_key;
            a.active += b.active;
            a.tiny += b.tiny;
            a.excess_count += b.excess_count;
            a.fill_sum += b.fill_sum;
            a.mass_sum += b.mass_sum;
            a.excess_sum += b.excess_sum;
            a.min_iface = fminf(a.min_iface, b.min_iface);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) G.cellp[blockIdx.x] = sh[0];
}

__global__ void k_diag_columns(DiagArgs G) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G.D.nx) return;
    double s = 0.0;
    float lo = 3.4e38f, hi = -3.4e38f;
    for (int j = 0; j < G.D.ny; ++j) {
        const float h = G.fs_h[G.D.col(j, i)];
        s += (double)h;
        lo = fminf(lo, h);
        hi = fmaxf(hi, h);
    }
    G.col_eta[i] = s;
    G.col_min[i] = lo;
    G.col_max[i] = hi;
}

// the xz slice at slice_j: pressure, total pressure, vorticity and masks
__global__ void k_diag_slice(DiagArgs G) {
    const Dom &D = G.D;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= D.nz * D.nx) return;
    const int k = t / D.nx, i = t - k * D.nx, j = G.slice_j;
    const lbm_params &P = G.P;
    const int c = D.cell(k, j, i);
    const bool inactive = diag_inactive(G, c, k, j, i);
    const bool xper = !P.x_solid;
    // vorticity dv/dx - du/dz of (ux, uz) in double; du/dz wraps in z as np.roll does
    double dvdx;
    if (xper) {
        const int ip = i + 1 == D.nx ? 0 : i + 1, im = i == 0 ? D.nx - 1 : i - 1;
        dvdx = ((double)G.uz[D.cell(k, j, ip)] - (double)G.uz[D.cell(k, j, im)]) / 2.0;
    } else if (i == 0) {
        dvdx = (double)G.uz[D.cell(k, j, 1)] - (double)G.uz[c];
    } else if (i == D.nx - 1) {
        dvdx = (double)G.uz[c] - (double)G.uz[D.cell(k, j, i - 1)];
    } else {
        dvdx = ((double)G.uz[D.cell(k, j, i + 1)] - (double)G.uz[D.cell(k, j, i - 1)]) / 2.0;
    }
    const int kp = k + 1 == D.nz ? 0 : k + 1, km = k == 0 ? D.nz - 1 : k - 1;
    const double dudz = ((double)G.ux[D.cell(kp, j, i)] - (double)G.ux[D.cell(km, j, i)]) / 2.0;
    const double vort = dvdx - dudz;
    // pressure: the lattice perturbation in Pa, plus the mode's hydrostatic parts
    const double dx = P.dx, z = ((double)k + 0.5) * dx;
    const double plb = G.rho_phys * (double)P.vel_scale * (double)P.vel_scale * ((G.rho[c] - (double)P.rho0) / 3.0);
    double pt = plb, pp = plb;
    const double rg = G.rho_phys * G.gravity_phys;
    const bool column = G.fs && !G.vof;
    const double surf = G.fs ? (double)G.fs_h[D.col(j, i)] : 0.0;
    if (G.fs) {
        if (P.use_component_balanced_pressure) {
            const int tp = G.types_are_prev ? G.type_prev[c] : G.type[c];
            const bool open = diag_open(G, k, j, i);
            pt = plb + rg * (double)prh_of(P, k, open, tp);
            pp = pt;
        } else if (P.use_hydrostatic_balanced_pressure) {
            pt = plb + rg * ((double)P.fs_base_m - z);
            pp = column ? plb : pt;
        } else {
            pt = plb;
            pp = column ? pt - rg * fmax(surf - z, 0.0) : pt;
        }
    }
    G.sl_p[t] = pp;
    G.sl_pt[t] = pt;
    G.sl_v[t] = vort;
    uint8_t m = inactive ? 1 : 0;
    if (!inactive) {
        const float ph = phi_cell(P, D, G.bed.h, k, j, i);
        if (ph > 0.0f && (double)ph <= 10.0 * dx) m |= 2;
        if (column && z <= surf + 0.5 * dx && z >= surf - 3.0 * dx) m |= 4;
    }
    G.sl_mask[t] = m;
}

// high_pass_xz (run_ab_case.py:111-137) of a slice field at (k, i): linear
// ghost values at the ends of z, and of x when x is not periodic
LBM_DEV double diag_hp(const double *f, int nz, int nx, bool xper, int k, int i) {
    const double v = f[k * nx + i];
    const double zp = k + 1 < nz ? f[(k + 1) * nx + i] : 2.0 * v - f[(k - 1) * nx + i];
    const double zm = k > 0 ? f[(k - 1) * nx + i] : 2.0 * v - f[(k + 1) * nx + i];
    double xp, xm;
    if (xper) {
        xp = f[k * nx + (i + 1 == nx ? 0 : i + 1)];
        xm = f[k * nx + (i == 0 ? nx - 1 : i - 1)];
    } else {
        xp = i + 1 < nx ? f[k * nx + i + 1] : 2.0 * v - f[k * nx + i - 1];
        xm = i > 0 ? f[k * nx + i - 1] : 2.0 * v - f[k * nx + i + 1];
    }
    return v - 0.25 * (zp + zm + xp + xm);
}

// Pass 0 sums the values of each band; pass 1 sums the squared deviations
// from the band means (G.slice_mean) for the centred statistics and the
// squares for the high-pass ones, so that no large mean cancels.
__global__ void __launch_bounds__(DIAG_SLICE_THREADS) k_diag_slice_sum(DiagArgs G, int pass) {
    const int nz = G.D.nz, nx = G.D.nx;
    const bool xper = !G.P.x_solid;
    DiagSlicePart my;
    for (int b = 0; b < 2; ++b) {
        for (int q = 0; q < 6; ++q) my.s[b][q] = my.s2[b][q] = 0.0;
        my.n[b] = 0;
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nz * nx; t += gridDim.x * blockDim.x) {
        const int k = t / nx, i = t - k * nx;
        // the free-surface band of the VOF mode: interface cells of the slice
        // and their four xz neighbours (run_ab_case.py:557-568)
        uint8_t m = G.sl_mask[t];
        if (G.fs && G.vof && !(m & 1)) {
            auto seed = [&](int kk, int ii) {
                const int cc = G.D.cell(kk, G.slice_j, ii);
                const float fl = G.fill[cc];
                return (G.sl_mask[kk * nx + ii] & 1) == 0 && fl > 0.0f && fl < 1.0f;
            };
            if (seed(k, i) || (k > 0 && seed(k - 1, i)) || (k + 1 < nz && seed(k + 1, i)) ||
                (i > 0 && seed(k, i - 1)) || (i + 1 < nx && seed(k, i + 1)))
                m |= 4;
        }
        if (!(m & 6)) continue;
        double v[6];
        v[0] = G.sl_p[t];
        v[1] = diag_hp(G.sl_p, nz, nx, xper, k, i);
        v[2] = G.sl_pt[t];
        v[3] = diag_hp(G.sl_pt, nz, nx, xper, k, i);
        v[4] = G.sl_v[t];
        v[5] = diag_hp(G.sl_v, nz, nx, xper, k, i);
        for (int b = 0; b < 2; ++b) {
            if (!(m & (2 << b))) continue;
            for (int q = 0; q < 6; ++q) {
                if (pass == 0) {
                    my.s[b][q] += v[q];
                } else {
                    const double d = (q & 1) ? v[q] : v[q] - G.slice_mean[b * 6 + q];
                    my.s2[b][q] += d * d;
                }
            }
            my.n[b]++;
        }
    }
    __shared__ DiagSlicePart sh[DIAG_SLICE_THREADS];
    sh[threadIdx.x] = my;
    __syncthreads();
    for (int w = DIAG_SLICE_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            for (int b = 0; b < 2; ++b) {
                for (int q = 0; q < 6; ++q) {
                    sh[threadIdx.x].s[b][q] += sh[threadIdx.x + w].s[b][q];
                    sh[threadIdx.x].s2[b][q] += sh[threadIdx.x + w].s2[b][q];
                }
                sh[threadIdx.x].n[b] += sh[threadIdx.x + w].n[b];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) G.slp[pass * G.nslp + blockIdx.x] = sh[0];
}

// the band means of pass 0, in a fixed order
__global__ void k_diag_slice_mean(DiagArgs G) {
    if (threadIdx.x != 0) return;
    for (int b = 0; b < 2; ++b)
        for (int q = 0; q < 6; ++q) {
            double s = 0.0;
            long long n = 0;
            for (int u = 0; u < G.nslp; ++u) {
                s += G.slp[u].s[b][q];
                n += G.slp[u].n[b];
            }
            G.slice_mean[b * 6 + q] = n > 0 ? s / (double)n : 0.0;
        }
}

LBM_DEV double diag_rms(double s2, long long n) {
    if (n <= 0) return __longlong_as_double(0x7ff8000000000000ll);
    return sqrt(s2 / (double)n);
}

__global__ void k_diag_final(DiagArgs G) {
    const double NaN = __longlong_as_double(0x7ff8000000000000ll);
    const Dom &D = G.D;
    const lbm_params &P = G.P;
    if (threadIdx.x != 0) return;
    lbm_diag o;
    memset(&o, 0, sizeof o);
    DiagCellPart a = G.cellp[0];
    for (int b = 1; b < G.ncellp; ++b) {
        const DiagCellPart &p = G.cellp[b];
        a.max_key = a.max_key > p.max_key ? a.max_key : p.max_key;
        a.active += p.active;
        a.tiny += p.tiny;
        a.excess_count += p.excess_count;
        a.fill_sum += p.fill_sum;
        a.mass_sum += p.mass_sum;
        a.excess_sum += p.excess_sum;
        a.min_iface = fminf(a.min_iface, p.min_iface);
    }
    const double dx = P.dx;
    o.active_cells = a.active;
    o.max_speed_fs_type = -1;
    o.max_speed_fs_fill = NaN;
    o.max_speed_wet_neighbors = o.max_speed_full_neighbors = o.max_speed_gas_neighbors = -1;
    if (a.active > 0) {
        const float sp = __uint_as_float((unsigned)(a.max_key >> 32));
        const int c = (int)(0xffffffffu - (unsigned)(a.max_key & 0xffffffffull));
        const int k = c / (int)D.a, r = c - k * (int)D.a, j = r / D.nx, i = r - j * D.nx;
        o.max_speed_phys = sp;
        const float a2 = G.ux[c], b2 = G.uy[c], d2 = G.uz[c];
        o.max_speed_lb = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(a2, a2), __fmul_rn(b2, b2)), __fmul_rn(d2, d2)));
        o.max_k = k; o.max_j = j; o.max_i = i;
        o.max_speed_x = ((double)i + 0.5) * dx;
        o.max_speed_y = ((double)j + 0.5) * dx;
        o.max_speed_z = ((double)k + 0.5) * dx;
        if (G.fs) {
            o.max_speed_fs_type = G.type[c];
            o.max_speed_fs_fill = G.fill[c];
            int wet = 0, full = 0, gas = 0;
            for (int q = 1; q < 19; ++q) {
                const int cx = q == 1 || q == 7 || q == 10 || q == 11 || q == 14 ? 1
                             : (q == 2 || q == 8 || q == 9 || q == 12 || q == 13 ? -1 : 0);
                const int cy = q == 3 || q == 7 || q == 8 || q == 15 || q == 18 ? 1
                             : (q == 4 || q == 9 || q == 10 || q == 16 || q == 17 ? -1 : 0);
                const int cz = q == 5 || q == 11 || q == 12 || q == 15 || q == 16 ? 1
                             : (q == 6 || q == 13 || q == 14 || q == 17 || q == 18 ? -1 : 0);
                int ni = i + cx;
                bool valid = true;
                if (!P.x_solid) ni = (ni + D.nx) % D.nx;
                else if (ni < 0 || ni >= D.nx) valid = false;
                const int nj = (j + cy + D.ny) % D.ny, nk = k + cz;
                if (nk < 0 || nk >= D.nz) valid = false;
                if (valid && diag_open(G, nk, nj, ni)) {
                    const int cn = D.cell(nk, nj, ni);
                    if (G.type[cn] == LBM_FS_GAS) {
                        gas++;
                    } else {
                        wet++;
                        if (G.fill[cn] > 0.5f) full++;
                    }
                }
            }
            o.max_speed_wet_neighbors = wet;
            o.max_speed_full_neighbors = full;
            o.max_speed_gas_neighbors = gas;
        }
    } else {
        o.max_speed_lb = o.max_speed_phys = NaN;
        o.max_speed_x = o.max_speed_y = o.max_speed_z = NaN;
        o.max_k = o.max_j = o.max_i = -1;
    }
    o.water_volume = o.vof_mass_total = o.vof_min_interface_fill = o.vof_pending_excess_mass = NaN;
    o.vof_tiny_interface_count = o.vof_pending_excess_count = -1;
    o.surface_min = o.surface_max = o.surface_symmetry_l2 = o.surface_eta_hp_rms = NaN;
    o.surface_left_max = o.surface_right_max = NaN;
    if (G.fs) {
        o.water_volume = a.fill_sum * dx * dx * dx;
        if (G.vof) {
            o.vof_mass_total = a.mass_sum;
            o.vof_min_interface_fill = a.min_iface < 3.0e38f ? (double)a.min_iface : NaN;
            o.vof_tiny_interface_count = a.tiny;
            o.vof_pending_excess_mass = a.excess_sum;
            o.vof_pending_excess_count = a.excess_count;
        }
        // surface line: eta(x) = mean over y of the height minus the base level
        const int nx = D.nx;
        double lo = 3.4e38, hi = -3.4e38, sym = 0.0, hp = 0.0, lmax = -3.4e38, rmax = -3.4e38;
        const double base = P.fs_base_m, Lx = (double)nx * dx;
        for (int i = 0; i < nx; ++i) {
            lo = fmin(lo, (double)G.col_min[i]);
            hi = fmax(hi, (double)G.col_max[i]);
            const double e = G.col_eta[i] / (double)D.ny - base;
            const double er = G.col_eta[nx - 1 - i] / (double)D.ny - base;
            sym += (e - er) * (e - er);
            double h;
            if (P.x_solid) {
                if (i == 0) h = e - (G.col_eta[1] / (double)D.ny - base);
                else if (i == nx - 1) h = e - (G.col_eta[nx - 2] / (double)D.ny - base);
                else h = e - 0.5 * ((G.col_eta[i - 1] + G.col_eta[i + 1]) / (double)D.ny - 2.0 * base);
            } else {
                const int im = i == 0 ? nx - 1 : i - 1, ip = i + 1 == nx ? 0 : i + 1;
                h = e - 0.5 * ((G.col_eta[im] + G.col_eta[ip]) / (double)D.ny - 2.0 * base);
            }
            hp += h * h;
            if (((double)i + 0.5) * dx < 0.5 * Lx) lmax = fmax(lmax, e);
            else rmax = fmax(rmax, e);
        }
        o.surface_min = lo;
        o.surface_max = hi;
        o.surface_symmetry_l2 = sqrt(sym / (double)nx);
        o.surface_eta_hp_rms = sqrt(hp / (double)nx);
        o.surface_left_max = lmax > -3.0e38 ? lmax : NaN;
        o.surface_right_max = rmax > -3.0e38 ? rmax : NaN;
    }
    // slice statistics: the second pass's partials
    const DiagSlicePart *p1 = G.slp + G.nslp;
    DiagSlicePart s = p1[0];
    for (int b = 1; b < G.nslp; ++b)
        for (int u = 0; u < 2; ++u) {
            for (int q = 0; q < 6; ++q) s.s2[u][q] += p1[b].s2[u][q];
            s.n[u] += p1[b].n[u];
        }
    double r[2][6];
    for (int u = 0; u < 2; ++u)
        for (int q = 0; q < 6; ++q) r[u][q] = diag_rms(s.s2[u][q], s.n[u]);
    o.p_rms = r[0][0]; o.p_hp_rms = r[0][1]; o.p_total_rms = r[0][2]; o.p_total_hp_rms = r[0][3];
    o.vort_rms = r[0][4]; o.vort_hp_rms = r[0][5];
    o.band_cells = s.n[0];
    if (G.fs) {
        o.fs_p_rms = r[1][0]; o.fs_p_hp_rms = r[1][1]; o.fs_p_total_rms = r[1][2]; o.fs_p_total_hp_rms = r[1][3];
        o.fs_vort_rms = r[1][4]; o.fs_vort_hp_rms = r[1][5];
        o.fs_band_cells = s.n[1];
    } else {
        o.fs_p_rms = o.fs_p_hp_rms = o.fs_p_total_rms = o.fs_p_total_hp_rms = o.fs_vort_rms = o.fs_vort_hp_rms = NaN;
        o.fs_band_cells = 0;
    }
    *G.out = o;
}

}  // namespace lbm
