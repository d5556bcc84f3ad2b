// lbm_vof.cuh - VOF / free-surface LBM kernels (CODEX.py:1289-2373).
//
// One step of the VOF path runs, after the stream, the reference's fixed
// sequence (CODEX.py:3898-3920): mass exchange, mass update and
// pre-classification, three rounds of excess redistribution and
// finalisation, interface layer, orphan removal, detached-cell advection
// and residual compression, a last redistribution, the trapped-gas
// collapse (flood fill from the top row, FP64 sums), the column height,
// refill and coalescence repair.
//
// The reference's redistribution, orphan and detached kernels let many
// threads add into the same cell (atomics, order-dependent in f32).  Here
// they are split into a donor pass that reads a snapshot and records what
// each donor sends, and a receiver pass in which every cell adds its
// incoming shares in a fixed order (direction q, then distance): the
// result is deterministic and equal to the CPU oracle's.  Global sums are
// FP64 with a fixed 256-wide pairwise tree (lbm_tree_sum in the oracle).
#pragma once

#include "lbm_stages.cuh"

namespace lbm {

constexpr float VOF_E12 = 1.0e-12f;
constexpr float VOF_E8 = 1.0e-8f;
constexpr float VOF_E7 = 1.0e-7f;
constexpr float VOF_E6 = 1.0e-6f;
constexpr float FILL_LO = 1e-4f;                // CODEX.py:1225
constexpr float FILL_HI = (float)(1.0 - 1e-4);  // CODEX.py:1227


// neighbour (k,j,i) + (dk,dj,di): x periodic or bounded by the solid walls,
// y periodic, z bounded
LBM_DEV bool vnbr(const Dom &D, bool xs, int k, int j, int i, int di, int dj, int dk, int &n) {
    int ni = i + di;
    if (!xs) {
        ni %= D.nx;
        if (ni < 0) ni += D.nx;
    } else if (ni < 0 || ni >= D.nx) {
        return false;
    }
    int nj = (j + dj) % D.ny;
    if (nj < 0) nj += D.ny;
    const int nk = k + dk;
    if (nk < 0 || nk >= D.nz) return false;
    n = D.cell(nk, nj, ni);
    return true;
}
LBM_DEV void vkji(const Dom &D, int c, int &k, int &j, int &i) {
    k = c / (int)D.a;
    int r = c - k * (int)D.a;
    j = r / D.nx;
    i = r - j * D.nx;
}
LBM_DEV float rho_ref(const VofArgs &V, int c) {
    float r = V.rho[c];
    if (r < VOF_E8) r = V.P.rho0;
    return r;
}

// lattice_open[0] and lattice_open_frac[0] of every cell for the step's
// geometry (the VOF kernels look them up for 18 neighbours per cell)
// Donor-in-reach flags of the receiver passes.  A donor (excess mass or an
// orphan) marks the coarse block of VOF_CB^3 cells it lies in and the 26
// around it (wrapping as the neighbour lookup does), so every cell within
// VOF_CB cells of a donor sits in a marked block; a receiver in an unmarked
// block has no donor in reach, and its loop over the donors would add
// nothing.  Wrapped neighbours fall in the next block only when the
// periodic extents are multiples of VOF_CB; otherwise (near_ok 0) the flags
// are not used.
LBM_DEV void vof_mark_near(const VofArgs &V, int k, int j, int i) {
    if (!V.near_ok) return;
    const int bk = k / VOF_CB, bj = j / VOF_CB, bi = i / VOF_CB;
    for (int dk = -1; dk <= 1; ++dk) {
        const int zk = bk + dk;
        if (zk < 0 || zk >= V.cbz) continue;
        for (int dj = -1; dj <= 1; ++dj) {
            const int yj = (bj + dj + V.cby) % V.cby;
            for (int di = -1; di <= 1; ++di) {
                int xi = bi + di;
                if (V.P.x_solid) {
                    if (xi < 0 || xi >= V.cbx) continue;
                } else {
                    xi = (xi + V.cbx) % V.cbx;
                }
                V.near[((size_t)zk * V.cby + yj) * V.cbx + xi] = 1;
            }
        }
    }
}
LBM_DEV bool vof_near(const VofArgs &V, int k, int j, int i) {
    return !V.near_ok || V.near[((size_t)(k / VOF_CB) * V.cby + j / VOF_CB) * V.cbx + i / VOF_CB] != 0;
}

__global__ void k_vof_open(VofArgs V, BedView B) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)V.D.n) return;
    int k, j, i;
    vkji(V.D, c, k, j, i);
    // far from the bed and every other geometry (solid x walls close links,
    // not cells): open, full open fraction
    if (geo_far_except_x(V.P, V.D, B, k, j, i)) {
        V.open[c] = 1;
        V.lf0[c] = 1.0f;
        return;
    }
    GeoLinks L;
    Geo g = geo_cell(V.P, V.slot, V.D, B, k, j, i, L, true);
    V.open[c] = (int8_t)(g.lo & 1u);
    V.lf0[c] = g.fast ? 1.0f : L.lf[0];
}

// compute_vof_mass_exchange, CODEX.py:1305-1350 (delta into fa[0..n))
template <int S>
__global__ void k_vof_exchange(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (c >= (int)D.n) return;
    float dm = 0.0f;
    if (V.open[c] && V.type[c] == LBM_FS_INTERFACE) {
        int k, j, i;
        vkji(D, c, k, j, i);
        const typename Store<S>::T *f = (const typename Store<S>::T *)V.f;
        const float fc = V.fill[c];
#pragma unroll
        for (int q = 1; q < 19; ++q) {
            int n;
            if (!vnbr(D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n)) continue;
            if (!(V.open[n] && V.type[n] != LBM_FS_GAS)) continue;
            float lw = 1.0f;
            if (V.type[n] == LBM_FS_INTERFACE) lw = 0.5f * (fc + V.fill[n]);
            if (lw > 0.0f)
                dm += lw * (Store<S>::ld(f, (size_t)oppq(q) * D.n + c, oppq(q), V.P.rho0) -
                            Store<S>::ld(f, (size_t)q * D.n + n, q, V.P.rho0));
        }
    }
    V.fa[c] = dm;
}

LBM_DEV void add_count(int *ctr, bool b) {
    const unsigned m = __activemask();
    const int s = __popc(__ballot_sync(m, b));
    if ((threadIdx.x & 31) == (__ffs(m) - 1) && s) atomicAdd(ctr, s);
}

// apply_vof_mass_update_and_preclassify, CODEX.py:1353-1414
__global__ void k_vof_apply(VofArgs V, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool counted = false;
    if (c < (int)V.D.n) {
        const int8_t old = V.type[c];
        V.type_prev[c] = old;
        if (!V.open[c]) {
            V.mass_excess[c] = 0.0f;
            V.excess_dir[c] = 0;
            V.mass[c] = 0.0f;
            V.fill[c] = 0.0f;
            V.type[c] = LBM_FS_GAS;
        } else {
            const float rr = rho_ref(V, c);
            float m = V.mass[c];
            if (old == LBM_FS_INTERFACE) m += V.fa[c];
            else if (old == LBM_FS_LIQUID) m = rr;
            else m = 0.0f;
            float ex = 0.0f;
            int8_t ed = 0;
            if (m < 0.0f) { ex = m; ed = -1; m = 0.0f; }
            else if (m > rr) { ex = m - rr; ed = 1; m = rr; }
            float fl = m / rr;
            int8_t ct = LBM_FS_INTERFACE;
            if (fl > FILL_LO && fl < V.P.vof_empty_fill_threshold) { ex = m; ed = -1; m = 0.0f; fl = 0.0f; ct = LBM_FS_GAS; }
            else if (fl <= FILL_LO) { fl = 0.0f; ct = LBM_FS_GAS; }
            else if (fl >= FILL_HI) { fl = 1.0f; ct = LBM_FS_LIQUID; }
            V.mass[c] = m;
            V.mass_excess[c] = ex;
            V.excess_dir[c] = ed;
            counted = fabsf(ex) > VOF_E7;
            V.fill[c] = fl;
            V.type[c] = ct;
        }
    }
    add_count(cnt, counted);
}

// redistribute_vof_mass_excess, CODEX.py:1417-1574: donor pass.  Reads the
// snapshots m0 (mass) and x0 (excess); records per donor its direction,
// normal, capacity and weight sum.
__global__ void k_vof_redist_donor(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (c >= (int)D.n) return;
    float *nxv = V.fa, *nyv = V.fa + D.n, *nzv = V.fa + 2 * D.n, *cap = V.fa + 3 * D.n, *wsum = V.fa + 4 * D.n;
    int8_t *dir = V.ba, *donor = V.ba + D.n;
    const float ex = V.x0[c];
    if (!(fabsf(ex) > VOF_E12)) {
        donor[c] = 0;
        return;
    }
    int k, j, i;
    vkji(D, c, k, j, i);
    int d = V.excess_dir[c];
    if (d == 0) {
        d = 1;
        if (ex < 0.0f) d = -1;
    }
    int ip = i + 1, im = i - 1;
    if (!V.P.x_solid) {
        ip = (i + 1) % D.nx;
        im = (i - 1 + D.nx) % D.nx;
    } else {
        if (ip >= D.nx) ip = D.nx - 1;
        if (im < 0) im = 0;
    }
    const int jp = (j + 1) % D.ny, jm = (j - 1 + D.ny) % D.ny;
    int kp = k + 1, km = k - 1;
    if (kp >= D.nz) kp = D.nz - 1;
    if (km < 0) km = 0;
    float nx_ = -(V.fill[D.cell(k, j, ip)] - V.fill[D.cell(k, j, im)]);
    float ny_ = -(V.fill[D.cell(k, jp, i)] - V.fill[D.cell(k, jm, i)]);
    float nz_ = -(V.fill[D.cell(kp, j, i)] - V.fill[D.cell(km, j, i)]);
    const float nm = sqrtf(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
    if (nm > VOF_E8) {
        const float inv = 1.0f / nm;
        nx_ *= inv;
        ny_ *= inv;
        nz_ *= inv;
    }
    float ws = 0.0f, cs = 0.0f;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        int n;
        if (!vnbr(D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n) || V.open[n] != 1) continue;
        const float nd = (float)cxq(q) * nx_ + (float)cyq(q) * ny_ + (float)czq(q) * nz_;
        const bool elig = d > 0 ? V.type[n] != LBM_FS_LIQUID : V.type[n] != LBM_FS_GAS;
        if (!elig) continue;
        float room;
        if (ex > 0.0f) {
            float rr = V.rho[n];
            if (rr < VOF_E8) rr = V.P.rho0;
            room = rr - V.m0[n];
        } else {
            room = V.m0[n];
        }
        if (room > VOF_E12) {
            cs += room;
            const float wgt = d > 0 ? nd : -nd;
            if (wgt > 0.0f) ws += wgt * room;
        }
    }
    donor[c] = 1;
    vof_mark_near(V, k, j, i);
    dir[c] = (int8_t)d;
    nxv[c] = nx_;
    nyv[c] = ny_;
    nzv[c] = nz_;
    cap[c] = cs;
    wsum[c] = ws;
}

// receiver pass: each cell adds its incoming shares in order of q
__global__ void k_vof_redist_recv(VofArgs V) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (r >= (int)D.n) return;
    const float *nxv = V.fa, *nyv = V.fa + D.n, *nzv = V.fa + 2 * D.n, *cap = V.fa + 3 * D.n, *wsum = V.fa + 4 * D.n;
    const int8_t *dir = V.ba, *donor = V.ba + D.n;
    int k, j, i;
    vkji(D, r, k, j, i);
    float acc = V.m0[r];
    if (V.open[r] == 1 && vof_near(V, k, j, i)) {
#pragma unroll
        for (int q = 1; q < 19; ++q) {
            int d;
            if (!vnbr(D, V.P.x_solid, k, j, i, -cxq(q), -cyq(q), -czq(q), d)) continue;
            if (!donor[d] || !(cap[d] > VOF_E12)) continue;
            int dk, dj, di;
            vkji(D, d, dk, dj, di);
            int chk;
            if (!vnbr(D, V.P.x_solid, dk, dj, di, cxq(q), cyq(q), czq(q), chk) || chk != r) continue;
            const int dd = dir[d];
            const bool elig = dd > 0 ? V.type[r] != LBM_FS_LIQUID : V.type[r] != LBM_FS_GAS;
            if (!elig) continue;
            const float ex = V.x0[d];
            const float nd = (float)cxq(q) * nxv[d] + (float)cyq(q) * nyv[d] + (float)czq(q) * nzv[d];
            const float wgt = dd > 0 ? nd : -nd;
            float room;
            if (ex > 0.0f) {
                float rr = V.rho[r];
                if (rr < VOF_E8) rr = V.P.rho0;
                room = rr - V.m0[r];
            } else {
                room = V.m0[r];
            }
            if (!(room > VOF_E12)) continue;
            float share = ex * room / cap[d];
            if (wsum[d] > VOF_E12 && wgt > 0.0f) share = ex * wgt * room / wsum[d];
            else if (wsum[d] > VOF_E12) share = 0.0f;
            acc += share;
        }
    }
    if (donor[r] && !(cap[r] > VOF_E12)) acc += V.x0[r];
    V.mass[r] = acc;
    if (donor[r]) {
        V.mass_excess[r] = 0.0f;
        V.excess_dir[r] = 0;
    }
}

// finalize_vof_classification_from_mass, CODEX.py:1577-1624
__global__ void k_vof_finalize(VofArgs V, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    int counted = 0;
    if (c < (int)V.D.n) {
        V.mass_excess[c] = 0.0f;
        V.excess_dir[c] = 0;
        if (!V.open[c]) {
            V.mass[c] = 0.0f;
            V.fill[c] = 0.0f;
            V.type[c] = LBM_FS_GAS;
        } else {
            const float rr = rho_ref(V, c);
            float m = V.mass[c];
            float ex = 0.0f;
            int8_t ed = 0;
            if (m < 0.0f) { ex = m; ed = -1; m = 0.0f; counted++; }
            if (m > rr) { ex = m - rr; ed = 1; m = rr; counted++; }
            float fl = m / rr;
            int8_t ct = LBM_FS_INTERFACE;
            if (fl > FILL_LO && fl < V.P.vof_empty_fill_threshold) {
                ex = m; ed = -1; m = 0.0f; fl = 0.0f; ct = LBM_FS_GAS; counted++;
            } else if (fl <= FILL_LO) { fl = 0.0f; ct = LBM_FS_GAS; }
            else if (fl >= FILL_HI) { fl = 1.0f; ct = LBM_FS_LIQUID; }
            V.mass[c] = m;
            V.mass_excess[c] = ex;
            V.excess_dir[c] = ed;
            V.fill[c] = fl;
            V.type[c] = ct;
        }
    }
    const unsigned m = __activemask();
    const int s = __reduce_add_sync(m, counted);
    if ((threadIdx.x & 31) == (__ffs(m) - 1) && s) atomicAdd(cnt, s);
}

// enforce_vof_interface_layer, CODEX.py:1627-1656 (reads the type snapshot t0)
// Snapshot of the types for the interface layer (t0 = type) that also marks
// the coarse blocks holding an open gas cell (second half of V.near)
__global__ void k_vof_types_gas_mark(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)V.D.n) return;
    const int8_t t = V.type[c];
    V.t0[c] = t;
    if (V.near_ok && t == LBM_FS_GAS && V.open[c] == 1) {
        int k, j, i;
        vkji(V.D, c, k, j, i);
        const size_t nb = (size_t)V.cbx * V.cby * V.cbz;
        V.near[nb + ((size_t)(k / VOF_CB) * V.cby + j / VOF_CB) * V.cbx + i / VOF_CB] = 1;
    }
}
// one thread per coarse block: marked (first half of V.near) when a block
// within one block (wrapping as the neighbour lookup does) holds an open gas cell
__global__ void k_vof_gas_dilate(VofArgs V) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = V.cbx * V.cby * V.cbz;
    if (b >= nb) return;
    const int bi = b % V.cbx, bj = (b / V.cbx) % V.cby, bk = b / (V.cbx * V.cby);
    uint8_t any = 0;
    for (int dk = -1; dk <= 1 && !any; ++dk) {
        const int zk = bk + dk;
        if (zk < 0 || zk >= V.cbz) continue;
        for (int dj = -1; dj <= 1 && !any; ++dj) {
            const int yj = (bj + dj + V.cby) % V.cby;
            for (int di = -1; di <= 1 && !any; ++di) {
                int xi = bi + di;
                if (V.P.x_solid) {
                    if (xi < 0 || xi >= V.cbx) continue;
                } else {
                    xi = (xi + V.cbx) % V.cbx;
                }
                any = V.near[nb + ((size_t)zk * V.cby + yj) * V.cbx + xi];
            }
        }
    }
    V.near[b] = any;
}

__global__ void k_vof_interface_layer(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (c >= (int)D.n) return;
    if (!(V.open[c] == 1 && V.t0[c] == LBM_FS_LIQUID)) return;
    int k, j, i;
    vkji(D, c, k, j, i);
    if (!vof_near(V, k, j, i)) return;   // no open gas cell within one cell
    bool touches = false;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        int n;
        if (!vnbr(D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n)) continue;
        if (V.open[n] == 1 && V.t0[n] == LBM_FS_GAS) {
            touches = true;
            break;
        }
    }
    if (touches) {
        V.type[c] = LBM_FS_INTERFACE;
        V.fill[c] = 1.0f;
        V.mass[c] = V.rho[c];
    }
}

// remove_orphan_vof_interface_cells, CODEX.py:1659-1776: decision pass on
// the snapshots m0 (mass), x0 (fill), t0 (type)
__global__ void k_vof_orphan_donor(VofArgs V, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    bool counted = false;
    if (c < (int)D.n) {
        int8_t *orphan = V.ba;
        float *capw = V.fa, *topw = V.fa + D.n;
        const int R = V.P.vof_orphan_search_radius;
        const float othr = V.P.vof_orphan_empty_threshold;
        orphan[c] = 0;
        if (V.open[c] == 1 && V.t0[c] != LBM_FS_GAS && V.x0[c] > V.P.vof_empty_fill_threshold) {
            int k, j, i;
            vkji(D, c, k, j, i);
            int wet = 0, res = 0;
#pragma unroll
            for (int q = 1; q < 19; ++q) {
                int n;
                if (!vnbr(D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n) || V.open[n] != 1) continue;
                if (V.t0[n] != LBM_FS_GAS) {
                    wet++;
                    if (V.x0[n] >= othr) {
                        res++;
                        break;   // a resolved neighbour: not an orphan (res == 0 below fails)
                    }
                }
            }
            if (res == 0 && (V.x0[c] < othr || wet <= V.P.vof_orphan_max_weak_neighbors)) {
                const float m = V.m0[c];
                float cw = 0.0f, tw = 0.0f;
                for (int q = 1; q < 19; ++q)
                    for (int dist = 2; dist <= R; ++dist) {
                        int n;
                        const int di = dist * cxq(q), dj = dist * cyq(q), dk = dist * czq(q);
                        if (!vnbr(D, V.P.x_solid, k, j, i, di, dj, dk, n)) continue;
                        if (!(V.open[n] == 1 && V.t0[n] != LBM_FS_GAS && V.x0[n] >= othr)) continue;
                        float rr = V.rho[n];
                        if (rr < VOF_E8) rr = V.P.rho0;
                        const float room = rr - V.m0[n];
                        const float d2 = (float)(di * di + dj * dj + dk * dk);
                        tw += V.x0[n] / d2;
                        if (room > VOF_E12) cw += room / d2;
                    }
                if (m > VOF_E12 && (cw > VOF_E12 || tw > VOF_E12)) {
                    orphan[c] = 1;
                    vof_mark_near(V, k, j, i);
                    capw[c] = cw;
                    topw[c] = tw;
                    counted = true;
                }
            }
        }
    }
    add_count(cnt, counted);
}

// receiver pass of the orphan removal
__global__ void k_vof_orphan_recv(VofArgs V) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (r >= (int)D.n) return;
    const int8_t *orphan = V.ba;
    const float *capw = V.fa, *topw = V.fa + D.n;
    const int R = V.P.vof_orphan_search_radius;
    const float othr = V.P.vof_orphan_empty_threshold;
    int k, j, i;
    vkji(D, r, k, j, i);
    float acc = orphan[r] ? 0.0f : V.m0[r];
    // orphans reach R cells: the flags cover VOF_CB
    if (V.open[r] == 1 && V.t0[r] != LBM_FS_GAS && V.x0[r] >= othr && (R > VOF_CB || vof_near(V, k, j, i))) {
        float rr = V.rho[r];
        if (rr < VOF_E8) rr = V.P.rho0;
        const float room = rr - V.m0[r];
        for (int q = 1; q < 19; ++q)
            for (int dist = 2; dist <= R; ++dist) {
                int d;
                const int di = dist * cxq(q), dj = dist * cyq(q), dk = dist * czq(q);
                if (!vnbr(D, V.P.x_solid, k, j, i, -di, -dj, -dk, d) || !orphan[d]) continue;
                int ok, oj, oi;
                vkji(D, d, ok, oj, oi);
                int chk;
                if (!vnbr(D, V.P.x_solid, ok, oj, oi, di, dj, dk, chk) || chk != r) continue;
                const float d2 = (float)(di * di + dj * dj + dk * dk);
                float wgt = 0.0f;
                float den = capw[d];
                if (capw[d] > VOF_E12) {
                    if (room > VOF_E12) wgt = room / d2;
                } else {
                    wgt = V.x0[r] / d2;
                    den = topw[d];
                }
                if (den > VOF_E12 && wgt > 0.0f) acc += V.m0[d] * wgt / den;
            }
    }
    V.mass[r] = acc;
    if (orphan[r]) {
        V.fill[r] = 0.0f;
        V.type[r] = LBM_FS_GAS;
    }
}

// vof_unresolved_detached_cell, CODEX.py:1779-1810
LBM_DEV bool detached_cell(const VofArgs &V, int c, int k, int j, int i) {
    if (!(V.open[c] == 1 && V.type[c] != LBM_FS_GAS && V.fill[c] > FILL_LO)) return false;
    int wet = 0, res = 0;
    const float othr = V.P.vof_orphan_empty_threshold;
    const int maxw = V.P.vof_detached_max_wet_neighbors, maxr = V.P.vof_detached_max_resolved_neighbors;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        int n;
        if (!vnbr(V.D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n) || V.open[n] != 1) continue;
        if (V.type[n] != LBM_FS_GAS) {
            wet++;
            if (V.fill[n] >= othr) res++;
            if (wet > maxw || res > maxr) return false;   // the counts only grow
        }
    }
    return true;
}
// vof_gas_neighbor_rate, CODEX.py:1813-1832
LBM_DEV float gas_rate(const VofArgs &V, int k, int j, int i, int di, int dj, int dk, float rate) {
    if (!(rate > 0.0f)) return 0.0f;
    int n;
    if (!vnbr(V.D, V.P.x_solid, k, j, i, di, dj, dk, n)) return 0.0f;
    if (V.open[n] == 1 && V.type[n] == LBM_FS_GAS) return rate;
    return 0.0f;
}

// advect_detached_vof_cells (compress = 0, CODEX.py:1861-1914) and
// compress_detached_vof_residuals (compress = 1, 1917-1993): decision pass.
// mv[6c+e] = mass moved from donor c along e = +x,-x,+y,-y,+z,-z.
__global__ void k_vof_detached_donor(VofArgs V, int compress, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    bool counted = false;
    if (c < (int)D.n) {
        float *mv = V.fa + 6 * (size_t)c;
        int8_t *isd = V.ba;
        double moved_total = 0.0;
        int k, j, i;
        vkji(D, c, k, j, i);
        const bool det = detached_cell(V, c, k, j, i);
        isd[c] = det ? 1 : 0;
        if (det) {
            // the apply pass reads the moved masses of detached cells only
#pragma unroll
            for (int e = 0; e < 6; ++e) mv[e] = 0.0f;
            const float m = V.mass[c];
            const float vx = V.ux[c], vy = V.uy[c], vz = V.uz[c];
            float r[6];
            if (!compress) {
                if (m > VOF_E12) {
                    r[0] = gas_rate(V, k, j, i, 1, 0, 0, vx);
                    r[1] = gas_rate(V, k, j, i, -1, 0, 0, -vx);
                    r[2] = gas_rate(V, k, j, i, 0, 1, 0, vy);
                    r[3] = gas_rate(V, k, j, i, 0, -1, 0, -vy);
                    r[4] = gas_rate(V, k, j, i, 0, 0, 1, vz);
                    r[5] = gas_rate(V, k, j, i, 0, 0, -1, -vz);
                    const float rs = r[0] + r[1] + r[2] + r[3] + r[4] + r[5];
                    if (rs > VOF_E12) {
                        float scale = 1.0f;
                        if (rs > 0.95f) scale = 0.95f / rs;
                        float moved = 0.0f;
#pragma unroll
                        for (int e = 0; e < 6; ++e) {
                            if (r[e] > 0.0f) {
                                const float mvd = m * r[e] * scale;
                                mv[e] = mvd;
                                moved += mvd;
                            }
                        }
                        if (moved > VOF_E12) {
                            counted = true;
                            moved_total = (double)moved;
                        }
                    }
                }
            } else {
                const float rr = rho_ref(V, c);
                const float fl = m / rr;
                if (fl > FILL_LO && fl < V.P.vof_detached_residual_fill_threshold) {
                    r[0] = gas_rate(V, k, j, i, 1, 0, 0, vx);
                    r[1] = gas_rate(V, k, j, i, -1, 0, 0, -vx);
                    r[2] = gas_rate(V, k, j, i, 0, 1, 0, vy);
                    r[3] = gas_rate(V, k, j, i, 0, -1, 0, -vy);
                    r[4] = gas_rate(V, k, j, i, 0, 0, 1, vz);
                    r[5] = gas_rate(V, k, j, i, 0, 0, -1, -vz);
                    int best = -1;
                    float br = 0.0f;
#pragma unroll
                    for (int e = 0; e < 6; ++e)
                        if (r[e] > br) { br = r[e]; best = e; }
                    if (br > VOF_E12 && best >= 0) {
                        const float mvd = m * 1.0f * 1.0f;
                        mv[best] = mvd;
                        if (mvd > VOF_E12) {
                            counted = true;
                            moved_total = (double)mvd;
                        }
                    }
                }
            }
        }
        V.dd[c] = moved_total;
    }
    add_count(cnt, counted);
}

// receiver pass: donors lose what they send, other cells gather in e order
__global__ void k_vof_detached_apply(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (c >= (int)D.n) return;
    const int8_t *isd = V.ba;
    const int DI[6] = {1, -1, 0, 0, 0, 0}, DJ[6] = {0, 0, 1, -1, 0, 0}, DK[6] = {0, 0, 0, 0, 1, -1};
    float d = 0.0f;
    if (isd[c]) {
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const float m = V.fa[6 * (size_t)c + e];
            if (m > VOF_E12) d += -m;
        }
    } else {
        int k, j, i;
        vkji(D, c, k, j, i);
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            int s;
            if (!vnbr(D, V.P.x_solid, k, j, i, -DI[e], -DJ[e], -DK[e], s)) continue;
            if (!isd[s]) continue;
            int sk, sj, si;
            vkji(D, s, sk, sj, si);
            int chk;
            if (!vnbr(D, V.P.x_solid, sk, sj, si, DI[e], DJ[e], DK[e], chk) || chk != c) continue;
            const float m = V.fa[6 * (size_t)s + e];
            if (m > VOF_E12) d += m;
        }
    }
    if (fabsf(d) > VOF_E12) V.mass[c] += d;
}

// FP64 256-wide pairwise tree (lbm_tree_sum): one level
__global__ void __launch_bounds__(256) k_tree_level(const double *in, long long len, double *out) {
    __shared__ double a[256];
    const int t = threadIdx.x;
    const long long idx = (long long)blockIdx.x * 256 + t;
    a[t] = idx < len ? in[idx] : 0.0;
    for (int s = 128; s >= 1; s >>= 1) {
        __syncthreads();
        if (t < s) a[t] = a[t] + a[t + s];
    }
    if (t == 0) out[blockIdx.x] = a[0];
}
// float counter slot <- (float) sum
__global__ void k_store_sum(const double *sum, float *dst) { *dst = (float)*sum; }

// vof_gas_fraction_at, CODEX.py:1996-2008
LBM_DEV float gas_fraction(const VofArgs &V, int c) {
    float g = 0.0f;
    if (V.open[c] == 1) {
        if (V.type[c] == LBM_FS_GAS) g = 1.0f;
        else if (V.fill[c] < 1.0f) {
            g = 1.0f - V.fill[c];
            if (g < 0.0f) g = 0.0f;
            if (g > 1.0f) g = 1.0f;
        }
    }
    return g;
}

// collapse: flood-fill seeds (top row) and one Jacobi level of the
// 6-connected search (distance s -> s + 1); equals the capped BFS of the
// reference's propagate_vof_exterior_gas_marks (CODEX.py:2021-2054)
__global__ void k_vof_flood_seed(VofArgs V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)V.D.n) return;
    const int k = c / (int)V.D.a;
    V.dist[c] = (k == V.D.nz - 1 && gas_fraction(V, c) > VOF_E6) ? 0 : -1;
}
__global__ void k_vof_flood_level(VofArgs V, int s, int *maxlev) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int)V.D.n) return;
    if (V.dist[c] >= 0 || !(gas_fraction(V, c) > VOF_E6)) return;
    int k, j, i;
    vkji(V.D, c, k, j, i);
    bool hit = false;
#pragma unroll
    for (int q = 1; q < 7; ++q) {
        int n;
        if (!vnbr(V.D, V.P.x_solid, k, j, i, cxq(q), cyq(q), czq(q), n)) continue;
        if (V.dist[n] == s) hit = true;
    }
    if (hit) {
        V.dist[c] = s + 1;
        atomicMax(maxlev, s + 1);
    }
}
// summarize_vof_trapped_gas_collapse, first tree level of the three FP64
// sums (trapped mass, trapped volume, exterior capacity)
__global__ void __launch_bounds__(256) k_vof_collapse_sums(VofArgs V, double *outm, double *outv, double *outc) {
    __shared__ double a[3][256];
    const int t = threadIdx.x;
    const long long c = (long long)blockIdx.x * 256 + t;
    double tm = 0.0, tv = 0.0, tc = 0.0;
    if (c < (long long)V.D.n) {
        const float g = gas_fraction(V, (int)c);
        if (g > VOF_E6) {
            if (V.dist[c] < 0) {
                const float rr = rho_ref(V, (int)c);
                const float dx = V.P.dx;
                tm = (double)(g * rr);
                tv = (double)(g * dx * dx * dx);
            } else if (V.type[c] != LBM_FS_GAS) {
                const float m = V.mass[c];
                if (m > 0.0f) tc = (double)m;
            }
        }
    }
    a[0][t] = tm;
    a[1][t] = tv;
    a[2][t] = tc;
    for (int s = 128; s >= 1; s >>= 1) {
        __syncthreads();
        if (t < s) {
            a[0][t] = a[0][t] + a[0][t + s];
            a[1][t] = a[1][t] + a[1][t + s];
            a[2][t] = a[2][t] + a[2][t + s];
        }
    }
    if (t == 0) {
        outm[blockIdx.x] = a[0][0];
        outv[blockIdx.x] = a[1][0];
        outc[blockIdx.x] = a[2][0];
    }
}
// the collapse decision: candidate and applied figures, removal scale
__global__ void k_vof_collapse_decide(const double *sm, const double *sv, const double *sc, float maxvol,
                                      float *fcount) {
    const float cm = (float)*sm, cv = (float)*sv, cp = (float)*sc;
    fcount[3] = cm;
    fcount[0] = cv;
    fcount[4] = cp;
    fcount[1] = 0.0f;
    fcount[2] = 0.0f;
    if (cv > 0.0f && cv <= maxvol && cp >= cm && cp > VOF_E12) {
        fcount[1] = cv;
        fcount[2] = cm / cp;
    }
}
// apply_vof_trapped_gas_collapse, CODEX.py:2098-2126
__global__ void k_vof_collapse_apply(VofArgs V, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool counted = false;
    if (c < (int)V.D.n) {
        const float scale = V.fcount[2];
        if (scale > 0.0f) {
            const float g = gas_fraction(V, c);
            if (g > VOF_E6) {
                const float rr = rho_ref(V, c);
                if (V.dist[c] < 0) {
                    V.mass[c] = rr;
                    V.fill[c] = 1.0f;
                    V.type[c] = LBM_FS_LIQUID;
                    counted = true;
                } else if (V.type[c] != LBM_FS_GAS) {
                    float m = V.mass[c] * (1.0f - scale);
                    if (m < 0.0f) m = 0.0f;
                    float fl = m / rr;
                    int8_t ct = LBM_FS_INTERFACE;
                    if (fl <= FILL_LO) { fl = 0.0f; m = 0.0f; ct = LBM_FS_GAS; }
                    else if (fl >= FILL_HI) { fl = 1.0f; m = rr; ct = LBM_FS_LIQUID; }
                    V.mass[c] = m;
                    V.fill[c] = fl;
                    V.type[c] = ct;
                }
            }
        }
    }
    add_count(cnt, counted);
}

// update_free_surface_height_from_vof, CODEX.py:2146-2161 (k in order)
__global__ void k_vof_height(VofArgs V) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    if (a >= (int)D.a) return;
    const float ho = V.fs_h[a];
    float depth = 0.0f;
    for (int k = 0; k < D.nz; ++k) {
        const int c = k * (int)D.a + a;
        if (V.open[c] == 1) depth += V.fill[c] * V.lf0[c] * V.P.dx;
    }
    V.fs_h_last[a] = ho;
    V.fs_h[a] = V.bed_h[a] + depth;
}

// repair_vof_coalescence_links, CODEX.py:2319-2373.  A source has
// type_prev == GAS and a repaired cell type_prev != GAS, so sources are
// never rewritten: the kernel is race-free.
template <int S>
__global__ void k_vof_coalesce(VofArgs V, int *cnt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const Dom &D = V.D;
    int reps = 0;
    int k = 0, j = 0, i = 0;
    if (c < (int)D.n) vkji(D, c, k, j, i);
    // vof_near: a cell that turned wet lies within one cell (marked by k_refill_vof_mark)
    if (c < (int)D.n && V.open[c] == 1 && V.type[c] != LBM_FS_GAS && V.type_prev[c] != LBM_FS_GAS &&
        vof_near(V, k, j, i)) {
        typename Store<S>::T *f = (typename Store<S>::T *)V.f;
#pragma unroll
        for (int q = 1; q < 19; ++q) {
            int sir = i - cxq(q);
            int si = sir;
            int sj = (j - cyq(q) + D.ny) % D.ny;
            int sk = k - czq(q);
            bool sv = true;
            if (!V.P.x_solid) si = (sir + D.nx) % D.nx;
            else if (sir < 0 || sir >= D.nx) sv = false;
            if (sk < 0 || sk >= D.nz) sv = false;
            if (!sv) continue;
            const int s = D.cell(sk, sj, si);
            if (V.open[s] == 1 && V.type_prev[s] == LBM_FS_GAS && V.type[s] != LBM_FS_GAS) {
                f[(size_t)q * D.n + c] = f[(size_t)q * D.n + s];
                reps++;
            }
        }
        if (reps) {
            float rn = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const float fq = Store<S>::ld_rw(f, (size_t)q * D.n + c, q, V.P.rho0);
                rn += fq;
                mx += fq * (float)cxq(q);
                my += fq * (float)cyq(q);
                mz += fq * (float)czq(q);
            }
            V.rho[c] = rn;
            if (rn > VOF_E8) {
                V.ux[c] = mx / rn;
                V.uy[c] = my / rn;
                V.uz[c] = mz / rn;
            }
        }
    }
    const unsigned m = __activemask();
    const int s = __reduce_add_sync(m, reps);
    if ((threadIdx.x & 31) == (__ffs(m) - 1) && s) atomicAdd(cnt, s);
}

// exterior labels of the last collapse pass (0 before any)
__global__ void k_vof_exterior(int n, const int *dist, int32_t *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) out[c] = dist[c] >= 0 ? 1 : 0;
}

}  // namespace lbm
