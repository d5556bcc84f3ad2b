// lbm_tile.cuh - the interior step kernel: one pass per step over the
// planes that are provably away from every wall.
//
// A block owns a 16x16 column tile and marches up a chunk of z planes.  For
// every plane it gathers the post-stream populations of its 256 cells
// (pull from the previous step's post-collision state, or the stored
// post-stream state for the first step of a call), takes the moments, and
// publishes the velocity of the cells and of the 64-cell ring around the
// tile (recomputed by 64 threads) to shared memory.  Once plane p is
// published, plane p-1 has its full 7-point velocity stencil: LES, then
// collision, then the post-collision populations go to HBM.  So each step
// reads every population once and writes it once (plus the ring re-reads,
// served by L2); the velocity never round-trips through HBM.
//
// Preconditions, established by the host: air mode without free surface,
// periodic x without the x fringe, nx and ny multiples of 16, and every
// plane in [zi0, zi1] far from the bed (the bed amplitude bounds the bed
// height) so no link there is cut and no cell below is solid.  The kernel
// re-checks the geometry of its cells and sets status bit 1 if a
// precondition fails.
#pragma once

#include <cuda.h>   // CUtensorMap (the type only; nothing links the driver library)

#include "lbm_stages.cuh"

namespace lbm {

// compute_LES without the wall model (the cell below is fluid by the
// preconditions), from a 7-point stencil
LBM_DEV float les_interior(const lbm_params &P, float uxp, float uxm, float uyp, float uym, float uzp, float uzm,
                           float vxp, float vxm, float vyp, float vym, float vzp, float vzm, float wxp, float wxm,
                           float wyp, float wym, float wzp, float wzm) {
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
    float nu_eff = P.nu0 + nu_t;
    float tau_eff = 0.5f + 3.0f * nu_eff;
    if (tau_eff > 2.0f) tau_eff = 2.0f;
    return 1.0f / tau_eff;
}

// Arithmetic of the interior kernels' per-cell stages (moments, LES rate,
// collision).  ArExact: the reference's operation order (the stages shared
// with the general kernels), bit-equal to the CPU oracle.  A faster policy
// with the same interface lives in lbm_fast.cuh.
struct ArExact {
    static LBM_DEV void macro(const lbm_params &P, const Dom &D, const float f[19], int k, float &r, float &vx,
                              float &vy, float &vz) {
        lbm::macro(P, D, f, k, false, LBM_FS_LIQUID, 0.0f, r, vx, vy, vz);
    }
    static LBM_DEV float les(const lbm_params &P, float uxp, float uxm, float uyp, float uym, float uzp, float uzm,
                             float vxp, float vxm, float vyp, float vym, float vzp, float vzm, float wxp, float wxm,
                             float wyp, float wym, float wzp, float wzm) {
        return les_interior(P, uxp, uxm, uyp, uym, uzp, uzm, vxp, vxm, vyp, vym, vzp, vzm, wxp, wxm, wyp, wym, wzp,
                            wzm);
    }
    static LBM_DEV void collide(const StepArgs &A, int c, int k, float r, float vx, float vy, float vz, float om,
                                float f[19]) {
        lbm::collide(A, c, k, false, false, false, 0.0f, r, vx, vy, vz, om, f);
    }
};

// populations entering the collide step for an interior cell
template <int S, int IN>
LBM_DEV void interior_front(const StepArgs &A, int k, int j, int i, float f[19]) {
    const int c = A.D.cell(k, j, i);
    if (IN == 0) {
        const typename Store<S>::T *src = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = Store<S>::ld(src, (size_t)q * A.D.n + (size_t)c, q, A.P.rho0);
    } else {
        stream_fast<S>(A, (const typename Store<S>::T *)A.fsrc, k, j, i, c, f);
    }
}

__constant__ int c_tile_cx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
__constant__ int c_tile_cy[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1};
__constant__ int c_tile_cz[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};

// ring cell r (0..63) around a 16x16 tile: rows below/above, columns left/right
LBM_DEV void ring_cell(int r, int &rx, int &ry) {
    if (r < 16) { rx = r; ry = -1; }
    else if (r < 32) { rx = r - 16; ry = LBM_TILE; }
    else if (r < 48) { rx = -1; ry = r - 32; }
    else { rx = LBM_TILE; ry = r - 48; }
}

// populations entering the collide step for the 64 ring cells of plane p,
// gathered by all 256 threads (item m = (q, r) with q = m / 64) into
// ringf[q][r]
template <int S, int IN>
LBM_DEV void ring_gather(const StepArgs &A, int p, int t, float (*ringf)[64]) {
    const Dom &D = A.D;
    const typename Store<S>::T *src = (const typename Store<S>::T *)A.fsrc;
#pragma unroll
    for (int u = 0; u < 5; ++u) {
        const int m = t + 256 * u;
        if (m < 64 * 19) {
            const int r = m & 63, q = m >> 6;
            int rx, ry;
            ring_cell(r, rx, ry);
            int si = blockIdx.x * LBM_TILE + rx, sj = blockIdx.y * LBM_TILE + ry, sk = p;
            if (IN == 1) {
                si -= c_tile_cx[q];
                sj -= c_tile_cy[q];
                sk -= c_tile_cz[q];
            }
            si = (si + 2 * D.nx) % D.nx;
            sj = (sj + 2 * D.ny) % D.ny;
            const size_t idx = (size_t)q * D.n + (size_t)D.cell(sk, sj, si);
            float v;
            if (S == LBM_STORE_F32) v = __ldg((const float *)src + idx);
            else v = Store<S>::ld(src, idx, q, A.P.rho0);
            ringf[q][r] = v;
        }
    }
}

LBM_DEV void check_far(const StepArgs &A, bool stream_geo, int k, int j, int i) {
    bool ok = geo_far(A.P, A.D, A.bed_c, k, j, i);
    if (stream_geo) ok = ok && geo_far(A.P, A.D, A.bed_s, k, j, i);
    if (!ok) atomicOr(A.status, 2u);
}

template <int S, int IN, bool LES>
__global__ void __launch_bounds__(256, 2) k_tile(StepArgs A) {
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int i = blockIdx.x * LBM_TILE + tx, j = blockIdx.y * LBM_TILE + ty;
    const int z0 = A.zi0 + blockIdx.z * A.chunk;
    const int z1 = min(z0 + A.chunk, A.zi1 + 1);  // planes [z0, z1) are collided here
    __shared__ float su[3][3][LBM_TILE + 2][LBM_TILE + 2];  // [plane slot][component][x][y]
    __shared__ float ringf[LES ? 19 : 1][64];               // ring populations of the current plane

    // ring cell whose moments this thread takes (threads 0..63)
    int rx = 0, ry = 0;
    ring_cell(t & 63, rx, ry);
    const int ri = (blockIdx.x * LBM_TILE + rx + D.nx) % D.nx;
    const int rj = (blockIdx.y * LBM_TILE + ry + D.ny) % D.ny;
    const bool ring = LES && t < 64;

    float fp[19];
    float rp = 0.0f, vxp = 0.0f, vyp = 0.0f, vzp = 0.0f;
    const size_t n = D.n;
    for (int p = z0 - 1; p <= z1; ++p) {
        const int sl = p % 3;
        const bool interior = p >= A.zi0 && p <= A.zi1;
        float fc[19];
        float r = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
        if (interior) {
            interior_front<S, IN>(A, p, j, i, fc);
            macro(P, D, fc, p, false, LBM_FS_LIQUID, 0.0f, r, vx, vy, vz);
            if (LES) {
                su[sl][0][tx + 1][ty + 1] = vx;
                su[sl][1][tx + 1][ty + 1] = vy;
                su[sl][2][tx + 1][ty + 1] = vz;
            }
            if (LES) ring_gather<S, IN>(A, p, t, ringf);
        } else if (LES) {
            // plane handled by the general kernels: velocity from their pre-pass
            const int c = D.cell(p, j, i);
            su[sl][0][tx + 1][ty + 1] = __ldg(A.u_les + c);
            su[sl][1][tx + 1][ty + 1] = __ldg(A.u_les + n + c);
            su[sl][2][tx + 1][ty + 1] = __ldg(A.u_les + 2 * n + c);
            if (ring) {
                const int cr = D.cell(p, rj, ri);
                su[sl][0][rx + 1][ry + 1] = __ldg(A.u_les + cr);
                su[sl][1][rx + 1][ry + 1] = __ldg(A.u_les + n + cr);
                su[sl][2][rx + 1][ry + 1] = __ldg(A.u_les + 2 * n + cr);
            }
        }
        if (LES) __syncthreads();
        if (LES && interior) {
            // moments of the ring cells from the cooperatively gathered populations
            if (ring) {
                float fr[19], rr, a, b, d;
#pragma unroll
                for (int q = 0; q < 19; ++q) fr[q] = ringf[q][t];
                macro(P, D, fr, p, false, LBM_FS_LIQUID, 0.0f, rr, a, b, d);
                su[sl][0][rx + 1][ry + 1] = a;
                su[sl][1][rx + 1][ry + 1] = b;
                su[sl][2][rx + 1][ry + 1] = d;
            }
            // (no barrier: the collide below reads other threads' velocities
            // only in plane p - 1; plane p's are read from the next iteration)
        }
        const int k = p - 1;
        if (k >= z0 && k < z1) {
            const int c = D.cell(k, j, i);
            check_far(A, IN == 1, k, j, i);
            if (k == A.zi0) check_far(A, IN == 1, k - 1, j, i);
            float om = P.omega0;
            if (LES) {
                const int sm = (p + 1) % 3, s0 = (p + 2) % 3, sp = sl;  // planes k-1, k, k+1
                const int y = ty + 1, x = tx + 1;
                om = les_interior(P, su[s0][0][x + 1][y], su[s0][0][x - 1][y], su[s0][0][x][y + 1],
                                  su[s0][0][x][y - 1], su[sp][0][x][y], su[sm][0][x][y], su[s0][1][x + 1][y],
                                  su[s0][1][x - 1][y], su[s0][1][x][y + 1], su[s0][1][x][y - 1], su[sp][1][x][y],
                                  su[sm][1][x][y], su[s0][2][x + 1][y], su[s0][2][x - 1][y], su[s0][2][x][y + 1],
                                  su[s0][2][x][y - 1], su[sp][2][x][y], su[sm][2][x][y]);
                if (A.flags & F_WRITE_ALL_OMEGA) A.omega[c] = om;
                if (k == A.zi0 || k == A.zi1) {
                    // velocity of the interior planes next to the general ones,
                    // for the general kernels' stencils
                    A.u_out[c] = vxp;
                    A.u_out[n + c] = vyp;
                    A.u_out[2 * n + c] = vzp;
                }
            }
            if (A.flags & F_WRITE_MACRO) {
                A.rho[c] = rp; A.ux[c] = vxp; A.uy[c] = vyp; A.uz[c] = vzp;
            }
            if (!(rp == rp) || fabsf(rp) > 3.0e38f) atomicOr(A.status, 1u);
            collide(A, c, k, false, false, false, 0.0f, rp, vxp, vyp, vzp, om, fp);
            typename Store<S>::T *dst = (typename Store<S>::T *)A.fdst;
#pragma unroll
            for (int q = 0; q < 19; ++q) Store<S>::st(dst, (size_t)q * n + (size_t)c, fp[q], q, P.rho0);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) fp[q] = fc[q];
        rp = r; vxp = vx; vyp = vy; vzp = vz;
        if (LES) __syncthreads();
    }
}

// ------------------------------------------------- pipelined interior kernel
// k_tile_pipe: k_tile for FP32 populations with the gathers of plane p + 2
// in flight while plane p is worked on.  Each thread copies its own cell's
// 19 pulled populations (and 4-5 ring items) straight into shared memory
// with cp.async (4-byte copies, no registers held), in a ring of 3 plane
// slots; a commit group per plane keeps the waits in order.  Per-column
// work is hoisted out of the z loop: source offsets, the ring items'
// addresses, and the far-from-the-bed check (monotone in k, so the lowest
// plane of the chunk decides).  Arithmetic, and so every result, is that of
// k_tile.
constexpr int PIPE_SLOTS = 3;
constexpr int PIPE_SMEM_FLOATS =
    PIPE_SLOTS * 19 * 256 + PIPE_SLOTS * 19 * 64 + 3 * 3 * (LBM_TILE + 2) * (LBM_TILE + 2);
constexpr int PIPE_SMEM_BYTES = PIPE_SMEM_FLOATS * 4;

LBM_DEV void cp_async4(float *smem, const float *gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
LBM_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
LBM_DEV void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int IN, bool LES, class Ar = ArExact>
LBM_DEV void tile_pipe_body(const StepArgs &A, float *smem, int bx, int by, int bz) {
    float *sf = smem;                                   // [slot][q][256] own-cell populations
    float *sr = smem + PIPE_SLOTS * 19 * 256;           // [slot][q][64] ring populations
    float (*su)[3][LBM_TILE + 2][LBM_TILE + 2] =        // [plane slot][component][x][y]
        (float (*)[3][LBM_TILE + 2][LBM_TILE + 2])(sr + PIPE_SLOTS * 19 * 64);
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int i = bx * LBM_TILE + tx, j = by * LBM_TILE + ty;
    const int z0 = A.zi0 + bz * A.chunk;
    const int z1 = min(z0 + A.chunk, A.zi1 + 1);  // planes [z0, z1) are collided here
    const int n = (int)D.n, nxy = D.nx * D.ny;
    const float *fsrc = (const float *)A.fsrc;
    float *fdst = (float *)A.fdst;

    // far-from-the-bed precondition of this column (status bit 1)
    {
        const int kc = max(z0, A.zi0);
        bool ok = geo_far(P, D, A.bed_c, kc, j, i) && (IN == 0 || geo_far(P, D, A.bed_s, kc, j, i));
        if (z0 == A.zi0)
            ok = ok && geo_far(P, D, A.bed_c, z0 - 1, j, i) && (IN == 0 || geo_far(P, D, A.bed_s, z0 - 1, j, i));
        if (!ok) atomicOr(A.status, 2u);
    }
    // neighbour offsets of the pull gather (periodic x and y)
    const int col = j * D.nx + i;
    const int xm = (i == 0) ? D.nx - 1 : -1, xp = (i + 1 == D.nx) ? 1 - D.nx : 1;
    const int ym = (j == 0) ? (D.ny - 1) * D.nx : -D.nx, yp = (j + 1 == D.ny) ? (1 - D.ny) * D.nx : D.nx;
    // ring items of this thread: ring cell r = t & 63, q = (t >> 6) + 4u
    int rx = 0, ry = 0;
    ring_cell(t & 63, rx, ry);
    const int ri = (bx * LBM_TILE + rx + D.nx) % D.nx;
    const int rj = (by * LBM_TILE + ry + D.ny) % D.ny;
    int roff[5];
#pragma unroll
    for (int u = 0; u < 5; ++u) {
        const int q = (t >> 6) + 4 * u;
        int si = ri, sj = rj, dz = 0;
        if (q < 19) {
            if (IN == 1) {
                si -= c_tile_cx[q];
                sj -= c_tile_cy[q];
                dz = -c_tile_cz[q];
            }
            si = si < 0 ? si + D.nx : (si >= D.nx ? si - D.nx : si);
            sj = sj < 0 ? sj + D.ny : (sj >= D.ny ? sj - D.ny : sj);
        }
        roff[u] = q * n + dz * nxy + sj * D.nx + si;
    }
    const bool ring = LES && t < 64;

    // copies of plane p into slot p % 3 (own cell, and the ring with LES)
    auto issue = [&](int p) {
        if (p >= A.zi0 && p <= A.zi1 && p <= z1) {
            const int slot = p % PIPE_SLOTS;
            const int base = p * nxy + col;
            float *dst = sf + slot * 19 * 256 + t;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                int off = 0;
                if (IN == 1) {
                    if (cxq(q) > 0) off += xm; else if (cxq(q) < 0) off += xp;
                    if (cyq(q) > 0) off += ym; else if (cyq(q) < 0) off += yp;
                    if (czq(q) > 0) off -= nxy; else if (czq(q) < 0) off += nxy;
                }
                cp_async4(dst + q * 256, fsrc + (q * n + base + off));
            }
            if (LES) {
                float *rdst = sr + slot * 19 * 64 + (t & 63);
#pragma unroll
                for (int u = 0; u < 5; ++u) {
                    const int q = (t >> 6) + 4 * u;
                    if (q < 19) cp_async4(rdst + q * 64, fsrc + (roff[u] + p * nxy));
                }
            }
        }
        cp_async_commit();
    };

    issue(z0 - 1);
    issue(z0);
    float fp[19];
    float rp = 0.0f, vxp = 0.0f, vyp = 0.0f, vzp = 0.0f;
    for (int p = z0 - 1; p <= z1; ++p) {
        const int sl = p % 3;
        const bool interior = p >= A.zi0 && p <= A.zi1;
        cp_async_wait1();       // plane p has landed (p + 1 may still be in flight)
        __syncthreads();        // ring items of plane p come from other threads
        float fc[19];
        float r = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
        if (interior) {
            const float *src = sf + sl * 19 * 256 + t;
#pragma unroll
            for (int q = 0; q < 19; ++q) fc[q] = src[q * 256];
        }
        issue(p + 2);           // into the slot consumed before the barrier above
        if (interior) {
            Ar::macro(P, D, fc, p, r, vx, vy, vz);
            if (LES) {
                su[sl][0][tx + 1][ty + 1] = vx;
                su[sl][1][tx + 1][ty + 1] = vy;
                su[sl][2][tx + 1][ty + 1] = vz;
                if (ring) {
                    const float *rs = sr + sl * 19 * 64 + t;
                    float fr[19], rr, a, b, d;
#pragma unroll
                    for (int q = 0; q < 19; ++q) fr[q] = rs[q * 64];
                    Ar::macro(P, D, fr, p, rr, a, b, d);
                    su[sl][0][rx + 1][ry + 1] = a;
                    su[sl][1][rx + 1][ry + 1] = b;
                    su[sl][2][rx + 1][ry + 1] = d;
                }
            }
        } else if (LES) {
            // plane handled by the general kernels: velocity from their pre-pass
            const int c = p * nxy + col;
            su[sl][0][tx + 1][ty + 1] = __ldg(A.u_les + c);
            su[sl][1][tx + 1][ty + 1] = __ldg(A.u_les + n + c);
            su[sl][2][tx + 1][ty + 1] = __ldg(A.u_les + 2 * n + c);
            if (ring) {
                const int cr = (p * D.ny + rj) * D.nx + ri;
                su[sl][0][rx + 1][ry + 1] = __ldg(A.u_les + cr);
                su[sl][1][rx + 1][ry + 1] = __ldg(A.u_les + n + cr);
                su[sl][2][rx + 1][ry + 1] = __ldg(A.u_les + 2 * n + cr);
            }
        }
        // No barrier here: the collide of plane p - 1 reads other threads'
        // velocities only in plane p - 1 (published in the previous
        // iteration, ordered by the barrier above); planes p and p - 2 are
        // read at the thread's own column, written by the thread itself.
        const int k = p - 1;
        if (k >= z0 && k < z1) {
            const int c = k * nxy + col;
            float om = P.omega0;
            if (LES) {
                const int sm = (p + 1) % 3, s0 = (p + 2) % 3, sp = sl;  // planes k-1, k, k+1
                const int y = ty + 1, x = tx + 1;
                om = Ar::les(P, su[s0][0][x + 1][y], su[s0][0][x - 1][y], su[s0][0][x][y + 1],
                                  su[s0][0][x][y - 1], su[sp][0][x][y], su[sm][0][x][y], su[s0][1][x + 1][y],
                                  su[s0][1][x - 1][y], su[s0][1][x][y + 1], su[s0][1][x][y - 1], su[sp][1][x][y],
                                  su[sm][1][x][y], su[s0][2][x + 1][y], su[s0][2][x - 1][y], su[s0][2][x][y + 1],
                                  su[s0][2][x][y - 1], su[sp][2][x][y], su[sm][2][x][y]);
                if (A.flags & F_WRITE_ALL_OMEGA) A.omega[c] = om;
                if (k == A.zi0 || k == A.zi1) {
                    // velocity of the interior planes next to the general ones,
                    // for the general kernels' stencils
                    A.u_out[c] = vxp;
                    A.u_out[n + c] = vyp;
                    A.u_out[2 * n + c] = vzp;
                }
            }
            if (A.flags & F_WRITE_MACRO) {
                A.rho[c] = rp; A.ux[c] = vxp; A.uy[c] = vyp; A.uz[c] = vzp;
            }
            if (!(rp == rp) || fabsf(rp) > 3.0e38f) atomicOr(A.status, 1u);
            Ar::collide(A, c, k, rp, vxp, vyp, vzp, om, fp);
#pragma unroll
            for (int q = 0; q < 19; ++q) fdst[q * n + c] = fp[q];
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) fp[q] = fc[q];
        rp = r; vxp = vx; vyp = vy; vzp = vz;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <int IN, bool LES>
__global__ void __launch_bounds__(256, 2) k_tile_pipe(StepArgs A) {
    extern __shared__ __align__(16) float smem[];
    tile_pipe_body<IN, LES>(A, smem, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ------------------------------------------- pipelined 16-bit interior kernel
// k_tile_pipe16: k_tile_pipe for shifted FP16/BF16 populations.  cp.async
// copies at least 4 bytes, so the block copies aligned pairs of 16-bit
// values: for each population and tile row the 9 pairs x0 .. x0+17 (x0-2 ..
// x0+15 for the populations pulled from x - 1), in which every cell of the
// row finds its pulled value; the ring rows likewise, and for the two ring
// columns the pair that holds each value.  Values are widened with the
// storage's own conversion (Store<S>::ld) when read from shared memory.
constexpr int P16_ROWW = 9;                              // words (pairs) per staged row
constexpr int P16_MAIN = 19 * 16 * P16_ROWW;             // words per plane slot
constexpr int P16_RROW = 19 * 2 * P16_ROWW;              // ring rows, words
constexpr int P16_RCOL = 19 * 2 * 16;                    // ring columns, words
constexpr int P16_RING = P16_RROW + P16_RCOL;
constexpr int P16_SMEM_BYTES =
    (PIPE_SLOTS * P16_MAIN + PIPE_SLOTS * P16_RING) * 4 + 3 * 3 * (LBM_TILE + 2) * (LBM_TILE + 2) * 4;

LBM_DEV void cp_async4v(void *smem, const void *gmem) {
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
LBM_DEV int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <int S, int IN, bool LES, class Ar = ArExact>
LBM_DEV void tile_pipe16_body(const StepArgs &A, float *smem, int bx, int by, int bz) {
    typedef typename Store<S>::T T;
    uint32_t *sw = (uint32_t *)smem;                     // [slot][P16_MAIN] words
    uint32_t *rw = sw + PIPE_SLOTS * P16_MAIN;           // [slot][P16_RING] words
    float (*su)[3][LBM_TILE + 2][LBM_TILE + 2] =         // [plane slot][component][x][y]
        (float (*)[3][LBM_TILE + 2][LBM_TILE + 2])(rw + PIPE_SLOTS * P16_RING);
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int x0 = bx * LBM_TILE, y0 = by * LBM_TILE;
    const int i = x0 + tx, j = y0 + ty;
    const int z0 = A.zi0 + bz * A.chunk;
    const int z1 = min(z0 + A.chunk, A.zi1 + 1);  // planes [z0, z1) are collided here
    const int n = (int)D.n, nxy = D.nx * D.ny;
    const T *fsrc = (const T *)A.fsrc;
    T *fdst = (T *)A.fdst;
    {
        const int kc = max(z0, A.zi0);
        bool ok = geo_far(P, D, A.bed_c, kc, j, i) && (IN == 0 || geo_far(P, D, A.bed_s, kc, j, i));
        if (z0 == A.zi0)
            ok = ok && geo_far(P, D, A.bed_c, z0 - 1, j, i) && (IN == 0 || geo_far(P, D, A.bed_s, z0 - 1, j, i));
        if (!ok) atomicOr(A.status, 2u);
    }
    const int col = j * D.nx + i;
    int rx = 0, ry = 0;
    ring_cell(t & 63, rx, ry);
    const int ri = (x0 + rx + D.nx) % D.nx;
    const int rj = (y0 + ry + D.ny) % D.ny;
    const bool ring = LES && t < 64;

    // copies of plane p into slot p % 3
    auto issue = [&](int p) {
        if (p >= A.zi0 && p <= A.zi1 && p <= z1) {
            const int slot = p % PIPE_SLOTS;
            uint32_t *dst = sw + slot * P16_MAIN;
#pragma unroll
            for (int v = 0; v < (P16_MAIN + 255) / 256; ++v) {
                const int m = t + 256 * v;
                if (m < P16_MAIN) {
                    const int q = m / (16 * P16_ROWW), r = m - q * (16 * P16_ROWW);
                    const int row = r / P16_ROWW, pr = r - row * P16_ROWW;
                    const int cx = IN ? c_tile_cx[q] : 0, cy = IN ? c_tile_cy[q] : 0, cz = IN ? c_tile_cz[q] : 0;
                    const int xs = cx > 0 ? x0 - 2 : x0;
                    const int sx = wrapi(xs + 2 * pr, D.nx), sy = wrapi(y0 + row - cy, D.ny);
                    cp_async4v(dst + m, fsrc + ((size_t)q * n + (size_t)(p - cz) * nxy + (size_t)sy * D.nx + sx));
                }
            }
            if (LES) {
                uint32_t *rdst = rw + slot * P16_RING;
#pragma unroll
                for (int v = 0; v < (P16_RING + 255) / 256; ++v) {
                    const int m = t + 256 * v;
                    if (m < P16_RROW) {
                        const int q = m / (2 * P16_ROWW), r2 = m - q * (2 * P16_ROWW);
                        const int side = r2 / P16_ROWW, pr = r2 - side * P16_ROWW;
                        const int cx = IN ? c_tile_cx[q] : 0, cy = IN ? c_tile_cy[q] : 0, cz = IN ? c_tile_cz[q] : 0;
                        const int xs = cx > 0 ? x0 - 2 : x0;
                        const int sx = wrapi(xs + 2 * pr, D.nx);
                        const int sy = wrapi((side ? y0 + LBM_TILE : y0 - 1) - cy, D.ny);
                        cp_async4v(rdst + m, fsrc + ((size_t)q * n + (size_t)(p - cz) * nxy + (size_t)sy * D.nx + sx));
                    } else if (m < P16_RING) {
                        const int m2 = m - P16_RROW;
                        const int q = m2 / 32, r2 = m2 - q * 32;
                        const int side = r2 / 16, rr = r2 - side * 16;
                        const int cx = IN ? c_tile_cx[q] : 0, cy = IN ? c_tile_cy[q] : 0, cz = IN ? c_tile_cz[q] : 0;
                        const int sx = wrapi((side ? x0 + LBM_TILE : x0 - 1) - cx, D.nx) & ~1;
                        const int sy = wrapi(y0 + rr - cy, D.ny);
                        cp_async4v(rdst + m, fsrc + ((size_t)q * n + (size_t)(p - cz) * nxy + (size_t)sy * D.nx + sx));
                    }
                }
            }
        }
        cp_async_commit();
    };

    issue(z0 - 1);
    issue(z0);
    float fp[19];
    float rp = 0.0f, vxp = 0.0f, vyp = 0.0f, vzp = 0.0f;
    for (int p = z0 - 1; p <= z1; ++p) {
        const int sl = p % 3;
        const bool interior = p >= A.zi0 && p <= A.zi1;
        cp_async_wait1();       // plane p has landed (p + 1 may still be in flight)
        __syncthreads();        // the staged rows come from other threads
        float fc[19];
        float r = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
        if (interior) {
            const T *sb = (const T *)(sw + sl * P16_MAIN);
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int off = (IN && cxq(q) != 0) ? 1 : 0;
                fc[q] = Store<S>::ld_rw(sb, (size_t)(q * 16 * 2 * P16_ROWW + ty * 2 * P16_ROWW + tx + off), q, P.rho0);
            }
        }
        float frr[19];
        if (interior && ring) {
            const T *rb = (const T *)(rw + sl * P16_RING);
            const int rr = t;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int cx = IN ? cxq(q) : 0;
                size_t e;
                if (rr < 32) {
                    const int side = rr >> 4, rx2 = rr & 15;
                    e = (size_t)(q * 2 * 2 * P16_ROWW + side * 2 * P16_ROWW + rx2 + (cx != 0 ? 1 : 0));
                } else {
                    const int side = (rr - 32) >> 4, ry2 = rr & 15;
                    const int sx = wrapi((side ? x0 + LBM_TILE : x0 - 1) - cx, D.nx);
                    e = (size_t)(2 * P16_RROW + 2 * (q * 32 + side * 16 + ry2) + (sx & 1));
                }
                frr[q] = Store<S>::ld_rw(rb, e, q, P.rho0);
            }
        }
        issue(p + 2);           // into the slot consumed before the barrier above
        if (interior) {
            Ar::macro(P, D, fc, p, r, vx, vy, vz);
            if (LES) {
                su[sl][0][tx + 1][ty + 1] = vx;
                su[sl][1][tx + 1][ty + 1] = vy;
                su[sl][2][tx + 1][ty + 1] = vz;
                if (ring) {
                    float rr2, a, b, d;
                    Ar::macro(P, D, frr, p, rr2, a, b, d);
                    su[sl][0][rx + 1][ry + 1] = a;
                    su[sl][1][rx + 1][ry + 1] = b;
                    su[sl][2][rx + 1][ry + 1] = d;
                }
            }
        } else if (LES) {
            // plane handled by the general kernels: velocity from their pre-pass
            const int c = p * nxy + col;
            su[sl][0][tx + 1][ty + 1] = __ldg(A.u_les + c);
            su[sl][1][tx + 1][ty + 1] = __ldg(A.u_les + n + c);
            su[sl][2][tx + 1][ty + 1] = __ldg(A.u_les + 2 * n + c);
            if (ring) {
                const int cr = (p * D.ny + rj) * D.nx + ri;
                su[sl][0][rx + 1][ry + 1] = __ldg(A.u_les + cr);
                su[sl][1][rx + 1][ry + 1] = __ldg(A.u_les + n + cr);
                su[sl][2][rx + 1][ry + 1] = __ldg(A.u_les + 2 * n + cr);
            }
        }
        // no barrier: other threads' velocities are read one plane back
        const int k = p - 1;
        if (k >= z0 && k < z1) {
            const int c = k * nxy + col;
            float om = P.omega0;
            if (LES) {
                const int sm = (p + 1) % 3, s0 = (p + 2) % 3, sp = sl;  // planes k-1, k, k+1
                const int y = ty + 1, x = tx + 1;
                om = Ar::les(P, su[s0][0][x + 1][y], su[s0][0][x - 1][y], su[s0][0][x][y + 1],
                                  su[s0][0][x][y - 1], su[sp][0][x][y], su[sm][0][x][y], su[s0][1][x + 1][y],
                                  su[s0][1][x - 1][y], su[s0][1][x][y + 1], su[s0][1][x][y - 1], su[sp][1][x][y],
                                  su[sm][1][x][y], su[s0][2][x + 1][y], su[s0][2][x - 1][y], su[s0][2][x][y + 1],
                                  su[s0][2][x][y - 1], su[sp][2][x][y], su[sm][2][x][y]);
                if (A.flags & F_WRITE_ALL_OMEGA) A.omega[c] = om;
                if (k == A.zi0 || k == A.zi1) {
                    A.u_out[c] = vxp;
                    A.u_out[n + c] = vyp;
                    A.u_out[2 * n + c] = vzp;
                }
            }
            if (A.flags & F_WRITE_MACRO) {
                A.rho[c] = rp; A.ux[c] = vxp; A.uy[c] = vyp; A.uz[c] = vzp;
            }
            if (!(rp == rp) || fabsf(rp) > 3.0e38f) atomicOr(A.status, 1u);
            Ar::collide(A, c, k, rp, vxp, vyp, vzp, om, fp);
#pragma unroll
            for (int q = 0; q < 19; ++q) Store<S>::st(fdst, (size_t)q * n + (size_t)c, fp[q], q, P.rho0);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) fp[q] = fc[q];
        rp = r; vxp = vx; vyp = vy; vzp = vz;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <int S, int IN, bool LES>
__global__ void __launch_bounds__(256, 2) k_tile_pipe16(StepArgs A) {
    extern __shared__ __align__(16) float smem[];
    tile_pipe16_body<S, IN, LES>(A, smem, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ------------------------------------------------ TMA-staged interior kernel
// k_tile_tma: the fused step (pull from the previous step's post-collision
// state) with LES for FP32 populations, staged by the tensor memory
// accelerator.  For population q one 4-D tile copy (x, y, z, q) brings the
// box x in [xs, xs + W), y in [y0 - 1 - cy, y0 + 17 - cy), plane p - cz into
// shared memory: it holds the pulled value of each tile cell and of each ring
// cell (x0 - 1 .. x0 + 16 before the shift by -cx).  W = 24 from xs = x0 - 4
// when cx = 0; W = 20 from xs = x0 - 4 (cx = 1) or xs = x0 (cx = -1), so x
// coordinates stay multiples of 4 floats (16 bytes) and each box starts on a
// 128-byte boundary of its slot.  Lane 0 of each warp issues 2 or 3 of the
// 19 copies of a plane into a ring of 3 slots, each completing on its own
// mbarrier; no other thread spends instructions on addresses or copies.  Plane
// p + 1 is copied while plane p is worked on, and the populations of plane
// p - 1 are read again from their slot when it is collided (registers stay
// at 96, no spills).  A tile copy cannot wrap the periodic x and y
// boundaries, so this kernel covers the tiles off the domain edge, and
// k_tile_edges (the cp.async-staged body of k_tile_pipe) the ring of edge
// tiles.  This grid is launched behind k_tile_edges as a programmatic
// dependent, so its blocks fill the SMs that grid's tail leaves idle.
// Arithmetic, and so every result, is that of k_tile.
constexpr int TMA_H = LBM_TILE + 2;                    // box rows
constexpr int TMA_REG24 = 448, TMA_REG20 = 384;        // floats per population (24x18, 20x18, padded to 128 B)
__host__ __device__ constexpr unsigned tma_cx0_mask(int q = 0) {
    return q == 19 ? 0u : (((cxq(q) == 0) ? 1u : 0u) << q) | tma_cx0_mask(q + 1);
}
__host__ __device__ constexpr int popc32(unsigned v) {   // no loop or call: folds for a constant argument
    const unsigned a = v - ((v >> 1) & 0x55555555u);
    const unsigned b = (a & 0x33333333u) + ((a >> 2) & 0x33333333u);
    return (int)((((b + (b >> 4)) & 0x0F0F0F0Fu) * 0x01010101u) >> 24);
}
__host__ __device__ constexpr int tma_shift(int q) {   // box column of tile x = 0
    return cxq(q) == 0 ? 4 : (cxq(q) > 0 ? 3 : 1);
}
constexpr unsigned TMA_CX0 = tma_cx0_mask();
__host__ __device__ constexpr int tma_base(int q) {    // floats before population q in a slot
    return TMA_REG20 * q + (TMA_REG24 - TMA_REG20) * popc32(TMA_CX0 & ((1u << q) - 1u));
}
constexpr int TMA_SLOT = tma_base(19);                 // floats per plane slot
constexpr unsigned TMA_BYTES = 9u * 24u * TMA_H * 4u + 10u * 20u * TMA_H * 4u;   // bytes landing per plane
constexpr int TMA_SMEM_BYTES = 128 + PIPE_SLOTS * TMA_SLOT * 4 + 3 * 3 * (LBM_TILE + 2) * (LBM_TILE + 2) * 4 +
                               PIPE_SLOTS * 8;
constexpr int TMA_WAIT_LIMIT = 1 << 22;                // try_wait rounds before a wait gives up (status bit 2)
static_assert(TMA_SLOT == 9 * TMA_REG24 + 10 * TMA_REG20, "slot layout");
static_assert(tma_base(1) == TMA_REG24 && tma_base(3) == TMA_REG24 + 2 * TMA_REG20 && tma_base(18) == 8 * TMA_REG24 + 10 * TMA_REG20,
              "population offsets");
static_assert((TMA_REG24 * 4) % 128 == 0 && (TMA_REG20 * 4) % 128 == 0, "boxes start on 128-byte boundaries");

// Layout of a plane slot.  FP32: boxes 24 or 20 values wide (tma_base,
// tma_shift above).  16-bit storage: one box of 32 x 18 values per
// population from x0 - 8 (16-byte aligned x), 1,152 bytes, which covers the
// columns x0 - 2 .. x0 + 17 that any shift needs.
constexpr int TMA16_W = 32, TMA16_REG = TMA16_W * TMA_H;
template <int S> struct TmaTile {   // FP16 / BF16 shifted populations
    typedef typename Store<S>::T T;
    static constexpr int SLOT = 19 * TMA16_REG;                 // values per slot
    static constexpr unsigned BYTES = 19u * TMA16_REG * 2u;     // bytes landing per plane
    static constexpr int WA = TMA16_W, WB = TMA16_W;            // the two row pitches (one here)
    static LBM_DEV int base(int q) { return q * TMA16_REG; }
    static LBM_DEV int x_start(int x0, int) { return x0 - 8; }
    __host__ __device__ static constexpr int shift(int q) { return 8 - cxq(q); }
    __host__ __device__ static constexpr bool wide(int) { return true; }   // row pitch WA
};
template <> struct TmaTile<LBM_STORE_F32> {
    typedef float T;
    static constexpr int SLOT = TMA_SLOT;
    static constexpr unsigned BYTES = TMA_BYTES;
    static constexpr int WA = 24, WB = 20;
    static LBM_DEV int base(int q) { return tma_base(q); }
    static LBM_DEV int x_start(int x0, int cx) { return cx < 0 ? x0 : x0 - 4; }
    __host__ __device__ static constexpr int shift(int q) { return tma_shift(q); }
    __host__ __device__ static constexpr bool wide(int q) { return cxq(q) == 0; }
};
template <int S>
constexpr int tma_smem_bytes() {
    return 128 + PIPE_SLOTS * TmaTile<S>::SLOT * (int)sizeof(typename TmaTile<S>::T) +
           3 * 3 * (LBM_TILE + 2) * (LBM_TILE + 2) * 4 + PIPE_SLOTS * 8;
}
static_assert((TMA16_REG * 2) % 128 == 0, "16-bit boxes start on 128-byte boundaries");
static_assert(tma_smem_bytes<LBM_STORE_F32>() == TMA_SMEM_BYTES, "FP32 slot layout");

LBM_DEV unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
LBM_DEV void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
LBM_DEV void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
LBM_DEV bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}
LBM_DEV void tma_load_4d(unsigned dst, const CUtensorMap *map, int x, int y, int z, int w, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
        : "memory");
}

LBM_DEV void mbar_inval(unsigned bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}

// One tile (x0, y0) and z chunk bz of the fused interior step staged by tile
// copies (the body of k_tile_tma, also run per work item by the ensemble's
// kb_tile_tma).  m24 / m20: tensor maps of the source populations (kernel
// parameters).  false: a wait gave up (status bit 2 set, the block's copies
// in flight waited for); the caller leaves.
template <int S, class Ar>
LBM_DEV bool tile_tma_body(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20,
                           unsigned char *tma_smem, int x0, int y0, int bz) {
    typedef TmaTile<S> L;
    typedef typename L::T T;
    T *sf = (T *)(tma_smem + ((128u - (smem_addr(tma_smem) & 127u)) & 127u));   // [slot][L::SLOT]
    float (*su)[3][LBM_TILE + 2][LBM_TILE + 2] =        // [plane slot][component][x][y]
        (float (*)[3][LBM_TILE + 2][LBM_TILE + 2])(sf + PIPE_SLOTS * L::SLOT);
    uint64_t *bar = (uint64_t *)((float *)(sf + PIPE_SLOTS * L::SLOT) + 3 * 3 * (LBM_TILE + 2) * (LBM_TILE + 2));
    const lbm_params &P = A.P;
    const Dom &D = A.D;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int i = x0 + tx, j = y0 + ty;
    const int z0 = A.zi0 + bz * A.chunk;
    const int z1 = min(z0 + A.chunk, A.zi1 + 1);  // planes [z0, z1) are collided here
    const int n = (int)D.n, nxy = D.nx * D.ny;
    T *fdst = (T *)A.fdst;
    {
        const int kc = max(z0, A.zi0);
        bool ok = geo_far(P, D, A.bed_c, kc, j, i) && geo_far(P, D, A.bed_s, kc, j, i);
        if (z0 == A.zi0) ok = ok && geo_far(P, D, A.bed_c, z0 - 1, j, i) && geo_far(P, D, A.bed_s, z0 - 1, j, i);
        if (!ok) atomicOr(A.status, 2u);
    }
    const int col = j * D.nx + i;
    int rx = 0, ry = 0;
    ring_cell(t & 63, rx, ry);
    const int ri = (x0 + rx + D.nx) % D.nx;
    const int rj = (y0 + ry + D.ny) % D.ny;
    const bool ring = t < 64;
    if (t == 0) {
        for (int s = 0; s < PIPE_SLOTS; ++s) mbar_init(smem_addr(bar + s), 1u);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();

    // tile copies of plane p into slot p % 3, issued by lane 0 of every warp
    // (populations w, w + 8, w + 16): copies issued by one warp's lanes
    // leave one at a time, those of different warps side by side.  The
    // expected byte count may be posted after some copies have completed
    // (the transaction count goes negative until then; the phase cannot
    // complete before thread 0 has arrived).
    auto issue = [&](int p) {
        if ((t & 31) == 0 && p >= A.zi0 && p <= A.zi1 && p <= z1) {
            const int slot = p % PIPE_SLOTS;
            const unsigned b = smem_addr(bar + slot);
            if (t == 0) mbar_expect_tx(b, L::BYTES);
            for (int q = t >> 5; q < 19; q += 8) {
                tma_load_4d(smem_addr(sf + slot * L::SLOT + L::base(q)), L::wide(q) ? m24 : m20,
                            L::x_start(x0, cxq(q)), y0 - 1 - cyq(q), p - czq(q), q, b);
            }
        }
    };

    // Plane p + 1 is copied while plane p is worked on; the populations of
    // plane p - 1, collided in iteration p, are read again from their slot
    // instead of being held in registers (and its velocity from su).
    issue(z0 - 1);
    unsigned phase = 0u;   // bit s: parity of the next completion of slot s
    float rp = 0.0f;       // density of plane p - 1
    for (int p = z0 - 1; p <= z1; ++p) {
        const int sl = p % 3;
        const bool interior = p >= A.zi0 && p <= A.zi1;
        bool gave_up = false;
        if (interior) {
            // bounded wait for the copies of plane p (F_TEST_WAIT_TIMEOUT:
            // give up at once, to exercise the error path below)
            const unsigned b = smem_addr(bar + sl);
            if (A.flags & F_TEST_WAIT_TIMEOUT) {
                gave_up = true;
            } else {
                int it = 0;
                while (!mbar_try_wait(b, (phase >> sl) & 1u))
                    if (++it == TMA_WAIT_LIMIT) {
                        gave_up = true;
                        break;
                    }
            }
        }
        // slot (p + 1) % 3 is free: every thread is done with plane p - 2
        if (__syncthreads_or(gave_up)) {
            // A wait gave up: status bit 2, and the whole block leaves.  The
            // copies of plane p are the only ones in flight (plane p - 1's
            // completed in the last iteration), so they are waited for first,
            // again with a bound, before the block's shared memory goes away.
            if (t == 0) atomicOr(A.status, 4u);
            const unsigned b = smem_addr(bar + sl);
            for (int it = 0; it < TMA_WAIT_LIMIT && !mbar_try_wait(b, (phase >> sl) & 1u); ++it) {
            }
            return false;
        }
        if (interior) phase ^= 1u << sl;
        issue(p + 1);
        float r = 0.0f;
        const T *sb = sf + sl * L::SLOT;
        if (interior) {
            if (ring) {
                // ring cell: box row ry + 1, column rx + L::shift(q)
                float fr[19], rr, a, b, d;
                const T *bA = sb + (ry + 1) * L::WA + rx, *bB = sb + (ry + 1) * L::WB + rx;
#pragma unroll
                for (int q = 0; q < 19; ++q)
                    fr[q] = Store<S>::ld_rw(L::wide(q) ? bA : bB, (size_t)(L::base(q) + L::shift(q)), q, P.rho0);
                Ar::macro(P, D, fr, p, rr, a, b, d);
                su[sl][0][rx + 1][ry + 1] = a;
                su[sl][1][rx + 1][ry + 1] = b;
                su[sl][2][rx + 1][ry + 1] = d;
            }
            // own cell: box row ty + 1, column tx + L::shift(q)
            float fc[19], vx, vy, vz;
            const T *bA = sb + (ty + 1) * L::WA + tx, *bB = sb + (ty + 1) * L::WB + tx;
#pragma unroll
            for (int q = 0; q < 19; ++q)
                fc[q] = Store<S>::ld_rw(L::wide(q) ? bA : bB, (size_t)(L::base(q) + L::shift(q)), q, P.rho0);
            Ar::macro(P, D, fc, p, r, vx, vy, vz);
            su[sl][0][tx + 1][ty + 1] = vx;
            su[sl][1][tx + 1][ty + 1] = vy;
            su[sl][2][tx + 1][ty + 1] = vz;
        } else {
            // plane handled by the general kernels: velocity from their pre-pass
            const int c = p * nxy + col;
            su[sl][0][tx + 1][ty + 1] = __ldg(A.u_les + c);
            su[sl][1][tx + 1][ty + 1] = __ldg(A.u_les + n + c);
            su[sl][2][tx + 1][ty + 1] = __ldg(A.u_les + 2 * n + c);
            if (ring) {
                const int cr = (p * D.ny + rj) * D.nx + ri;
                su[sl][0][rx + 1][ry + 1] = __ldg(A.u_les + cr);
                su[sl][1][rx + 1][ry + 1] = __ldg(A.u_les + n + cr);
                su[sl][2][rx + 1][ry + 1] = __ldg(A.u_les + 2 * n + cr);
            }
        }
        // no barrier: other threads' velocities are read one plane back
        const int k = p - 1;
        if (k >= z0 && k < z1) {
            const int c = k * nxy + col;
            const int sm = (p + 1) % 3, s0 = (p + 2) % 3, sp = sl;  // planes k-1, k, k+1
            const int y = ty + 1, x = tx + 1;
            const float om = Ar::les(P, su[s0][0][x + 1][y], su[s0][0][x - 1][y], su[s0][0][x][y + 1],
                                          su[s0][0][x][y - 1], su[sp][0][x][y], su[sm][0][x][y], su[s0][1][x + 1][y],
                                          su[s0][1][x - 1][y], su[s0][1][x][y + 1], su[s0][1][x][y - 1],
                                          su[sp][1][x][y], su[sm][1][x][y], su[s0][2][x + 1][y], su[s0][2][x - 1][y],
                                          su[s0][2][x][y + 1], su[s0][2][x][y - 1], su[sp][2][x][y], su[sm][2][x][y]);
            const float vxp = su[s0][0][x][y], vyp = su[s0][1][x][y], vzp = su[s0][2][x][y];
            if (A.flags & F_WRITE_ALL_OMEGA) A.omega[c] = om;
            if (k == A.zi0 || k == A.zi1) {
                // velocity of the interior planes next to the general ones,
                // for the general kernels' stencils
                A.u_out[c] = vxp;
                A.u_out[n + c] = vyp;
                A.u_out[2 * n + c] = vzp;
            }
            if (A.flags & F_WRITE_MACRO) {
                A.rho[c] = rp; A.ux[c] = vxp; A.uy[c] = vyp; A.uz[c] = vzp;
            }
            if (!(rp == rp) || fabsf(rp) > 3.0e38f) atomicOr(A.status, 1u);
            float fp[19];
            const T *pb = sf + s0 * L::SLOT;
            const T *bA = pb + (ty + 1) * L::WA + tx, *bB = pb + (ty + 1) * L::WB + tx;
#pragma unroll
            for (int q = 0; q < 19; ++q)
                fp[q] = Store<S>::ld_rw(L::wide(q) ? bA : bB, (size_t)(L::base(q) + L::shift(q)), q, P.rho0);
            Ar::collide(A, c, k, rp, vxp, vyp, vzp, om, fp);
#pragma unroll
            for (int q = 0; q < 19; ++q) Store<S>::st(fdst, (size_t)(q * n + c), fp[q], q, P.rho0);
        }
        rp = r;
    }
    // every copy has been waited for: retire the barriers before the shared
    // memory is used again (the next work item of a queue)
    __syncthreads();
    if (t == 0)
        for (int s = 0; s < PIPE_SLOTS; ++s) mbar_inval(smem_addr(bar + s));
    return true;
}

template <int S, class Ar = ArExact>
__global__ void __launch_bounds__(256, 2)
    k_tile_tma(StepArgs A, const __grid_constant__ CUtensorMap m24, const __grid_constant__ CUtensorMap m20) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    // tiles off the domain edge
    tile_tma_body<S, Ar>(A, &m24, &m20, tma_smem, (blockIdx.x + 1) * LBM_TILE, (blockIdx.y + 1) * LBM_TILE,
                         blockIdx.z);
    // complete only after the edge-tile grid this one was launched behind,
    // so that the work after it sees both grids' results
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

// tile e of the ring of edge tiles of a TX x TY tiling: the rows by = 0
// and by = TY - 1, then the columns bx = 0 and bx = TX - 1 between them
LBM_DEV void edge_tile(int e, int TX, int TY, int &bx, int &by) {
    if (e < TX) { bx = e; by = 0; return; }
    e -= TX;
    if (TY > 1) {
        if (e < TX) { bx = e; by = TY - 1; return; }
        e -= TX;
    }
    by = 1 + (e >> 1);
    bx = (e & 1) ? TX - 1 : 0;
}

// the fused interior step with LES on the edge tiles (grid.x = their
// count), cp.async-staged (k_tile_pipe's or k_tile_pipe16's body).  k_tile_tma is launched after it as a
// programmatic dependent: it may start as soon as every block of this grid
// is running (the two grids share no output)
template <int S, class Ar = ArExact>
__global__ void __launch_bounds__(256, 2) k_tile_edges(StepArgs A) {
    extern __shared__ __align__(16) float smem[];
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    int bx = 0, by = 0;
    edge_tile(blockIdx.x, A.D.nx / LBM_TILE, A.D.ny / LBM_TILE, bx, by);
    if constexpr (S == LBM_STORE_F32) tile_pipe_body<1, true, Ar>(A, smem, bx, by, blockIdx.z);
    else tile_pipe16_body<S, 1, true, Ar>(A, smem, bx, by, blockIdx.z);
}

// ----------------------------------------------- launch of the fused interior
#ifndef LBM_EDGE_CHUNK_DIV
#define LBM_EDGE_CHUNK_DIV 2
#endif
// the two interior grids take more than 48 KB of shared memory: raise the
// per-kernel limits once per device and arithmetic policy
template <int S, class Ar>
static bool tma_smem_ready_t() {
    static bool done[64] = {false}, ok[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!done[dev]) {
        done[dev] = true;
        const int edge_bytes = S == LBM_STORE_F32 ? PIPE_SMEM_BYTES : P16_SMEM_BYTES;
        ok[dev] = cudaFuncSetAttribute(k_tile_tma<S, Ar>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       tma_smem_bytes<S>()) == cudaSuccess &&
                  cudaFuncSetAttribute(k_tile_edges<S, Ar>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       edge_bytes) == cudaSuccess;
    }
    return ok[dev];
}

// The fused interior step with LES: the edge tiles (cp.async staging), then
// the tiles off the edge (tile copies) as a programmatic dependent launch.
// false: not launched (no tile off the edge, or shared memory refused).
template <int S, class Ar>
static bool launch_tile_tma_t(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st) {
    const int ni = A.zi1 - A.zi0 + 1;
    if (ni <= 0 || A.chunk <= 0) return true;
    const int TX = A.D.nx / LBM_TILE, TY = A.D.ny / LBM_TILE;
    if (TX < 3 || TY < 3 || !tma_smem_ready_t<S, Ar>()) return false;
    const unsigned zc = (unsigned)((ni + A.chunk - 1) / A.chunk);
    const int edge_bytes = S == LBM_STORE_F32 ? PIPE_SMEM_BYTES : P16_SMEM_BYTES;
    // the edge grid marches shorter z chunks: more, shorter blocks, so that
    // its last wave ends sooner and the grid behind it starts sooner
    StepArgs Ae = A;
    Ae.chunk = A.chunk / LBM_EDGE_CHUNK_DIV > 8 ? A.chunk / LBM_EDGE_CHUNK_DIV : (A.chunk < 8 ? A.chunk : 8);
    const unsigned zce = (unsigned)((ni + Ae.chunk - 1) / Ae.chunk);
    k_tile_edges<S, Ar><<<dim3(2 * TX + 2 * TY - 4, 1, zce), 256, edge_bytes, st>>>(Ae);
    // tiles off the edge: a programmatic dependent launch (it may start while
    // the grid above drains; plain stream order when the attribute is refused)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(TX - 2, TY - 2, zc);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = tma_smem_bytes<S>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_tile_tma<S, Ar>, A, *m24, *m20) != cudaSuccess) {
        cudaGetLastError();
        k_tile_tma<S, Ar><<<cfg.gridDim, 256, tma_smem_bytes<S>(), st>>>(A, *m24, *m20);
    }
    launch_count_add(2);
    return true;
}

// stream only (the last pass of a call) for interior cells
template <int S>
LBM_DEV void stream_interior_body(const StepArgs &A, int bx, int by, int bz) {
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int i = bx * LBM_TILE + tx, j = by * LBM_TILE + ty;
    const int k = A.zi0 + bz;
    if (k > A.zi1) return;
    const int c = A.D.cell(k, j, i);
    check_far(A, true, k, j, i);
    float f[19];
    stream_fast<S>(A, (const typename Store<S>::T *)A.fsrc, k, j, i, c, f);
    typename Store<S>::T *dst = (typename Store<S>::T *)A.fdst;
#pragma unroll
    for (int q = 0; q < 19; ++q) Store<S>::st(dst, (size_t)q * A.D.n + (size_t)c, f[q], q, A.P.rho0);
}
template <int S>
__global__ void __launch_bounds__(256) k_stream_interior(StepArgs A) {
    stream_interior_body<S>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

}  // namespace lbm
