// lbm_fast.cuh - the fast arithmetic policy of the interior kernels.
//
// Same physics as ArExact (macro_step, compute_LES without the wall model,
// collide_regularized / collide_KBC of CODEX.py:2943-3416 for a plain
// interior air cell), reorganised for fewer instructions; compiled in its
// own translation unit with multiply-add contraction (reciprocals and square
// roots stay correctly rounded).  Results differ from the reference's
// operation order by rounding only.
//
// Pair form.  D3Q19 velocities come in nine opposite pairs (q, q') with
// c_q' = -c_q and equal weights.  For a pair,
//   feq_q  = A + B,  feq_q' = A - B,
//   A = rho w (1 - 1.5 u.u + 4.5 (c.u)^2),  B = 3 rho w (c.u),
// and the regularized non-equilibrium part w/(2 cs^4) Q_q:Pi is the same for
// q and q' (Q_q = c_q c_q - cs^2 I is even in c).  Pi, the second moment of
// f - feq, needs only the pair sums f_q + f_q' - 2A.  So the collision
// evaluates one A, B and Hermite projection per pair instead of one
// equilibrium and one projection per direction.  The positivity limiter
// (alpha, eps = 1e-6) is evaluated only when some post-collision value
// falls below eps, with the reference's semantics.
#pragma once

#include "lbm_tile.cuh"

namespace lbm {

// the nine pairs: representative q (listed first in lbm_lattice.py order
// among its pair) and its opposite
#define LBM_PAIRS(X) X(0, 1, 2) X(1, 3, 4) X(2, 5, 6) X(3, 7, 9) X(4, 8, 10) X(5, 11, 13) X(6, 12, 14) X(7, 15, 17) X(8, 16, 18)

// c . u of the representative of pair p
template <int Q>
LBM_DEV float pair_cu(float vx, float vy, float vz) {
    constexpr int a = cxq(Q), b = cyq(Q), c = czq(Q);
    float s = 0.0f;
    if (a > 0) s = vx; else if (a < 0) s = -vx;
    if (b > 0) s = s + vy; else if (b < 0) s = s - vy;
    if (c > 0) s = s + vz; else if (c < 0) s = s - vz;
    return s;
}

// the reference's positivity limiter on fsv given feq (rare path)
LBM_DEV void fast_limit(const float fe[19], float f[19]) {
    const float eps = 1e-6f;
    float alpha = 1.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (f[q] < eps) {
            const float den = f[q] - fe[q];
            if (den < 0.0f) {
                const float cand = (eps - fe[q]) / den;
                if (cand < alpha) alpha = cand;
            }
        }
    }
    if (alpha < 0.0f) alpha = 0.0f;
    if (alpha > 1.0f) alpha = 1.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = fe[q] + alpha * (f[q] - fe[q]);
}

template <int COLL>
struct ArFast {
    static LBM_DEV void macro(const lbm_params &P_, const Dom &D_, const float f[19], int k_, float &r, float &vx,
                              float &vy, float &vz) {
#ifdef LBM_FAST_EXACT_MACRO
        // the reference's summation order (sums only: nothing to contract)
        ArExact::macro(P_, D_, f, k_, r, vx, vy, vz);
        return;
#endif
        const float d1 = f[1] - f[2], d3 = f[3] - f[4], d5 = f[5] - f[6], d7 = f[7] - f[9], d8 = f[8] - f[10];
        const float d11 = f[11] - f[13], d12 = f[12] - f[14], d15 = f[15] - f[17], d16 = f[16] - f[18];
        const float s0 = (f[0] + f[1]) + (f[2] + f[3]) + (f[4] + f[5]) + (f[6] + f[7]);
        const float s1 = (f[8] + f[9]) + (f[10] + f[11]) + (f[12] + f[13]) + (f[14] + f[15]);
        const float s2 = (f[16] + f[17]) + f[18];
        r = (s0 + s1) + s2;
        const float jx = (d1 + d7) + (d11 - d8) - d12;
        const float jy = (d3 + d7) + (d8 + d15) - d16;
        const float jz = (d5 + d11) + (d12 + d15) + d16;
        const float inv = 1.0f / r;
        vx = jx * inv;
        vy = jy * inv;
        vz = jz * inv;
    }

    static LBM_DEV float les(const lbm_params &P, float uxp, float uxm, float uyp, float uym, float uzp, float uzm,
                             float vxp, float vxm, float vyp, float vym, float vzp, float vzm, float wxp, float wxm,
                             float wyp, float wym, float wzp, float wzm) {
        // central differences without their factor 1/2: S_ii = a/2,
        // S_ij = (b + c)/4, so 2 S:S = (sum a^2 + 0.5 sum (b + c)^2) / 2
        const float axx = uxp - uxm, ayy = vyp - vym, azz = wzp - wzm;
        const float bxy = (uyp - uym) + (vxp - vxm);
        const float bxz = (uzp - uzm) + (wxp - wxm);
        const float byz = (vzp - vzm) + (wyp - wym);
        const float diag = axx * axx + ayy * ayy + azz * azz;
        const float off = bxy * bxy + bxz * bxz + byz * byz;
        const float x = 0.5f * diag + 0.25f * off + 1e-6f;   // 2 S:S + 1e-6
        const float smag = sqrtf(x);
        const float nu_t = fminf(P.cs_delta_sq * smag, P.nu_t_max);
        const float tau = fminf(0.5f + 3.0f * (P.nu0 + nu_t), 2.0f);
        return 1.0f / tau;
    }

    static LBM_DEV void collide(const StepArgs &A, int c, int k, float r, float vx, float vy, float vz, float om,
                                float f[19]) {
        const lbm_params &P = A.P;
        if (COLL == LBM_COLLIDE_KBC && (P.c_backscatter > 0.0f || (P.enable_top_sponge && k > A.D.nz - 3))) {
            // stochastic backscatter and the top sponge: the reference arithmetic
            lbm::collide<COLL>(A, c, k, false, false, false, 0.0f, r, vx, vy, vz, om, f);
            return;
        }
        const float u2 = vx * vx + vy * vy + vz * vz;
        const float K = 1.0f - 1.5f * u2;
        const float rw0 = r * (1.0f / 3.0f), rw1 = r * (1.0f / 18.0f), rw2 = r * (1.0f / 36.0f);
        float Ap[9], Bp[9];
#define LBM_AB(p, q, qb)                                                \
    {                                                                   \
        const float cu = pair_cu<q>(vx, vy, vz);                        \
        const float rw = (q <= 6) ? rw1 : rw2;                          \
        Ap[p] = rw * (K + 4.5f * cu * cu);                              \
        Bp[p] = (3.0f * rw) * cu;                                       \
    }
        LBM_PAIRS(LBM_AB)
#undef LBM_AB
        const float A0 = rw0 * K;
        float fe[19];
        bool low = false;
        if (COLL == LBM_COLLIDE_REGULARIZED) {
            float Dp[9];
#define LBM_D(p, q, qb) Dp[p] = (f[q] + f[qb]) - 2.0f * Ap[p];
            LBM_PAIRS(LBM_D)
#undef LBM_D
            // pairs: 0 x, 1 y, 2 z, 3 (1,1,0), 4 (-1,1,0), 5 (1,0,1), 6 (-1,0,1), 7 (0,1,1), 8 (0,-1,1)
            const float sxy = Dp[3] + Dp[4], sxz = Dp[5] + Dp[6], syz = Dp[7] + Dp[8];
            const float Pxx = Dp[0] + sxy + sxz, Pyy = Dp[1] + sxy + syz, Pzz = Dp[2] + sxz + syz;
            const float Pxy = Dp[3] - Dp[4], Pxz = Dp[5] - Dp[6], Pyz = Dp[7] - Dp[8];
            const float t3 = (Pxx + Pyy + Pzz) * (1.0f / 3.0f);
            const float hx = Pxx - t3, hy = Pyy - t3, hz = Pzz - t3;
            const float exy = hx + Pyy, exz = hx + Pzz, eyz = hy + Pzz;
            float h[9];
            h[0] = hx; h[1] = hy; h[2] = hz;
            h[3] = exy + 2.0f * Pxy; h[4] = exy - 2.0f * Pxy;
            h[5] = exz + 2.0f * Pxz; h[6] = exz - 2.0f * Pxz;
            h[7] = eyz + 2.0f * Pyz; h[8] = eyz - 2.0f * Pyz;
            const float omc = (1.0f - om) * LBM_INV_2CS4;   // the reference's f32 value of 1 / (2 cs^4)
            const float g1 = omc * (1.0f / 18.0f), g2 = omc * (1.0f / 36.0f);
            f[0] = A0 - (omc * (1.0f / 3.0f)) * t3;
            fe[0] = A0;
#define LBM_OUT(p, q, qb)                                               \
    {                                                                   \
        const float C = Ap[p] + ((q <= 6) ? g1 : g2) * h[p];            \
        f[q] = C + Bp[p];                                               \
        f[qb] = C - Bp[p];                                              \
        fe[q] = Ap[p] + Bp[p];                                          \
        fe[qb] = Ap[p] - Bp[p];                                         \
    }
            LBM_PAIRS(LBM_OUT)
#undef LBM_OUT
        } else {
            // BGK relaxation of the KBC path, f - om (f - feq)
            fe[0] = A0;
            f[0] = f[0] + om * (A0 - f[0]);
#define LBM_BGK(p, q, qb)                                               \
    {                                                                   \
        fe[q] = Ap[p] + Bp[p];                                          \
        fe[qb] = Ap[p] - Bp[p];                                         \
        f[q] = f[q] + om * (fe[q] - f[q]);                              \
        f[qb] = f[qb] + om * (fe[qb] - f[qb]);                          \
    }
            LBM_PAIRS(LBM_BGK)
#undef LBM_BGK
        }
        float m = f[0];
#pragma unroll
        for (int q = 1; q < 19; ++q) m = fminf(m, f[q]);
        low = m < 1e-6f;
        if (low) fast_limit(fe, f);
    }
};

}  // namespace lbm
