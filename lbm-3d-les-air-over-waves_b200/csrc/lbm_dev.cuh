// lbm_dev.cuh - device helpers of the B200 D3Q19 step engine.
//
// Every expression that produces a value stored in the state follows the
// operation order of the reference kernel it restates
// (LBM_3D_LES_air_over_waves_CODEX.py, cited as CODEX.py:line); the library
// is compiled with -fmad=false so no multiply-add is contracted.  Terms
// multiplied by a lattice-velocity component that is zero are dropped at
// compile time: x + (0*y) equals x except for the sign of a zero, which no
// later operation distinguishes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "lbm_b200.h"
#include "lbm_mathfn.h"

#define LBM_DEV __device__ __forceinline__

namespace lbm {

// Solver constants of every live context, for device code that is not
// inlined into a kernel (the near-wall paths).  Inlined code reads the
// copy passed by value in the kernel arguments instead.  Global memory
// (cached reads), so that a process can hold many contexts at once
// (batched ensembles, served requests).
#define LBM_MAX_SLOTS 1024
#ifdef LBM_DEVICE_TU
__device__ lbm_params c_params[LBM_MAX_SLOTS];
#elif defined(LBM_AUX_TU)
// translation units without near-wall paths: the out-of-line helpers that
// name c_params are compiled but never called there
__device__ lbm_params c_params[1];
#endif

// f32 constants of the collision kernels (CODEX.py:3165-3171, 3326-3328),
// evaluated exactly as Taichi does in f32: c_s2 = f32(1/3),
// inv_2cs4 = 1/(2*c_s2*c_s2) in f32 arithmetic = 4.4999995,
// 1/tau_sponge = 1/f32(0.95) in f32 arithmetic.
#define LBM_CS2 0.333333343267440796f
#define LBM_INV_2CS4 4.49999952316284180f
#define LBM_OM_SPONGE 1.05263161659240723f

// ---------------------------------------------------------------- lattice
// D3Q19 in the order of lbm_lattice.py:3-43, as constexpr functions so that
// unrolled loops fold them into immediates.
__host__ __device__ constexpr int cxq(int q) {
    return (q == 1 || q == 7 || q == 10 || q == 11 || q == 14) ? 1
         : (q == 2 || q == 8 || q == 9 || q == 12 || q == 13) ? -1 : 0;
}
__host__ __device__ constexpr int cyq(int q) {
    return (q == 3 || q == 7 || q == 8 || q == 15 || q == 18) ? 1
         : (q == 4 || q == 9 || q == 10 || q == 16 || q == 17) ? -1 : 0;
}
__host__ __device__ constexpr int czq(int q) {
    return (q == 5 || q == 11 || q == 12 || q == 15 || q == 16) ? 1
         : (q == 6 || q == 13 || q == 14 || q == 17 || q == 18) ? -1 : 0;
}
__host__ __device__ constexpr int oppq(int q) {
    return q == 0 ? 0 : (q <= 6 ? (q & 1 ? q + 1 : q - 1)
                       : (q <= 10 ? (q <= 8 ? q + 2 : q - 2)
                       : (q <= 14 ? (q <= 12 ? q + 2 : q - 2) : (q <= 16 ? q + 2 : q - 2))));
}
// mirror of q in z (free-slip top): same (cx, cy), opposite cz
__host__ __device__ constexpr int mirzq(int q) {
    return q == 5 ? 6 : q == 6 ? 5 : q == 11 ? 14 : q == 14 ? 11 : q == 12 ? 13 : q == 13 ? 12
         : q == 15 ? 18 : q == 18 ? 15 : q == 16 ? 17 : q == 17 ? 16 : q;
}
LBM_DEV float wq(int q) {
    return q == 0 ? (float)(1.0 / 3.0) : (q <= 6 ? (float)(1.0 / 18.0) : (float)(1.0 / 36.0));
}

// c . u with zero terms dropped, keeping the reference's left-to-right
// grouping ((cx*ux + cy*uy) + cz*uz)
template <int Q>
LBM_DEV float cdot(float vx, float vy, float vz) {
    constexpr int a = cxq(Q), b = cyq(Q), c = czq(Q);
    float s;
    bool have = false;
    s = 0.0f;
    if (a != 0) { s = a > 0 ? vx : -vx; have = true; }
    if (b != 0) { float t = b > 0 ? vy : -vy; s = have ? __fadd_rn(s, t) : t; have = true; }
    if (c != 0) { float t = c > 0 ? vz : -vz; s = have ? __fadd_rn(s, t) : t; have = true; }
    return s;
}

// calculate_feq, CODEX.py:623-643
template <int Q>
LBM_DEV float feq(float r, float vx, float vy, float vz, float u2) {
    float cu = 3.0f * cdot<Q>(vx, vy, vz);
    return r * wq(Q) * (1.0f + cu + 0.5f * cu * cu - 1.5f * u2);
}
LBM_DEV float usq(float vx, float vy, float vz) { return vx * vx + vy * vy + vz * vz; }

LBM_DEV int pymod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// ------------------------------------------------------- population storage
// F32: plain.  F16S / BF16S: shifted populations f - w_q*rho0 stored in 16
// bits, arithmetic in f32.  FP16 stores the shifted value times 2^8: the
// shifted values of slow or nearly hydrostatic flow (w_q (rho - rho0) of
// order 1e-5) would otherwise fall below FP16's normal range (6.1e-5) and
// lose relative precision; scaling by a power of two is exact both ways and
// still leaves |f - w_q rho0| up to 255 representable.  BF16 has FP32's
// exponent range and is stored unscaled.
#define LBM_F16_SCALE 256.0f
#define LBM_F16_UNSCALE 0.00390625f
template <int S> struct Store;
template <> struct Store<LBM_STORE_F32> {
    typedef float T;
    static LBM_DEV float ld(const float *p, size_t i, int, float) { return __ldg(p + i); }
    static LBM_DEV float ld_rw(const float *p, size_t i, int, float) { return p[i]; }
    static LBM_DEV void st(float *p, size_t i, float v, int, float) { p[i] = v; }
};
template <> struct Store<LBM_STORE_F16S> {
    typedef __half T;
    static LBM_DEV float ld(const __half *p, size_t i, int q, float rho0) {
        return __half2float(__ldg(p + i)) * LBM_F16_UNSCALE + wq(q) * rho0;
    }
    static LBM_DEV float ld_rw(const __half *p, size_t i, int q, float rho0) {
        return __half2float(p[i]) * LBM_F16_UNSCALE + wq(q) * rho0;
    }
    static LBM_DEV void st(__half *p, size_t i, float v, int q, float rho0) {
        p[i] = __float2half_rn((v - wq(q) * rho0) * LBM_F16_SCALE);
    }
};
template <> struct Store<LBM_STORE_BF16S> {
    typedef __nv_bfloat16 T;
    static LBM_DEV float ld(const __nv_bfloat16 *p, size_t i, int q, float rho0) {
        return __bfloat162float(__ldg(p + i)) + wq(q) * rho0;
    }
    static LBM_DEV float ld_rw(const __nv_bfloat16 *p, size_t i, int q, float rho0) {
        return __bfloat162float(p[i]) + wq(q) * rho0;
    }
    static LBM_DEV void st(__nv_bfloat16 *p, size_t i, float v, int q, float rho0) {
        p[i] = __float2bfloat16_rn(v - wq(q) * rho0);
    }
};

// ------------------------------------------------------------- domain view
struct Dom {
    int nx, ny, nz;
    size_t n;   // cells (< 2^31)
    size_t a;   // columns
    LBM_DEV int cell(int k, int j, int i) const { return (k * ny + j) * nx + i; }
    LBM_DEV int col(int j, int i) const { return j * nx + i; }
};

// 2-D bed state of one step
struct BedView {
    const float *h;      // water_h (bed height)
    const float *hmax;   // max of h over the 3x3 column neighbourhood
    const float *uw, *vw, *ww;
    const float *cg;     // per-column link-endpoint cache (bed-only geometry), or null
};
// components of the column cache, [component][column]
enum { CG_ETA = 0, CG_UW = 9, CG_DEN = 36, CG_N = 37 };

// free-surface view (height path derives cell states from the column height)
struct FsView {
    const float *h;        // free_surface_h used for classification
    const float *h_last;   // previous height (refill detection)
    const float *fill;     // stored fill (VOF)
    const int8_t *type;    // stored type (VOF)
};

}  // namespace lbm
