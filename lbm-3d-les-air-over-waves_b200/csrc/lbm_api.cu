// lbm_api.cu - C ABI of the B200 D3Q19 step engine (include/lbm_b200.h).
//
// Step orchestration.  The state of record between calls is the caller's
// bound buffers; inside one lbm_step call of K steps:
//
//   air (no free surface): the loop is rotated so that every step is ONE
//   pass over the populations -
//     collide(n+1) from the post-stream state,
//     fused(m -> m+1) = stream+BC of step m, then condition, macro, LES and
//       collide of step m+1, for m = n+1 .. n+K-1,
//     stream(n+K) back to the post-stream state the reference holds after
//       copy_post_and_swap (CODEX.py:3924).
//   With LES, each collide is preceded by a pre-pass that writes the
//   velocity of every cell for the strain-rate stencil.
//
//   height-function free surface: per step collide, stream (+ post-stream
//   macro), column flux, advection, refill (CODEX.py:3873-3925).
//
// The 2-D bed of step m lives in scratch slot m & 1, so the fused pass can
// see the bed of both steps it spans.
#include <cuda.h>
#include <cudaTypedefs.h>   // PFN_cuTensorMapEncodeTiled (resolved at run time: no driver library link)
#include <cuda_runtime.h>

#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "lbm_b200.h"
#include "lbm_launch.h"

using namespace lbm;

namespace {


// constant-memory parameter slots (LBM_MAX_SLOTS live contexts at a time)
std::mutex g_slot_mutex;
bool g_slot_used[LBM_MAX_SLOTS] = {false};

int acquire_slot() {
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    for (int s = 0; s < LBM_MAX_SLOTS; ++s)
        if (!g_slot_used[s]) {
            g_slot_used[s] = true;
            return s;
        }
    return -1;
}
void release_slot(int s) {
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    if (s >= 0 && s < LBM_MAX_SLOTS) g_slot_used[s] = false;
}

}  // namespace

struct lbm_ctx {
    lbm_params P;
    int slot = -1;
    Dom D;
    lbm_buffers b;
    bool bound = false;
    std::string err;
    int cur = 0;
    int64_t nstep = 0;
    cudaStream_t last_stream = 0;
    // scratch owned by the library
    float *bed_h[2] = {nullptr, nullptr}, *bed_hmax[2] = {nullptr, nullptr};
    float *bed_uw[2] = {nullptr, nullptr}, *bed_vw[2] = {nullptr, nullptr}, *bed_ww[2] = {nullptr, nullptr};
    float *bed_cg[2] = {nullptr, nullptr};  // per-column link-endpoint cache (bed-only geometry)
    bool use_cg = false;
    int tile_chunk = 0;   // planes per block of the interior kernel (0: heuristic)
    int arith = LBM_ARITH_EXACT;   // arithmetic of the fused interior grids (lbm_set_arithmetic)
    // VOF scratch (VOF contexts only)
    int8_t *v_open = nullptr, *v_t0 = nullptr, *v_ba = nullptr;
    float *v_lf0 = nullptr, *v_m0 = nullptr, *v_x0 = nullptr, *v_fa = nullptr;
    double *v_dd = nullptr, *v_tree = nullptr;
    uint8_t *v_near = nullptr;   // coarse donor-in-reach flags of the VOF receiver passes
    int *v_dist = nullptr;
    float *u_les = nullptr;
    int *dcount = nullptr;
    unsigned *dstatus = nullptr;
    float *dfcount = nullptr;
    std::vector<void *> owned;
    double bed_bound = 0.0;   // upper bound of the bed height over the run
    // optional per-launch timing of the interior kernel
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // pairs (start, stop)
    size_t ev_used = 0;
    int64_t timed_cells = 0;
    // step graphs (air mode): one captured graph per (steps per call, step parity, current buffer); the kernels
    // of a captured call read the step number from the device clock, set by one launch before each replay
    struct StepGraph {
        int steps, parity, cur, cur_after;
        long long launches;
        cudaGraphExec_t exec;
    };
    bool graphs = false, capturing = false, warm = false;
    int64_t cap_n0 = 0;
    long long *dclock = nullptr;
    float *stash = nullptr;     // FP32 post-condition populations of the general planes (16-bit storage)
    size_t stash_cells = 0;
    int *wlist = nullptr;       // water stream: the cells of the general path ([n]) and their count ([n])
    std::vector<StepGraph> graph_cache;
    // scratch of lbm_diagnostics (allocated by its first call)
    DiagCellPart *d_cellp = nullptr;
    DiagSlicePart *d_slp = nullptr;
    double *d_col_eta = nullptr;
    float *d_col_mm = nullptr;
    double *d_slice = nullptr;
    uint8_t *d_mask = nullptr;
    lbm_diag *d_out = nullptr;
    // tensor maps of f[0] and f[1] for the tile-copy interior kernel: boxes 24x18 and 20x18
    CUtensorMap tmap[2][2];
    void *tmap_src[2] = {nullptr, nullptr};   // buffers the maps were encoded for
    bool tmap_ok = false;
};

static void drop_graphs(lbm_ctx *ctx) {
    for (auto &g : ctx->graph_cache) cudaGraphExecDestroy(g.exec);
    ctx->graph_cache.clear();
}

static void timed_mark(lbm_ctx *ctx, cudaStream_t st) {
    if (ctx->ev_used == ctx->ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->ev.push_back(e);
    }
    cudaEventRecord(ctx->ev[ctx->ev_used++], st);
}

static int fail(lbm_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}
static int cuda_check(lbm_ctx *c, cudaError_t e, const char *what) {
    if (e != cudaSuccess) return fail(c, LBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return LBM_OK;
}
#define CK(expr, what)                                      \
    do {                                                    \
        int _s = cuda_check(ctx, (expr), what);             \
        if (_s != LBM_OK) return _s;                        \
    } while (0)
#define CK_LAUNCH(what) CK(cudaGetLastError(), what)

// Library scratch comes from the stream-ordered allocator: allocation and
// release are ordered on a stream and never synchronise the device, so a
// process that creates and destroys contexts while others run (a request
// server) does not stall their kernels.  Allocations outside a call's
// stream (lbm_bind) are made on the legacy stream and waited for there.
static int alloc(lbm_ctx *ctx, void **p, size_t bytes, cudaStream_t st = 0) {
    CK(cudaMallocAsync(p, bytes, st), "scratch allocation");
    if (st == 0) CK(cudaStreamSynchronize(0), "scratch allocation");
    ctx->owned.push_back(*p);
    return LBM_OK;
}

static inline int64_t P_nx(const lbm_ctx *c) { return c->P.nx; }
static inline int64_t P_ny(const lbm_ctx *c) { return c->P.ny; }

static BedView slot_view(const lbm_ctx *ctx, int s) {
    BedView v;
    v.h = ctx->bed_h[s];
    v.hmax = ctx->bed_hmax[s];
    v.uw = ctx->bed_uw[s];
    v.vw = ctx->bed_vw[s];
    v.ww = ctx->bed_ww[s];
    v.cg = ctx->use_cg ? ctx->bed_cg[s] : nullptr;
    return v;
}

// the column cache serves bed-only geometry in air mode: no cube, no phi
// geometry, periodic x, no free surface (the kernels that use it carry no
// free-surface code)
static bool wants_column_cache(const lbm_params &P) {
    return P.include_bed && !P.include_cube && !P.use_phi_open_fraction && !P.use_phi_open_flags && !P.x_solid &&
           !P.physics_water && P.fs_mode == LBM_FS_NONE;
}
static int refresh_column_cache(lbm_ctx *ctx, int s, cudaStream_t st) {
    if (!ctx->use_cg) return LBM_OK;
    launch_colgeo(ctx->P, ctx->D, slot_view(ctx, s), ctx->bed_cg[s], st);
    CK_LAUNCH("column cache");
    return LBM_OK;
}

static float step_time(const lbm_ctx *ctx, int64_t step) {
    return (float)((double)(step + 1) * ctx->P.dt_phys);  // CODEX.py:3874
}

static InitArgs init_args(lbm_ctx *ctx, int slot) {
    InitArgs I;
    memset(&I, 0, sizeof I);
    const lbm_buffers &b = ctx->b;
    I.P = ctx->P;
    I.slot = ctx->slot;
    I.D = ctx->D;
    I.bed = slot_view(ctx, slot);
    I.bed.cg = nullptr;   // setup kernels take the per-link path
    I.f_cur = b.f[ctx->cur];
    I.f_other = b.f[1 - ctx->cur];
    I.rho = b.rho; I.ux = b.ux; I.uy = b.uy; I.uz = b.uz; I.omega = b.omega;
    I.water_h = b.water_h; I.water_h_last = b.water_h_last;
    I.u_wave = b.u_wave; I.v_wave = b.v_wave; I.w_wave = b.w_wave;
    I.fs_h = b.fs_h; I.fs_h_last = b.fs_h_last; I.fs_flux_x = b.fs_flux_x; I.fs_flux_y = b.fs_flux_y;
    I.piecewise = b.piecewise_bed_z;
    I.u_inlet_profile = b.u_inlet_profile;
    I.rho_initial = b.rho_initial;
    I.noise = b.init_noise;
    I.fs_fill = b.fs_fill; I.fs_mass = b.fs_mass; I.fs_mass_excess = b.fs_mass_excess;
    I.fs_type = b.fs_type; I.fs_type_prev = b.fs_type_prev; I.fs_excess_dir = b.fs_excess_dir;
    return I;
}

static bool is_vof(const lbm_params &P) { return P.fs_mode != LBM_FS_NONE && P.fs_tracking == LBM_TRACK_VOF; }

static VofArgs vof_args(lbm_ctx *ctx, int slot, void *f) {
    VofArgs V;
    memset(&V, 0, sizeof V);
    const lbm_buffers &b = ctx->b;
    V.P = ctx->P;
    V.slot = ctx->slot;
    V.D = ctx->D;
    V.f = f;
    V.type = b.fs_type; V.type_prev = b.fs_type_prev; V.excess_dir = b.fs_excess_dir;
    V.fill = b.fs_fill; V.mass = b.fs_mass; V.mass_excess = b.fs_mass_excess;
    V.rho = b.rho; V.ux = b.ux; V.uy = b.uy; V.uz = b.uz;
    V.bed_h = ctx->bed_h[slot];
    V.fs_h = b.fs_h; V.fs_h_last = b.fs_h_last;
    V.open = ctx->v_open; V.lf0 = ctx->v_lf0;
    V.m0 = ctx->v_m0; V.x0 = ctx->v_x0; V.t0 = ctx->v_t0;
    V.fa = ctx->v_fa; V.ba = ctx->v_ba; V.dd = ctx->v_dd;
    V.dist = ctx->v_dist;
    V.near = ctx->v_near;
    V.cbx = (ctx->D.nx + VOF_CB - 1) / VOF_CB;
    V.cby = (ctx->D.ny + VOF_CB - 1) / VOF_CB;
    V.cbz = (ctx->D.nz + VOF_CB - 1) / VOF_CB;
    V.near_ok = ctx->v_near && ctx->D.ny % VOF_CB == 0 && (ctx->P.x_solid || ctx->D.nx % VOF_CB == 0);
    V.count = ctx->dcount;
    V.fcount = ctx->dfcount;
    return V;
}

static StepArgs step_args(lbm_ctx *ctx) {
    StepArgs A;
    memset(&A, 0, sizeof A);
    const lbm_buffers &b = ctx->b;
    A.P = ctx->P;
    A.slot = ctx->slot;
    A.D = ctx->D;
    A.rho = b.rho; A.ux = b.ux; A.uy = b.uy; A.uz = b.uz; A.omega = b.omega;
    A.u_les = ctx->u_les;
    A.u_out = ctx->u_les;
    A.fs_h = b.fs_h; A.fs_h_last = b.fs_h_last;
    A.fs_fill = b.fs_fill; A.fs_type = b.fs_type;
    A.u_inlet_profile = b.u_inlet_profile;
    A.counters = ctx->dcount;
    A.status = ctx->dstatus;
    A.zlo[0] = 0;
    A.zcnt[0] = ctx->P.nz;
    A.zi0 = 0;
    A.zi1 = -1;
    A.chunk = 0;
    return A;
}

// copy the bound bed state into slot s (start of a call)
static int load_bed_slot(lbm_ctx *ctx, int s, cudaStream_t st) {
    size_t bytes = ctx->D.a * sizeof(float);
    CK(cudaMemcpyAsync(ctx->bed_h[s], ctx->b.water_h, bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->bed_uw[s], ctx->b.u_wave, bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->bed_vw[s], ctx->b.v_wave, bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->bed_ww[s], ctx->b.w_wave, bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    launch_hmax(ctx->D, ctx->bed_h[s], ctx->bed_hmax[s], st);
    CK_LAUNCH("hmax");
    return refresh_column_cache(ctx, s, st);
}
// copy slot s (and the previous height) back to the bound buffers
static int store_bed_slot(lbm_ctx *ctx, int s, const float *h_prev, cudaStream_t st) {
    size_t bytes = ctx->D.a * sizeof(float);
    CK(cudaMemcpyAsync(ctx->b.water_h_last, h_prev, bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->b.water_h, ctx->bed_h[s], bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->b.u_wave, ctx->bed_uw[s], bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->b.v_wave, ctx->bed_vw[s], bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    CK(cudaMemcpyAsync(ctx->b.w_wave, ctx->bed_ww[s], bytes, cudaMemcpyDeviceToDevice, st), "bed copy");
    return LBM_OK;
}

static int bed_step(lbm_ctx *ctx, int64_t m, cudaStream_t st) {
    int s = (int)(m & 1), sp = (int)((m - 1) & 1);
    launch_bed(ctx->P, ctx->D, ctx->bed_h[sp], ctx->bed_h[s], ctx->bed_hmax[s], ctx->bed_uw[s], ctx->bed_vw[s],
               ctx->bed_ww[s], ctx->b.piecewise_bed_z, step_time(ctx, m), st, ctx->capturing ? ctx->dclock : nullptr,
               (long long)(m - ctx->cap_n0));
    CK_LAUNCH("bed");
    return refresh_column_cache(ctx, s, st);
}

// Split of the planes between the interior tile kernel and the general
// kernels.  The tile path needs: air mode without free surface, periodic x
// without the x fringe, no cube, no phi geometry, nx and ny multiples of
// the tile.  Interior planes start one plane above the first plane that is
// provably above the bed at all times (so no link there is cut and the
// cell below is fluid) and end below the top row.
struct Plan {
    bool tile = false;
    bool classic = false;   // unpipelined interior kernel even for FP32 (LBM_B200_TILE_KERNEL=classic)
    bool no_tma = false;    // cp.async-staged interior kernel instead of tile copies (LBM_B200_TILE_KERNEL=pipe)
    int zi0 = 0, zi1 = -1, chunk = 64;
    int zlo[3] = {0, 0, 0}, zcnt[3] = {0, 0, 0};
};

static Plan plan_planes(const lbm_ctx *ctx) {
    const lbm_params &P = ctx->P;
    Plan R;
    R.zlo[0] = 0;
    R.zcnt[0] = P.nz;
    const char *off = getenv("LBM_B200_NO_TILE");
    if (off && off[0] == '1') return R;
    if (P.fs_mode != LBM_FS_NONE || P.x_solid || P.enable_x_fringe || P.include_cube || P.use_phi_open_fraction ||
        P.use_phi_open_flags || P.nx % LBM_TILE || P.ny % LBM_TILE)
        return R;
    int kf = 0;
    if (P.include_bed) {
        double hb = ctx->bed_bound;
        double dx = (double)P.dx;
        kf = (int)ceil(hb / dx + 0.5 + 1e-3 + 1e-5 * ((double)P.nz + fabs(hb) / dx));
        if (kf < 0) kf = 0;
    }
    int zi0 = kf + 1, zi1 = P.nz - 2;
    if (zi0 < 1) zi0 = 1;
    if (zi1 < zi0) return R;
    R.tile = true;
    const char *tk = getenv("LBM_B200_TILE_KERNEL");
    R.classic = tk && strcmp(tk, "classic") == 0;
    R.no_tma = tk && strcmp(tk, "pipe") == 0;
    R.zi0 = zi0;
    R.zi1 = zi1;
    // planes per block: enough blocks for ~4 waves of 2 blocks per SM, at
    // least 8 planes (each chunk recomputes 2 neighbour planes), at most 64
    const int ni = zi1 - zi0 + 1;
    const int tiles = (P.nx / LBM_TILE) * (P.ny / LBM_TILE);
    const int want_chunks = (4 * 2 * 148 + tiles - 1) / tiles;
    int chunk = (ni + want_chunks - 1) / want_chunks;
    if (chunk < 8) chunk = 8;
    if (chunk > 64) chunk = 64;
    if (ctx->tile_chunk > 0) chunk = ctx->tile_chunk;   // set by lbm_set_tile_chunk (autotuner)
    const char *ch = getenv("LBM_B200_TILE_CHUNK");
    if (ch && atoi(ch) > 0) chunk = atoi(ch);
    R.chunk = chunk;
    R.zlo[0] = 0;
    R.zcnt[0] = zi0;
    R.zlo[1] = zi1 + 1;
    R.zcnt[1] = P.nz - (zi1 + 1);
    return R;
}

static void apply_plan(StepArgs &A, const Plan &R) {
    for (int r = 0; r < 3; ++r) {
        A.zlo[r] = R.zlo[r];
        A.zcnt[r] = R.zcnt[r];
    }
    A.zi0 = R.zi0;
    A.zi1 = R.zi1;
    A.chunk = R.chunk;
}

// cuTensorMapEncodeTiled, found through the runtime's driver entry points
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::mutex mu;
    static bool tried = false;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor maps over the populations f[q][z][y][x] as a 4-D tensor
// (x, y, z, q) for the tile-copy interior kernel.  FP32: boxes 24 and 20
// values wide; 16-bit storage: one box 32 values wide (both map slots).
// Requirements of tile copies: 16-byte aligned base, strides multiples of
// 16 bytes (nx a multiple of 8), inner box extent a multiple of 16 bytes.
static bool tile_maps_ready(lbm_ctx *ctx) {
    if (ctx->tmap_ok && ctx->tmap_src[0] == ctx->b.f[0] && ctx->tmap_src[1] == ctx->b.f[1]) return true;
    ctx->tmap_ok = false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const bool f32 = ctx->P.pop_storage == LBM_STORE_F32;
    const cuuint64_t es_b = f32 ? 4 : 2;
    const cuuint64_t nx = (cuuint64_t)ctx->P.nx, ny = (cuuint64_t)ctx->P.ny, nz = (cuuint64_t)ctx->P.nz;
    if (nx % 8 != 0) return false;
    const cuuint64_t dims[4] = {nx, ny, nz, 19};
    const cuuint64_t strides[3] = {nx * es_b, nx * ny * es_b, nx * ny * nz * es_b};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    for (int b = 0; b < 2; ++b) {
        if (((uintptr_t)ctx->b.f[b] & 15u) != 0) return false;
        for (int w = 0; w < 2; ++w) {
            const cuuint32_t width = f32 ? (w == 0 ? 24u : 20u) : 32u;
            const cuuint32_t box[4] = {width, (cuuint32_t)(LBM_TILE + 2), 1u, 1u};
            if (enc(&ctx->tmap[b][w], f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 4,
                    ctx->b.f[b], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return false;
        }
    }
    ctx->tmap_src[0] = ctx->b.f[0];
    ctx->tmap_src[1] = ctx->b.f[1];
    ctx->tmap_ok = true;
    return true;
}

static int step_air(lbm_ctx *ctx, int K, cudaStream_t st) {
    const int64_t n = ctx->nstep;
    const bool les = ctx->P.use_les != 0;
    const Plan R = plan_planes(ctx);
    StepArgs A = step_args(ctx);
    apply_plan(A, R);
    int s;
    if ((s = bed_step(ctx, n + 1, st)) != LBM_OK) return s;
    int src = ctx->cur;
    A.fsrc = ctx->b.f[src];
    A.fdst = ctx->b.f[1 - src];
    A.bed_c = slot_view(ctx, (int)((n + 1) & 1));
    A.bed_s = A.bed_c;
    if (ctx->capturing) A.clock = ctx->dclock;   // step numbers below become offsets from the clock
    const int64_t key0 = ctx->capturing ? ctx->cap_n0 : 0;
    A.step = (uint64_t)(n + 1 - key0);
    // with LES the pre-pass stores the post-condition populations of the
    // general planes for their collide pass (column-cache path): in the
    // destination slots with FP32 populations, else in an FP32 stash
    // (allocated by the first eager call; a capture without it keeps the
    // general collide's own stream pass)
    const char *ns = getenv("LBM_B200_NO_STASH");   // the general collide repeats the stream (comparison runs)
    bool stash = les && ctx->use_cg && !(ns && ns[0] == '1');
    if (stash && ctx->P.pop_storage != LBM_STORE_F32) {
        const size_t ng = (size_t)(R.zcnt[0] + R.zcnt[1] + R.zcnt[2]) * P_nx(ctx) * P_ny(ctx);
        if (ctx->stash_cells < ng && !ctx->capturing) {
            float *p = nullptr;
            if ((s = alloc(ctx, (void **)&p, 19 * ng * sizeof(float), st)) != LBM_OK) return s;
            ctx->stash = p;
            ctx->stash_cells = ng;
        }
        stash = ctx->stash_cells >= ng;
        A.stash = ctx->stash;
    }
    // LBM_B200_TEST_TMA_TIMEOUT=1: the tile-copy kernel takes its wait-timeout
    // exit (status bit 2) at its first plane; used only by the error-path test
    const char *tt = getenv("LBM_B200_TEST_TMA_TIMEOUT");
    const int tflag = (R.classic ? F_TILE_CLASSIC : 0) | (stash ? F_STASH : 0) |
                      ((tt && tt[0] == '1') ? F_TEST_WAIT_TIMEOUT : 0);
    A.flags = ((K == 1) ? (F_WRITE_MACRO | F_WRITE_ALL_OMEGA) : 0) | tflag;
    // fused interior steps with LES: the tile-copy kernel (32-bit population indices)
    const bool tma = R.tile && les && !R.classic && !R.no_tma && 19.0 * (double)ctx->D.n < 2147483647.0 &&
                     tile_maps_ready(ctx);
    if (les) {
        launch_step_kernel(KER_PREPASS_CANON, A, st);
        CK_LAUNCH("prepass");
    }
    if (R.tile) {
        launch_step_kernel(KER_TILE_CANON, A, st);
        CK_LAUNCH("tile");
    }
    launch_step_kernel(KER_COLLIDE_CANON, A, st);
    CK_LAUNCH("collide");
    src = 1 - src;
    for (int64_t m = n + 1; m < n + K; ++m) {
        if ((s = bed_step(ctx, m + 1, st)) != LBM_OK) return s;
        A.fsrc = ctx->b.f[src];
        A.fdst = ctx->b.f[1 - src];
        A.bed_s = slot_view(ctx, (int)(m & 1));
        A.bed_c = slot_view(ctx, (int)((m + 1) & 1));
        A.step = (uint64_t)(m + 1 - key0);
        A.flags = ((m + 1 == n + K) ? (F_WRITE_MACRO | F_WRITE_ALL_OMEGA) : 0) | tflag;
        if (les) {
            launch_step_kernel(KER_PREPASS_FUSED, A, st);
            CK_LAUNCH("prepass fused");
        }
        if (R.tile) {
            if (ctx->timing) timed_mark(ctx, st);
            const CUtensorMap *m24 = &ctx->tmap[src][0], *m20 = &ctx->tmap[src][1];
            const bool done = tma && (ctx->arith == LBM_ARITH_FAST ? launch_tile_tma_fast(A, m24, m20, st)
                                                                   : launch_tile_tma(A, m24, m20, st));
            if (!done) launch_step_kernel(KER_TILE_FUSED, A, st);
            CK_LAUNCH("tile fused");
            if (ctx->timing) {
                timed_mark(ctx, st);
                ctx->timed_cells = (int64_t)(R.zi1 - R.zi0 + 1) * P_nx(ctx) * P_ny(ctx);
            }
        }
        launch_step_kernel(KER_COLLIDE_FUSED, A, st);
        CK_LAUNCH("fused");
        src = 1 - src;
    }
    CK(cudaMemsetAsync(ctx->dcount, 0, 3 * sizeof(int), st), "counter reset");
    A.fsrc = ctx->b.f[src];
    A.fdst = ctx->b.f[1 - src];
    A.bed_s = slot_view(ctx, (int)((n + K) & 1));
    A.bed_c = A.bed_s;
    A.flags = F_COUNT;
    launch_step_kernel(KER_STREAM, A, st);
    CK_LAUNCH("stream");
    if (R.tile) {
        launch_step_kernel(KER_STREAM_INTERIOR, A, st);
        CK_LAUNCH("stream interior");
    }
    ctx->cur = 1 - src;
    ctx->nstep = n + K;
    return LBM_OK;
}

// the list of the water stream's general cells (one int per cell and a count)
static int water_list(lbm_ctx *ctx, cudaStream_t st) {
    if (ctx->wlist) return LBM_OK;
    return alloc(ctx, (void **)&ctx->wlist, ((size_t)ctx->D.n + 1) * sizeof(int), st);
}

static int step_height(lbm_ctx *ctx, int K, cudaStream_t st) {
    const bool les = ctx->P.use_les != 0;
    int s;
    if ((s = water_list(ctx, st)) != LBM_OK) return s;
    for (int it = 0; it < K; ++it) {
        int64_t m = ctx->nstep + 1;
        if ((s = bed_step(ctx, m, st)) != LBM_OK) return s;
        StepArgs A = step_args(ctx);
        A.zlo[0] = 0;
        A.zcnt[0] = ctx->P.nz;
        A.bed_s = slot_view(ctx, (int)(m & 1));
        A.bed_c = A.bed_s;
        // under capture the step number is an offset from the device clock
        if (ctx->capturing) A.clock = ctx->dclock;
        A.step = (uint64_t)(m - (ctx->capturing ? ctx->cap_n0 : 0));
        A.fsrc = ctx->b.f[ctx->cur];
        A.fdst = ctx->b.f[1 - ctx->cur];
        A.flags = F_WRITE_MACRO | F_WRITE_ALL_OMEGA;
        if (les) {
            launch_step_kernel(KER_PREPASS_CANON, A, st);
            CK_LAUNCH("prepass");
        }
        // the compact kernels take the cells with local collide / plain-gather
        // stream, the general ones the rest, from a list
        launch_water_collide(A, ctx->wlist, ctx->wlist + ctx->D.n, st);
        CK_LAUNCH("collide");
        CK(cudaMemsetAsync(ctx->dcount, 0, 4 * sizeof(int), st), "counter reset");
        A.fsrc = ctx->b.f[1 - ctx->cur];
        A.fdst = ctx->b.f[ctx->cur];
        A.flags = F_COUNT;
        launch_water_stream(A, ctx->wlist, ctx->wlist + ctx->D.n, st);
        CK_LAUNCH("stream");
        launch_column_flux(A, ctx->b.fs_flux_x, ctx->b.fs_flux_y, st);
        CK_LAUNCH("column flux");
        launch_advect(ctx->P, ctx->D, ctx->bed_h[m & 1], ctx->b.fs_flux_x, ctx->b.fs_flux_y, ctx->b.fs_h, ctx->b.fs_h,
                      ctx->b.fs_h_last, step_time(ctx, m), st);
        CK_LAUNCH("advect");
        A.flags = 0;
        A.fdst = ctx->b.f[ctx->cur];
        launch_refill(A, nullptr, ctx->dcount + CNT_FS_REFILL, st);
        CK_LAUNCH("refill");
        ctx->nstep = m;
    }
    StepArgs A = step_args(ctx);
    A.bed_s = slot_view(ctx, (int)(ctx->nstep & 1));
    launch_height_types(A, ctx->b.fs_fill, ctx->b.fs_type, ctx->b.fs_type_prev, st);
    CK_LAUNCH("height types");
    return LBM_OK;
}

// VOF path: one step per iteration, the reference's order (CODEX.py:3873-3920)
static int step_vof(lbm_ctx *ctx, int K, cudaStream_t st) {
    const bool les = ctx->P.use_les != 0;
    int s;
    if ((s = water_list(ctx, st)) != LBM_OK) return s;
    for (int it = 0; it < K; ++it) {
        int64_t m = ctx->nstep + 1;
        if ((s = bed_step(ctx, m, st)) != LBM_OK) return s;
        const int slot = (int)(m & 1);
        StepArgs A = step_args(ctx);
        A.zlo[0] = 0;
        A.zcnt[0] = ctx->P.nz;
        A.bed_s = slot_view(ctx, slot);
        A.bed_c = A.bed_s;
        A.step = (uint64_t)m;
        A.fsrc = ctx->b.f[ctx->cur];
        A.fdst = ctx->b.f[1 - ctx->cur];
        A.flags = F_WRITE_MACRO | F_WRITE_ALL_OMEGA | F_VOF_STATE;
        VofArgs V = vof_args(ctx, slot, ctx->b.f[ctx->cur]);
        launch_vof_open(V, A.bed_s, st);
        CK_LAUNCH("vof open mask");
        if (les) {
            launch_step_kernel(KER_PREPASS_CANON, A, st);
            CK_LAUNCH("prepass");
        }
        // compact kernels for the cells with local collide / plain-gather stream, the general ones over a list
        launch_water_collide(A, ctx->wlist, ctx->wlist + ctx->D.n, st);
        CK_LAUNCH("collide");
        CK(cudaMemsetAsync(ctx->dcount, 0, 4 * sizeof(int), st), "counter reset");
        A.fsrc = ctx->b.f[1 - ctx->cur];
        A.fdst = ctx->b.f[ctx->cur];
        A.flags = F_COUNT | F_VOF_STATE;
        launch_water_stream(A, ctx->wlist, ctx->wlist + ctx->D.n, st);
        CK_LAUNCH("stream");
        const bool due = ctx->P.vof_collapse_enabled && (m % ctx->P.vof_collapse_interval) == 0;
        CK(vof_sequence(V, due, ctx->v_tree, st), "vof sequence");
        A.flags = F_VOF_STATE;
        A.fdst = ctx->b.f[ctx->cur];
        launch_refill_vof(A, V, ctx->b.fs_type_prev, ctx->wlist, ctx->dcount + CNT_FS_REFILL, st);
        CK_LAUNCH("refill");
        CK(cudaMemsetAsync(ctx->dcount + CNT_COALESCE, 0, sizeof(int), st), "counter reset");
        launch_vof_coalesce(V, st);
        CK_LAUNCH("coalescence repair");
        ctx->nstep = m;
    }
    return LBM_OK;
}

extern "C" {

const char *lbm_backend_name(void) { return "cuda-sm100a"; }
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

int lbm_create(const lbm_params *params, lbm_ctx **out) {
    if (!params || !out) return LBM_ERR_BAD_ARG;
    if (params->abi_version != LBM_ABI_VERSION || params->magic_end != LBM_PARAMS_MAGIC) return LBM_ERR_BAD_ARG;
    if (params->nx < 1 || params->ny < 1 || params->nz < 2) return LBM_ERR_BAD_ARG;
    if (params->pop_storage < 0 || params->pop_storage > 2) return LBM_ERR_BAD_ARG;
    if (params->x_solid && params->nx < 2) return LBM_ERR_BAD_ARG;
    lbm_ctx *ctx = new lbm_ctx();
    ctx->P = *params;
    ctx->D.nx = params->nx;
    ctx->D.ny = params->ny;
    ctx->D.nz = params->nz;
    ctx->D.a = (size_t)params->nx * params->ny;
    ctx->D.n = ctx->D.a * params->nz;
    if (ctx->D.n > 0x7fffffffULL) {
        delete ctx;
        return LBM_ERR_BAD_ARG;
    }
    {
        // LBM_B200_ARITH=fast|exact: the default arithmetic of new contexts
        const char *ar = getenv("LBM_B200_ARITH");
        ctx->arith = (ar && strcmp(ar, "fast") == 0) ? LBM_ARITH_FAST : LBM_ARITH_EXACT;
    }
    ctx->slot = acquire_slot();
    if (ctx->slot < 0) {
        delete ctx;
        return LBM_ERR_UNSUPPORTED;
    }
    cudaError_t e = upload_params(ctx->slot, ctx->P);
    if (e != cudaSuccess) {
        release_slot(ctx->slot);
        delete ctx;
        return LBM_ERR_CUDA;
    }
    *out = ctx;
    return LBM_OK;
}


int lbm_bind(lbm_ctx *ctx, const lbm_buffers *bufs) {
    if (!ctx || !bufs) return LBM_ERR_BAD_ARG;
    const lbm_buffers &b = *bufs;
    if (!b.f[0] || !b.f[1] || !b.rho || !b.ux || !b.uy || !b.uz || !b.omega || !b.water_h || !b.water_h_last ||
        !b.u_wave || !b.v_wave || !b.w_wave || !b.fs_h || !b.fs_h_last || !b.fs_flux_x || !b.fs_flux_y ||
        !b.piecewise_bed_z || !b.u_inlet_profile || !b.rho_initial || !b.init_noise || !b.fs_fill ||
        !b.fs_type || !b.fs_type_prev || !b.fs_mass || !b.fs_mass_excess || !b.fs_excess_dir)
        return fail(ctx, LBM_ERR_BAD_ARG, "lbm_bind: a required state buffer is NULL");
    drop_graphs(ctx);   // captured graphs hold the previous buffers' addresses
    ctx->b = b;
    if (!ctx->bound) {
        int s;
        size_t A = ctx->D.a * sizeof(float);
        for (int i = 0; i < 2; ++i) {
            if ((s = alloc(ctx, (void **)&ctx->bed_h[i], A)) || (s = alloc(ctx, (void **)&ctx->bed_hmax[i], A)) ||
                (s = alloc(ctx, (void **)&ctx->bed_uw[i], A)) || (s = alloc(ctx, (void **)&ctx->bed_vw[i], A)) ||
                (s = alloc(ctx, (void **)&ctx->bed_ww[i], A)))
                return s;
        }
        if (ctx->P.use_les && (s = alloc(ctx, (void **)&ctx->u_les, 3 * ctx->D.n * sizeof(float)))) return s;
        if (is_vof(ctx->P)) {
            const size_t n = ctx->D.n;
            const size_t nt = 6 * (n / 256 + 2);
            if ((s = alloc(ctx, (void **)&ctx->v_open, n)) || (s = alloc(ctx, (void **)&ctx->v_t0, n)) ||
                (s = alloc(ctx, (void **)&ctx->v_ba, 2 * n)) || (s = alloc(ctx, (void **)&ctx->v_lf0, 4 * n)) ||
                (s = alloc(ctx, (void **)&ctx->v_m0, 4 * n)) || (s = alloc(ctx, (void **)&ctx->v_x0, 4 * n)) ||
                (s = alloc(ctx, (void **)&ctx->v_fa, 24 * n)) || (s = alloc(ctx, (void **)&ctx->v_dd, 8 * n)) ||
                (s = alloc(ctx, (void **)&ctx->v_tree, 8 * nt)) || (s = alloc(ctx, (void **)&ctx->v_dist, 4 * n)) ||
                (s = alloc(ctx, (void **)&ctx->v_near, 2 * vof_near_bytes(ctx->D))))
                return s;
            CK(cudaMemset(ctx->v_dist, 0xff, 4 * n), "memset");
        }
        if (wants_column_cache(ctx->P)) {
            for (int i = 0; i < 2; ++i)
                if ((s = alloc(ctx, (void **)&ctx->bed_cg[i], (size_t)CG_N * A))) return s;
            ctx->use_cg = true;
        }
        if ((s = alloc(ctx, (void **)&ctx->dcount, CNT_N * sizeof(int))) ||
            (s = alloc(ctx, (void **)&ctx->dstatus, sizeof(unsigned))) ||
            (s = alloc(ctx, (void **)&ctx->dfcount, 8 * sizeof(float))))
            return s;
        CK(cudaMemset(ctx->dcount, 0, CNT_N * sizeof(int)), "memset");
        CK(cudaMemset(ctx->dstatus, 0, sizeof(unsigned)), "memset");
        CK(cudaMemset(ctx->dfcount, 0, 8 * sizeof(float)), "memset");
    }
    ctx->bound = true;
    return LBM_OK;
}

int lbm_init_geometry(lbm_ctx *ctx, void *stream) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->last_stream = st;
    ctx->cur = 0;
    ctx->nstep = 0;
    {
        // upper bound of the bed height for the interior-plane split
        const lbm_params &P = ctx->P;
        double hb = (double)P.bed_offset_m;
        if (P.bed_profile == LBM_BED_MOVING_SINE) hb += fabs((double)P.bed_amp1) + fabs((double)P.bed_amp2);
        if (P.bed_profile == LBM_BED_PIECEWISE) {
            std::vector<float> pw(P.nx);
            CK(cudaMemcpy(pw.data(), ctx->b.piecewise_bed_z, P.nx * sizeof(float), cudaMemcpyDeviceToHost),
               "piecewise copy");
            hb = -1e30;
            for (float v : pw) hb = v > hb ? v : hb;
        }
        ctx->bed_bound = hb;
    }
    InitArgs I = init_args(ctx, 0);
    launch_init_constants(I, st);
    CK_LAUNCH("init constants");
    size_t pop_bytes = ctx->D.n * 19 * (ctx->P.pop_storage == LBM_STORE_F32 ? 4 : 2);
    CK(cudaMemsetAsync(ctx->b.f[0], 0, pop_bytes, st), "memset f");
    CK(cudaMemsetAsync(ctx->b.f[1], 0, pop_bytes, st), "memset f");
    CK(cudaMemsetAsync(ctx->dcount, 0, CNT_N * sizeof(int), st), "memset counters");
    CK(cudaMemsetAsync(ctx->dstatus, 0, sizeof(unsigned), st), "memset status");
    CK(cudaMemsetAsync(ctx->dfcount, 0, 8 * sizeof(float), st), "memset counters");
    if (ctx->v_dist) CK(cudaMemsetAsync(ctx->v_dist, 0xff, ctx->D.n * sizeof(int), st), "memset exterior");
    // update_wave_bed_and_velocities(0.0): previous height = initial level
    launch_bed(ctx->P, ctx->D, ctx->b.water_h, ctx->bed_h[0], ctx->bed_hmax[0], ctx->bed_uw[0], ctx->bed_vw[0],
               ctx->bed_ww[0], ctx->b.piecewise_bed_z, 0.0f, st);
    CK_LAUNCH("bed");
    int s;
    if ((s = store_bed_slot(ctx, 0, ctx->b.water_h, st)) != LBM_OK) return s;
    I = init_args(ctx, 0);
    launch_fs_height_init(I, st);
    CK_LAUNCH("free-surface height");
    launch_classify_store(I, st);
    CK_LAUNCH("classify");
    if (ctx->P.fs_mode != LBM_FS_NONE && ctx->P.fs_tracking == LBM_TRACK_VOF && ctx->P.vof_initial_block) {
        launch_vof_block(I, st);
        CK_LAUNCH("vof block");
    }
    return LBM_OK;
}

int lbm_init_fields(lbm_ctx *ctx, void *stream) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->last_stream = st;
    int s;
    if ((s = load_bed_slot(ctx, (int)(ctx->nstep & 1), st)) != LBM_OK) return s;
    InitArgs I = init_args(ctx, (int)(ctx->nstep & 1));
    launch_init_fields(I, st);
    CK_LAUNCH("init fields");
    ctx->cur = 1 - ctx->cur;  // copy_post_and_swap, CODEX.py:3789
    if (is_vof(ctx->P)) {
        // CODEX.py:3790-3792
        const int slot = (int)(ctx->nstep & 1);
        VofArgs V = vof_args(ctx, slot, ctx->b.f[ctx->cur]);
        launch_vof_open(V, slot_view(ctx, slot), st);
        CK_LAUNCH("vof open mask");
        launch_vof_mass_init(I, st);
        CK_LAUNCH("vof mass");
        CK(vof_interface_layer(V, st), "vof interface layer");
        launch_vof_height(V, st);
        CK_LAUNCH("vof height");
    }
    return LBM_OK;
}

}  // extern "C"

// Modes whose step calls can be captured as graphs: air, and the height
// path with the kinematic height update (its advection does not read the
// step time; the prescribed solitary height does).  The VOF path decides on
// the host per step (trapped-gas collapse steps, the flood fill's stop).
static bool graph_mode(const lbm_params &P) {
    return P.fs_mode == LBM_FS_NONE || (P.fs_mode == LBM_FS_HEIGHT_KINEMATIC && P.fs_tracking != LBM_TRACK_VOF);
}

static int step_call(lbm_ctx *ctx, int32_t nsteps, cudaStream_t st) {
    int s;
    int64_t n0 = ctx->nstep;
    if ((s = load_bed_slot(ctx, (int)(n0 & 1), st)) != LBM_OK) return s;
    if (ctx->P.fs_mode == LBM_FS_NONE) s = step_air(ctx, nsteps, st);
    else if (is_vof(ctx->P)) s = step_vof(ctx, nsteps, st);
    else s = step_height(ctx, nsteps, st);
    if (s != LBM_OK) return s;
    int64_t n1 = ctx->nstep;
    return store_bed_slot(ctx, (int)(n1 & 1), ctx->bed_h[(n1 - 1) & 1], st);
}

// A call of nsteps as one graph launch.  The first call of a shape is
// captured (nothing runs during capture), then replayed like every later
// one.  LBM_ERR_UNSUPPORTED: capture refused; the caller runs the call eagerly.
static int step_graph(lbm_ctx *ctx, int32_t nsteps, cudaStream_t st) {
    const int par = (int)(ctx->nstep & 1), cur = ctx->cur;
    lbm_ctx::StepGraph *g = nullptr;
    for (auto &e : ctx->graph_cache)
        if (e.steps == nsteps && e.parity == par && e.cur == cur) g = &e;
    if (!g) {
        if (!ctx->dclock) {
            int s = alloc(ctx, (void **)&ctx->dclock, sizeof(long long), st);
            if (s != LBM_OK) return s;
        }
        const int64_t n0 = ctx->nstep;
        const long long l0 = launch_count();
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return LBM_ERR_UNSUPPORTED;
        }
        ctx->capturing = true;
        ctx->cap_n0 = n0;
        const int s = step_call(ctx, nsteps, st);
        ctx->capturing = false;
        ctx->cap_n0 = 0;
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &graph);
        const int cur_after = ctx->cur;
        const long long launches = launch_count() - l0;
        launch_count_add(-launches);   // nothing ran during the capture
        ctx->nstep = n0;
        ctx->cur = cur;
        cudaGraphExec_t exec = nullptr;
        const bool ok = s == LBM_OK && e == cudaSuccess && graph &&
                        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (graph) cudaGraphDestroy(graph);
        if (!ok) {
            cudaGetLastError();
            ctx->err.clear();
            return LBM_ERR_UNSUPPORTED;
        }
        ctx->graph_cache.push_back({nsteps, par, cur, cur_after, launches, exec});
        g = &ctx->graph_cache.back();
    }
    launch_clock_set(ctx->dclock, (long long)ctx->nstep, st);
    CK_LAUNCH("step clock");
    CK(cudaGraphLaunch(g->exec, st), "step graph launch");
    launch_count_add(g->launches);
    ctx->nstep += nsteps;
    ctx->cur = g->cur_after;
    return LBM_OK;
}

extern "C" {

int lbm_step(lbm_ctx *ctx, int32_t nsteps, void *stream) {
    if (!ctx || nsteps < 0) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    if (nsteps == 0) return LBM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->last_stream = st;
    // step graphs: air mode, a stream of the caller's, no per-launch timing,
    // after one eager call (which sets the kernels' shared-memory limits)
    if (ctx->graphs && st != 0 && graph_mode(ctx->P) && !ctx->timing && ctx->warm) {
        const int s = step_graph(ctx, nsteps, st);
        if (s != LBM_ERR_UNSUPPORTED) return s;
        ctx->graphs = false;   // capture refused: eager from now on
    }
    const int s = step_call(ctx, nsteps, st);
    if (s == LBM_OK) ctx->warm = true;
    return s;
}

int lbm_export_diagnostics(lbm_ctx *ctx, void *stream) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->last_stream = st;
    int s;
    if ((s = load_bed_slot(ctx, (int)(ctx->nstep & 1), st)) != LBM_OK) return s;
    InitArgs I = init_args(ctx, (int)(ctx->nstep & 1));
    ExportArgs E;
    E.phi = ctx->b.phi;
    E.obstacle = ctx->b.obstacle;
    E.near_obstacle = ctx->b.near_obstacle;
    E.lattice_open = ctx->b.lattice_open;
    E.lattice_open_frac = ctx->b.lattice_open_frac;
    E.lattice_wall_type = ctx->b.lattice_wall_type;
    E.prh = ctx->b.pressure_reference_head;
    E.gbf = ctx->b.gravity_body_fraction;
    E.types_are_prev = ctx->nstep > 0 ? 1 : 0;
    launch_export(I, E, st);
    CK_LAUNCH("export");
    if (ctx->b.vof_exterior_gas) {
        if (ctx->v_dist) {
            launch_vof_exterior(ctx->D, ctx->v_dist, ctx->b.vof_exterior_gas, st);
            CK_LAUNCH("exterior labels");
        } else {
            CK(cudaMemsetAsync(ctx->b.vof_exterior_gas, 0, ctx->D.n * sizeof(int32_t), st), "memset exterior");
        }
    }
    return LBM_OK;
}

int lbm_read_counters(lbm_ctx *ctx, lbm_counters *out) {
    if (!ctx || !out) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    int h[CNT_N];
    unsigned status = 0;
    float fc[8];
    CK(cudaStreamSynchronize(ctx->last_stream), "synchronize");
    CK(cudaMemcpy(h, ctx->dcount, sizeof h, cudaMemcpyDeviceToHost), "counter copy");
    CK(cudaMemcpy(&status, ctx->dstatus, sizeof status, cudaMemcpyDeviceToHost), "status copy");
    CK(cudaMemcpy(fc, ctx->dfcount, sizeof fc, cudaMemcpyDeviceToHost), "counter copy");
    memset(out, 0, sizeof *out);
    out->boundary_cut_link_count = h[CNT_CUT];
    out->free_surface_cut_link_count = h[CNT_FSCUT];
    out->free_surface_thin_gap_bridge_count = h[CNT_BRIDGE];
    out->free_surface_refill_count = h[CNT_FS_REFILL];
    out->free_surface_coalescence_repair_count = h[CNT_COALESCE];
    out->free_surface_vof_excess_count = h[CNT_VOF_EXCESS];
    out->free_surface_vof_orphan_count = h[CNT_ORPHAN];
    out->free_surface_vof_collapse_cell_count = h[CNT_COLLAPSE];
    out->free_surface_vof_detached_advect_count = h[CNT_DET];
    out->free_surface_vof_detached_compress_count = h[CNT_CMP];
    out->flood_sweeps_used = h[CNT_SWEEPS];
    out->free_surface_vof_collapse_candidate_volume_m3 = fc[0];
    out->free_surface_vof_collapse_applied_volume_m3 = fc[1];
    out->free_surface_vof_collapse_removal_scale = fc[2];
    out->free_surface_vof_collapse_candidate_mass = fc[3];
    out->free_surface_vof_collapse_exterior_capacity = fc[4];
    out->free_surface_vof_detached_advect_mass = fc[5];
    out->free_surface_vof_detached_compress_mass = fc[6];
    out->status_flags = (int32_t)status;
    out->step = ctx->nstep;
    out->current_f = ctx->cur;
    return LBM_OK;
}

int lbm_diagnostics(lbm_ctx *ctx, const lbm_diag_inputs *in, lbm_diag *out, void *stream) {
    if (!ctx || !in || !out) return LBM_ERR_BAD_ARG;
    if (!ctx->bound) return LBM_ERR_NOT_BOUND;
    if (in->slice_j < 0 || in->slice_j >= ctx->P.ny) return fail(ctx, LBM_ERR_BAD_ARG, "lbm_diagnostics: slice_j out of range");
    cudaStream_t st = (cudaStream_t)stream;
    ctx->last_stream = st;
    const int ncellp = 4 * 148, nslp = 148;
    const size_t nx = (size_t)ctx->P.nx, nzx = (size_t)ctx->P.nz * nx;
    int s;
    if (!ctx->d_out) {
        if ((s = alloc(ctx, (void **)&ctx->d_cellp, ncellp * sizeof(DiagCellPart), st)) ||
            (s = alloc(ctx, (void **)&ctx->d_slp, 2 * nslp * sizeof(DiagSlicePart) + 12 * sizeof(double), st)) ||
            (s = alloc(ctx, (void **)&ctx->d_col_eta, nx * sizeof(double), st)) ||
            (s = alloc(ctx, (void **)&ctx->d_col_mm, 2 * nx * sizeof(float), st)) ||
            (s = alloc(ctx, (void **)&ctx->d_slice, 3 * nzx * sizeof(double), st)) ||
            (s = alloc(ctx, (void **)&ctx->d_mask, nzx, st)) || (s = alloc(ctx, (void **)&ctx->d_out, sizeof(lbm_diag), st)))
            return s;
    }
    if ((s = load_bed_slot(ctx, (int)(ctx->nstep & 1), st)) != LBM_OK) return s;
    DiagArgs G;
    memset(&G, 0, sizeof G);
    const lbm_buffers &b = ctx->b;
    G.P = ctx->P;
    G.slot = ctx->slot;
    G.D = ctx->D;
    G.bed = slot_view(ctx, (int)(ctx->nstep & 1));
    G.bed.cg = nullptr;
    G.rho = b.rho; G.ux = b.ux; G.uy = b.uy; G.uz = b.uz;
    G.fill = b.fs_fill; G.mass = b.fs_mass; G.excess = b.fs_mass_excess; G.fs_h = b.fs_h;
    G.type = b.fs_type; G.type_prev = b.fs_type_prev;
    G.types_are_prev = ctx->nstep > 0 ? 1 : 0;
    G.fs = ctx->P.fs_mode != LBM_FS_NONE ? 1 : 0;
    G.vof = is_vof(ctx->P) ? 1 : 0;
    G.slice_j = in->slice_j;
    G.rho_phys = in->rho_phys;
    G.gravity_phys = in->gravity_phys;
    G.cellp = ctx->d_cellp;
    G.ncellp = ncellp;
    G.col_eta = ctx->d_col_eta;
    G.col_min = ctx->d_col_mm;
    G.col_max = ctx->d_col_mm + nx;
    G.sl_p = ctx->d_slice;
    G.sl_pt = ctx->d_slice + nzx;
    G.sl_v = ctx->d_slice + 2 * nzx;
    G.sl_mask = ctx->d_mask;
    G.slp = ctx->d_slp;
    G.nslp = nslp;
    G.slice_mean = (double *)(ctx->d_slp + 2 * nslp);
    G.out = ctx->d_out;
    launch_diagnostics(G, st);
    CK_LAUNCH("diagnostics");
    CK(cudaMemcpyAsync(out, ctx->d_out, sizeof(lbm_diag), cudaMemcpyDeviceToHost, st), "diagnostics copy");
    CK(cudaStreamSynchronize(st), "synchronize");
    return LBM_OK;
}

int lbm_set_kernel_timing(lbm_ctx *ctx, int32_t enable) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    ctx->timing = enable != 0;
    ctx->ev_used = 0;
    return LBM_OK;
}

int lbm_kernel_timing(lbm_ctx *ctx, double *total_ms, int64_t *launches, int64_t *cells_per_launch) {
    if (!ctx || !total_ms || !launches || !cells_per_launch) return LBM_ERR_BAD_ARG;
    double tot = 0.0;
    for (size_t e = 0; e + 1 < ctx->ev_used; e += 2) {
        float ms = 0.0f;
        CK(cudaEventSynchronize(ctx->ev[e + 1]), "event sync");
        CK(cudaEventElapsedTime(&ms, ctx->ev[e], ctx->ev[e + 1]), "event time");
        tot += ms;
    }
    *total_ms = tot;
    *launches = (int64_t)(ctx->ev_used / 2);
    *cells_per_launch = ctx->timed_cells;
    return LBM_OK;
}

int lbm_set_tile_chunk(lbm_ctx *ctx, int32_t planes) {
    if (!ctx || planes < 0 || planes > 4096) return LBM_ERR_BAD_ARG;
    if (planes != ctx->tile_chunk) drop_graphs(ctx);
    ctx->tile_chunk = planes;
    return LBM_OK;
}

int lbm_set_arithmetic(lbm_ctx *ctx, int32_t mode) {
    if (!ctx || (mode != LBM_ARITH_EXACT && mode != LBM_ARITH_FAST)) return LBM_ERR_BAD_ARG;
    if (mode != ctx->arith) drop_graphs(ctx);
    ctx->arith = mode;
    return LBM_OK;
}

int lbm_get_arithmetic(lbm_ctx *ctx, int32_t *mode) {
    if (!ctx || !mode) return LBM_ERR_BAD_ARG;
    *mode = ctx->arith;
    return LBM_OK;
}

int lbm_set_step_graphs(lbm_ctx *ctx, int32_t enable) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    if (enable && !graph_mode(ctx->P))
        return fail(ctx, LBM_ERR_UNSUPPORTED, "lbm_set_step_graphs: air mode or the kinematic height path only");
    if (!enable) drop_graphs(ctx);
    ctx->graphs = enable != 0;
    return LBM_OK;
}

int lbm_launch_count(int64_t *count) {
    if (!count) return LBM_ERR_BAD_ARG;
    *count = (int64_t)lbm::launch_count();
    return LBM_OK;
}

int lbm_destroy(lbm_ctx *ctx) {
    if (!ctx) return LBM_ERR_BAD_ARG;
    drop_graphs(ctx);
    for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
    // released in the order of the context's stream, after its last work
    for (void *p : ctx->owned) cudaFreeAsync(p, ctx->last_stream);
    release_slot(ctx->slot);
    delete ctx;
    return LBM_OK;
}

const char *lbm_last_error(lbm_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"

// ------------------------------------------------------------------ ensembles
// An ensemble of air contexts stepped together with one launch per phase of
// the step and group of domains (lbm_batch.cuh).  Domains are ordered by
// collision model and split into groups of at most BATCH_GROUP; each group has
// its block maps and work items (built once), a stream and an event, and its
// steps are issued on that stream, interleaved with the other groups', so the
// phases of different groups overlap on the device.  The per-domain step
// arguments travel in each launch's parameters; the bed tables (which depend
// on the step's parity) are uploaded at the start of each call.
struct BatchGroupPlan {
    int d0 = 0, nd = 0;                 // the group's domains: [d0, d0 + nd) of lbm_batch::ctx
    int collision = LBM_COLLIDE_REGULARIZED;
    int tile_blocks = 0;
    BatchLaunch L{};                    // bed phase
    long long *d_col0 = nullptr;
    int4 *d_gmap = nullptr, *d_smap = nullptr, *d_items = nullptr;
    int ngen = 0, nsi = 0, nitems = 0;
    // fused steps with LES: the tiles off the edge of the domains that allow
    // tile copies (inner, kb_tile_tma) and all other tiles (edge, kb_tile)
    int4 *d_edge = nullptr, *d_inner = nullptr;
    int nedge = 0, ninner = 0;
    int tma_blocks = 0;
    int *d_queue = nullptr;             // [3]: all items, edge items, inner items
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};

struct lbm_batch {
    std::vector<lbm_ctx *> ctx;         // grouped order (by collision model, then the caller's order)
    std::vector<Plan> plan;
    std::vector<bool> stash;
    std::vector<bool> tma;              // domains whose inner tiles take the tile-copy grid
    bool pdl = true;                    // tile-copy grid behind the edge grid as a programmatic dependent launch
    std::vector<BatchGroupPlan> groups;
    int storage = 0;
    int arith = LBM_ARITH_EXACT;        // of the interior planes, uniform over the ensemble
    bool les = false;
    std::vector<StepArgs> h_tab;        // [2][n] step arguments by the step's index in the call, mod 2
    BatchBed *d_bed = nullptr, *h_bed = nullptr;
    std::unique_ptr<BatchGroup> G;      // parameters of the launch being issued
    cudaEvent_t start = nullptr;
    std::string err;
};

static int batch_fail(lbm_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    return code;
}

static void batch_free(lbm_batch *b) {
    for (BatchGroupPlan &g : b->groups) {
        cudaFree(g.d_col0);
        cudaFree(g.d_gmap);
        cudaFree(g.d_smap);
        cudaFree(g.d_items);
        cudaFree(g.d_edge);
        cudaFree(g.d_inner);
        cudaFree(g.d_queue);
        if (g.done) cudaEventDestroy(g.done);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    b->groups.clear();
    if (b->start) cudaEventDestroy(b->start);
    b->start = nullptr;
    cudaFree(b->d_bed);
    cudaFreeHost(b->h_bed);
    b->d_bed = nullptr;
    b->h_bed = nullptr;
}

template <typename T>
static cudaError_t upload_vec(T **dst, const std::vector<T> &v) {
    cudaError_t e = cudaMalloc((void **)dst, (v.empty() ? 1 : v.size()) * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// One phase of one group: the group's step arguments for the step's parity q,
// with the step number and flags of the launch, into the launch parameters.
// edge: the fused interior step on the edge item list only (the inner items
// go to the tile-copy grid, which = KER_TILE_TMA).
static void batch_issue(lbm_batch *b, const BatchGroupPlan &g, int which, int q, unsigned long long step, int flags,
                        bool edge = false) {
    const int n = (int)b->ctx.size();
    BatchGroup &G = *b->G;
    G.ndom = g.nd;
    for (int d = 0; d < g.nd; ++d) {
        G.a[d] = b->h_tab[(size_t)q * n + g.d0 + d];
        G.a[d].step = step;
        G.a[d].flags = flags;
    }
    G.queue = g.d_queue;
    G.pdl = 0;
    int blocks = g.tile_blocks;
    if (which == KER_TILE_TMA) {
        for (int d = 0; d < g.nd; ++d) {
            lbm_ctx *c = b->ctx[g.d0 + d];
            const int src = G.a[d].fsrc == c->b.f[0] ? 0 : 1;
            G.tmap[d][0] = c->tmap[src][0];
            G.tmap[d][1] = c->tmap[src][1];
        }
        G.map = g.d_inner;
        G.nmap = g.ninner;
        G.queue = g.d_queue + 2;
        G.pdl = b->pdl && g.nedge ? 1 : 0;
        blocks = g.tma_blocks;
    } else if (edge) {
        G.map = g.d_edge;
        G.nmap = g.nedge;
        G.queue = g.d_queue + 1;
        G.pdl = b->pdl ? 1 : 0;   // the edge launch zeroes the tile-copy grid's counter (d_queue + 2) too
    } else if (which == KER_TILE_CANON || which == KER_TILE_FUSED) {
        G.map = g.d_items;
        G.nmap = g.nitems;
    } else if (which == KER_STREAM_INTERIOR) {
        G.map = g.d_smap;
        G.nmap = g.nsi;
    } else {
        G.map = g.d_gmap;
        G.nmap = g.ngen;
    }
    launch_batch_group(which, b->storage, G, b->les, g.collision, b->arith, blocks, g.stream);
}

extern "C" {

int lbm_batch_create(lbm_ctx *const *ctxs, int32_t n, lbm_batch **out) {
    if (!ctxs || n < 1 || !out) return LBM_ERR_BAD_ARG;
    *out = nullptr;
    lbm_batch *b = new lbm_batch();
    lbm_ctx *c0 = ctxs[0];
    std::vector<Plan> plans(n);
    for (int d = 0; d < n; ++d) {
        lbm_ctx *c = ctxs[d];
        if (!c || !c->bound) {
            delete b;
            return LBM_ERR_NOT_BOUND;
        }
        const Plan R = plan_planes(c);
        std::string why;
        if (c->P.fs_mode != LBM_FS_NONE) why = "air domains only";
        else if (!c->use_cg) why = "bed-only geometry with periodic x (column-cache path) only";
        else if (!R.tile || R.classic) why = "the interior-plane path is required (nx, ny multiples of 16)";
        else if (c->P.pop_storage != c0->P.pop_storage) why = "one population storage for the whole ensemble";
        else if ((c->P.use_les != 0) != (c0->P.use_les != 0)) why = "LES on for every domain or for none";
        else if (c->arith != c0->arith) why = "one arithmetic (lbm_set_arithmetic) for the whole ensemble";
        else if (c->nstep != c0->nstep || c->cur != c0->cur) why = "every domain at the same step";
        if (!why.empty()) {
            delete b;
            return fail(c, LBM_ERR_UNSUPPORTED, "lbm_batch_create: domain " + std::to_string(d) + ": " + why);
        }
        plans[d] = R;
    }
    b->storage = c0->P.pop_storage;
    b->arith = c0->arith;
    b->les = c0->P.use_les != 0;
    // domains by collision model (regularized, then KBC), each in the caller's order
    std::vector<int> order(n);
    for (int d = 0; d < n; ++d) order[d] = d;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (ctxs[x]->P.collision == LBM_COLLIDE_KBC) < (ctxs[y]->P.collision == LBM_COLLIDE_KBC);
    });
    for (int d : order) {
        b->ctx.push_back(ctxs[d]);
        b->plan.push_back(plans[d]);
    }
    // groups: runs of one collision model, split evenly into at most BATCH_GROUP
    // domains each (LBM_B200_BATCH_GROUP lowers the bound)
    int gmax = BATCH_GROUP;
    if (const char *gv = getenv("LBM_B200_BATCH_GROUP")) {
        const int v = atoi(gv);
        if (v >= 1 && v < gmax) gmax = v;
    }
    for (int r0 = 0; r0 < n;) {
        int r1 = r0;
        while (r1 < n && b->ctx[r1]->P.collision == b->ctx[r0]->P.collision) ++r1;
        const int len = r1 - r0, ng = (len + gmax - 1) / gmax;
        for (int k = 0, d = r0; k < ng; ++k) {
            BatchGroupPlan g;
            g.d0 = d;
            g.nd = len / ng + (k < len % ng ? 1 : 0);
            g.collision = b->ctx[r0]->P.collision;
            d += g.nd;
            b->groups.push_back(g);
        }
        r0 = r1;
    }
    cudaError_t e = cudaSuccess;
    std::string where;
    // LBM_B200_BATCH_TMA=0: the cp.async-staged grid for every interior tile
    const char *tv = getenv("LBM_B200_BATCH_TMA");
    const bool tma_on = !(tv && tv[0] == '0');
    b->tma.assign(n, false);
    // LBM_B200_BATCH_PDL=0: the tile-copy grid in plain stream order after the edge grid
    const char *pv = getenv("LBM_B200_BATCH_PDL");
    b->pdl = !(pv && pv[0] == '0');
    for (BatchGroupPlan &g : b->groups) {
        std::vector<long long> col0(1, 0);
        std::vector<int4> gmap, smap, items, edge, inner;
        for (int ld = 0; ld < g.nd; ++ld) {
            const int d = g.d0 + ld;
            lbm_ctx *c = b->ctx[d];
            const Plan &R = b->plan[d];
            const int nx = c->P.nx, ny = c->P.ny;
            col0.push_back(col0.back() + (long long)nx * ny);
            const int gx = (nx + 31) / 32, gy = (ny + 7) / 8, gz = R.zcnt[0] + R.zcnt[1] + R.zcnt[2];
            for (int bz = 0; bz < gz; ++bz)
                for (int by = 0; by < gy; ++by)
                    for (int bx = 0; bx < gx; ++bx) gmap.push_back(make_int4(ld, bx, by, bz));
            const int ni = R.zi1 - R.zi0 + 1, tx = nx / LBM_TILE, ty = ny / LBM_TILE;
            for (int bz = 0; bz < ni; ++bz)
                for (int by = 0; by < ty; ++by)
                    for (int bx = 0; bx < tx; ++bx) smap.push_back(make_int4(ld, bx, by, bz));
            const int nc = (ni + R.chunk - 1) / R.chunk;
            // tile copies for the tiles off this domain's edge (fused steps with LES)
            const bool tma = tma_on && b->les && !R.classic && !R.no_tma && tx >= 3 && ty >= 3 &&
                             19.0 * (double)c->D.n < 2147483647.0 && tile_maps_ready(c);
            for (int cz = 0; cz < nc; ++cz)
                for (int by = 0; by < ty; ++by)
                    for (int bx = 0; bx < tx; ++bx) {
                        const int4 it = make_int4(ld, bx, by, cz);
                        items.push_back(it);
                        if (tma && bx >= 1 && bx <= tx - 2 && by >= 1 && by <= ty - 2) inner.push_back(it);
                        else edge.push_back(it);
                    }
            b->tma[d] = tma;
        }
        // longest items first: the last items of each queue are the short ones
        auto longest_first = [&](std::vector<int4> &v) {
            std::stable_sort(v.begin(), v.end(), [&](const int4 &x, const int4 &y) {
                const Plan &Rx = b->plan[g.d0 + x.x], &Ry = b->plan[g.d0 + y.x];
                const int px = std::min(Rx.chunk, Rx.zi1 + 1 - (Rx.zi0 + x.w * Rx.chunk));
                const int py = std::min(Ry.chunk, Ry.zi1 + 1 - (Ry.zi0 + y.w * Ry.chunk));
                return px > py;
            });
        };
        g.tma_blocks = inner.empty() ? 0 : batch_tile_blocks(b->storage, b->les, g.collision, b->arith, true);
        if (g.tma_blocks <= 0) {   // no tile-copy grid: every item on the cp.async grid
            inner.clear();
            edge = items;
            for (int ld = 0; ld < g.nd; ++ld) b->tma[g.d0 + ld] = false;
        }
        longest_first(items);
        longest_first(edge);
        longest_first(inner);
        g.ngen = (int)gmap.size();
        g.nsi = (int)smap.size();
        g.nitems = (int)items.size();
        g.nedge = (int)edge.size();
        g.ninner = (int)inner.size();
        if ((e = upload_vec(&g.d_col0, col0)) != cudaSuccess || (e = upload_vec(&g.d_gmap, gmap)) != cudaSuccess ||
            (e = upload_vec(&g.d_smap, smap)) != cudaSuccess || (e = upload_vec(&g.d_items, items)) != cudaSuccess ||
            (e = upload_vec(&g.d_edge, edge)) != cudaSuccess || (e = upload_vec(&g.d_inner, inner)) != cudaSuccess ||
            (e = cudaMalloc((void **)&g.d_queue, 3 * sizeof(int))) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming)) != cudaSuccess) {
            where = "group tables";
            break;
        }
        g.L.nall = n;
        g.L.d0 = g.d0;
        g.L.col0 = g.d_col0;
        g.L.ndom = g.nd;
        g.L.ncols = col0.back();
        g.tile_blocks = batch_tile_blocks(b->storage, b->les, g.collision, b->arith);
        // LBM_B200_BATCH_TILE_BLOCKS: fewer resident blocks for the interior grid, leaving
        // SM room for the other groups' kernels
        if (const char *tb = getenv("LBM_B200_BATCH_TILE_BLOCKS")) {
            const int v = atoi(tb);
            if (v > 0 && v < g.tile_blocks) g.tile_blocks = v;
        }
        if (g.tile_blocks <= 0) {
            batch_free(b);
            delete b;
            return fail(c0, LBM_ERR_UNSUPPORTED, "lbm_batch_create: the interior grid's shared memory was refused");
        }
    }
    // 16-bit storage with LES: the general pre-pass hands its FP32 populations to the collide through the stash
    for (int d = 0; d < n && e == cudaSuccess; ++d) {
        lbm_ctx *c = b->ctx[d];
        const Plan &R = b->plan[d];
        bool st = false;
        if (b->les && b->storage != LBM_STORE_F32) {
            const size_t ng = (size_t)(R.zcnt[0] + R.zcnt[1] + R.zcnt[2]) * c->P.nx * c->P.ny;
            if (c->stash_cells < ng) {
                float *p = nullptr;
                if (alloc(c, (void **)&p, 19 * ng * sizeof(float)) != LBM_OK) {
                    batch_free(b);
                    delete b;
                    return LBM_ERR_CUDA;
                }
                c->stash = p;
                c->stash_cells = ng;
            }
            st = true;
        } else if (b->les) {
            st = true;   // FP32: the pre-pass leaves them in the destination slots
        }
        b->stash.push_back(st);
    }
    if (e == cudaSuccess) {
        where = "tables";
        if ((e = cudaMalloc((void **)&b->d_bed, 2 * n * sizeof(BatchBed))) == cudaSuccess &&
            (e = cudaMallocHost((void **)&b->h_bed, 2 * n * sizeof(BatchBed))) == cudaSuccess)
            e = cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        batch_free(b);
        delete b;
        return fail(c0, LBM_ERR_CUDA, "lbm_batch_create: " + where + ": " + cudaGetErrorString(e));
    }
    for (BatchGroupPlan &g : b->groups) g.L.bed = b->d_bed;
    b->h_tab.resize(2 * (size_t)n);
    b->G.reset(new BatchGroup());
    *out = b;
    return LBM_OK;
}

int lbm_batch_step(lbm_batch *b, int32_t nsteps, void *stream) {
    if (!b || nsteps < 0) return LBM_ERR_BAD_ARG;
    if (nsteps == 0) return LBM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int n = (int)b->ctx.size();
    const int64_t n0 = b->ctx[0]->nstep;
    const int cur0 = b->ctx[0]->cur;
    for (lbm_ctx *c : b->ctx)
        if (c->nstep != n0 || c->cur != cur0) return batch_fail(b, LBM_ERR_BAD_ARG, "lbm_batch_step: domains out of step");
    // the bound bed state into the slots of step n0; the step arguments of the call
    for (int d = 0; d < n; ++d) {
        lbm_ctx *c = b->ctx[d];
        c->last_stream = st;
        // the tensor maps follow the context's population buffers
        if (b->tma[d] && !tile_maps_ready(c))
            return batch_fail(b, LBM_ERR_CUDA, "lbm_batch_step: tensor maps of domain " + std::to_string(d));
        const int s = load_bed_slot(c, (int)(n0 & 1), st);
        if (s != LBM_OK) return batch_fail(b, s, c->err);
        for (int q = 0; q < 2; ++q) {
            StepArgs A = step_args(c);
            apply_plan(A, b->plan[d]);
            const int src = cur0 ^ q;
            A.fsrc = c->b.f[src];
            A.fdst = c->b.f[1 - src];
            A.bed_s = slot_view(c, (int)((n0 + q) & 1));
            A.bed_c = slot_view(c, (int)((n0 + 1 + q) & 1));
            A.stash = c->stash;
            b->h_tab[(size_t)q * n + d] = A;
            const int par = q;   // bed variant by the parity of the bed step
            BatchBed &B = b->h_bed[par * n + d];
            B.P = c->P;
            B.D = c->D;
            B.h_prev = c->bed_h[1 - par];
            B.h = c->bed_h[par];
            B.hmax = c->bed_hmax[par];
            B.uw = c->bed_uw[par];
            B.vw = c->bed_vw[par];
            B.ww = c->bed_ww[par];
            B.cg = c->use_cg ? c->bed_cg[par] : nullptr;
            B.piecewise = c->b.piecewise_bed_z;
        }
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(b->d_bed, b->h_bed, 2 * n * sizeof(BatchBed), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaEventRecord(b->start, st)) != cudaSuccess)
        return batch_fail(b, LBM_ERR_CUDA, cudaGetErrorString(e));
    for (BatchGroupPlan &g : b->groups)
        if ((e = cudaStreamWaitEvent(g.stream, b->start, 0)) != cudaSuccess)
            return batch_fail(b, LBM_ERR_CUDA, cudaGetErrorString(e));
    const int tflag = b->stash[0] ? F_STASH : 0;
    const int K = nsteps;
    // step s of every group, then step s + 1: the groups' streams run side by side
    for (int s = 0; s < K; ++s) {
        const int64_t m = n0 + s;   // s = 0: collide from the stored post-stream state; then fused steps
        const int flags = ((s == K - 1) ? (F_WRITE_MACRO | F_WRITE_ALL_OMEGA) : 0) | tflag;
        const int q = s & 1;
        const unsigned long long step = (unsigned long long)(m + 1);
        for (BatchGroupPlan &g : b->groups) {
            launch_batch_bed(g.L, m + 1, g.stream);
            if (s == 0) {
                if (b->les) batch_issue(b, g, KER_PREPASS_CANON, 0, step, flags);
                batch_issue(b, g, KER_TILE_CANON, 0, step, flags);
                batch_issue(b, g, KER_COLLIDE_CANON, 0, step, flags);
            } else {
                if (b->les) batch_issue(b, g, KER_PREPASS_FUSED, q, step, flags);
                if (g.ninner) {
                    batch_issue(b, g, KER_TILE_FUSED, q, step, flags, true);
                    batch_issue(b, g, KER_TILE_TMA, q, step, flags);
                } else {
                    batch_issue(b, g, KER_TILE_FUSED, q, step, flags);
                }
                batch_issue(b, g, KER_COLLIDE_FUSED, q, step, flags);
            }
        }
    }
    // the final stream back to the post-stream state
    for (BatchGroupPlan &g : b->groups) {
        for (int d = g.d0; d < g.d0 + g.nd; ++d)
            if ((e = cudaMemsetAsync(b->ctx[d]->dcount, 0, 3 * sizeof(int), g.stream)) != cudaSuccess)
                return batch_fail(b, LBM_ERR_CUDA, cudaGetErrorString(e));
        batch_issue(b, g, KER_STREAM, K & 1, (unsigned long long)(n0 + K), F_COUNT);
        batch_issue(b, g, KER_STREAM_INTERIOR, K & 1, (unsigned long long)(n0 + K), F_COUNT);
        if ((e = cudaEventRecord(g.done, g.stream)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(st, g.done, 0)) != cudaSuccess)
            return batch_fail(b, LBM_ERR_CUDA, cudaGetErrorString(e));
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return batch_fail(b, LBM_ERR_CUDA, cudaGetErrorString(e));
    const int src_final = cur0 ^ (K & 1);
    for (lbm_ctx *c : b->ctx) {
        c->cur = 1 - src_final;
        c->nstep = n0 + K;
        const int s = store_bed_slot(c, (int)((n0 + K) & 1), c->bed_h[(n0 + K - 1) & 1], st);
        if (s != LBM_OK) return batch_fail(b, s, c->err);
    }
    return LBM_OK;
}

int lbm_batch_destroy(lbm_batch *b) {
    if (!b) return LBM_ERR_BAD_ARG;
    batch_free(b);
    delete b;
    return LBM_OK;
}

const char *lbm_batch_last_error(lbm_batch *b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
