// lbm_launch.h - argument structs and launchers shared by the device
// translation unit (lbm_device.cu) and the host API (lbm_api.cu).
#pragma once

#include <cuda.h>   // CUtensorMap (the type only)
#include <cuda_runtime.h>

#include "lbm_b200.h"
#include "lbm_dev.cuh"

namespace lbm {

enum : int {
    F_WRITE_MACRO = 1,      // store rho/ux/uy/uz of this collide
    F_WRITE_ALL_OMEGA = 2,  // store omega for every active cell (else near-wall band only)
    F_COUNT = 4,            // count cut / free-surface / bridge links in stream
    F_VOF_STATE = 8,        // free-surface state from stored type/fill (else from column height)
    F_TILE_CLASSIC = 16,    // interior planes: the unpipelined tile kernel even for FP32
    F_STASH = 32,           // general planes: the pre-pass leaves its populations in the destination for the collide
    F_TEST_WAIT_TIMEOUT = 64,  // tile-copy kernel: treat the first wait as timed out (tests of the error path)
};

enum {
    KER_PREPASS_CANON = 0, KER_PREPASS_FUSED = 1, KER_COLLIDE_CANON = 2, KER_COLLIDE_FUSED = 3, KER_STREAM = 4,
    KER_TILE_CANON = 5, KER_TILE_FUSED = 6, KER_STREAM_INTERIOR = 7,
    KER_TILE_TMA = 10   // ensembles: the fused interior step with LES on the tiles off the domain edge, tile copies
};
// device counters of a context (int slots)
enum { CNT_CUT = 0, CNT_FSCUT = 1, CNT_BRIDGE = 2, CNT_FS_REFILL = 3, CNT_COALESCE = 4, CNT_VOF_EXCESS = 5,
       CNT_ORPHAN = 6, CNT_COLLAPSE = 7, CNT_DET = 8, CNT_CMP = 9, CNT_SWEEPS = 10, CNT_N = 16 };
#define LBM_TILE 16   // interior tile edge (x and y); the tile path needs nx, ny multiples of it

struct StepArgs {
    lbm_params P;
    int slot;
    Dom D;
    const void *fsrc;  // populations read
    void *fdst;        // populations written
    BedView bed_s;     // geometry of the stream stage
    BedView bed_c;     // geometry of the condition/collide stage
    float *rho, *ux, *uy, *uz, *omega;
    const float *u_les;  // [3][n] velocities for the LES stencil
    float *u_out;        // [3][n] pre-pass output
    const float *fs_h, *fs_h_last;
    const float *fs_fill;
    const int8_t *fs_type;
    const float *u_inlet_profile;
    int *counters;       // [0] cut, [1] fs cut, [2] bridge
    unsigned *status;    // bit 0: non-finite density
    uint64_t step;       // 1-based step number of the collide stage (RNG key); with clock, the offset from *clock
    const long long *clock;  // device step clock of a captured step graph (null: step is absolute)
    float *stash;        // 16-bit storage with F_STASH: [19][general cells of the launch] FP32 post-condition populations
    int flags;
    // z planes covered by a launch: up to 3 ranges [zlo, zlo + zcnt), grid.z = sum of zcnt
    int zlo[3], zcnt[3];
    // interior planes [zi0, zi1] handled by the tile kernel (chunk planes per block)
    int zi0, zi1, chunk;
};

struct InitArgs {
    lbm_params P;
    int slot;
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

// edge of the coarse blocks of the VOF receivers' donor-in-reach flags
constexpr int VOF_CB = 4;
inline size_t vof_near_bytes(const Dom &D) {
    return (size_t)((D.nx + VOF_CB - 1) / VOF_CB) * ((D.ny + VOF_CB - 1) / VOF_CB) * ((D.nz + VOF_CB - 1) / VOF_CB);
}

// state and scratch of the VOF kernels
struct VofArgs {
    lbm_params P;
    int slot;
    Dom D;
    void *f;                          // populations after the stream (read/written in place)
    int8_t *type, *type_prev, *excess_dir;
    float *fill, *mass, *mass_excess;
    float *rho, *ux, *uy, *uz;
    const float *bed_h;               // bed height of the step
    float *fs_h, *fs_h_last;
    int8_t *open;                     // lattice_open[0] of the step's geometry
    float *lf0;                       // lattice_open_frac[0]
    float *m0, *x0;                   // snapshots: mass, and excess or fill
    int8_t *t0;                       // snapshot: type
    float *fa;                        // 6 n floats
    int8_t *ba;                       // 2 n bytes
    double *dd;                       // n doubles
    int *dist;                        // flood-fill distance of the last collapse pass (-1: not reached)
    uint8_t *near;                    // [2][cbz][cby][cbx] blocks of VOF_CB^3 cells with a donor within reach
                                      // (vof_near_*); the second half: scratch of the interface layer's marks
    int cbx, cby, cbz;
    int near_ok;                      // the periodic extents are multiples of VOF_CB (else the flags are not used)
    int *count;                       // integer counters (CNT_*)
    float *fcount;                    // float counters
};

struct ExportArgs {
    float *phi;
    int32_t *obstacle, *near_obstacle;
    int8_t *lattice_open;
    float *lattice_open_frac;
    int8_t *lattice_wall_type;
    float *prh, *gbf;
    int types_are_prev;  // pressure reference from fs_type_prev (after a step) or fs_type (after init)
};

cudaError_t upload_params(int slot, const lbm_params &P);
long long launch_count();
void launch_count_add(long long n);   // kernels run by a graph replay (or taken back after a capture)

// bed at time t; with a step clock, at t = (float)((*clock + off + 1) * dt_phys) read on the device
void launch_bed(const lbm_params &P, const Dom &D, const float *h_prev, float *h, float *hmax, float *uw, float *vw,
                float *ww, const float *piecewise, float t, cudaStream_t st, const long long *clock = nullptr,
                long long off = 0);
// *clock = value (the first node of a step-graph replay)
void launch_clock_set(long long *clock, long long value, cudaStream_t st);
void launch_hmax(const Dom &D, const float *h, float *hmax, cudaStream_t st);
void launch_colgeo(const lbm_params &P, const Dom &D, const BedView &B, float *cg, cudaStream_t st);
void launch_step_kernel(int which, const StepArgs &A, cudaStream_t st);
// fused interior step with LES (FP32) staged by tile copies; m24 / m20 are
// the source populations' tensor maps with boxes 24x18x1x1 and 20x18x1x1.
// false: not launched (shared memory of that size unavailable)
bool launch_tile_tma(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st);
// the same two grids with the fast arithmetic policy (lbm_fast.cu)
bool launch_tile_tma_fast(const StepArgs &A, const CUtensorMap *m24, const CUtensorMap *m20, cudaStream_t st);
void launch_column_flux(const StepArgs &A, float *qx, float *qy, cudaStream_t st);
// the water stream (height or VOF path): the compact kernel on the cells of
// water_stream_class, then the general stream on the cells it left, listed in
// list[*count] (list: one int per cell)
void launch_water_stream(const StepArgs &A, int *list, int *count, cudaStream_t st);
// the water collide: the compact kernel on the cells of water_collide_local, then the general collide on the
// cells it left, listed in list[*count]
void launch_water_collide(const StepArgs &A, int *list, int *count, cudaStream_t st);
void launch_advect(const lbm_params &P, const Dom &D, const float *bed_h, const float *qx, const float *qy,
                   const float *h_in, float *h_out, float *h_last, float t, cudaStream_t st);
void launch_refill(const StepArgs &A, const int8_t *type_prev, int *count, cudaStream_t st);
// VOF path: list the cells that turned wet (list: one int per cell and a count), mark their coarse blocks in
// V.near for the coalescence repair, refill the listed cells
void launch_refill_vof(const StepArgs &A, const VofArgs &V, const int8_t *type_prev, int *list, int *count,
                       cudaStream_t st);
void launch_height_types(const StepArgs &A, float *fill, int8_t *type, int8_t *type_prev, cudaStream_t st);

void launch_init_constants(const InitArgs &I, cudaStream_t st);
void launch_fs_height_init(const InitArgs &I, cudaStream_t st);
void launch_classify_store(const InitArgs &I, cudaStream_t st);
void launch_vof_block(const InitArgs &I, cudaStream_t st);
void launch_init_fields(const InitArgs &I, cudaStream_t st);
void launch_vof_mass_init(const InitArgs &I, cudaStream_t st);
void launch_export(const InitArgs &I, const ExportArgs &E, cudaStream_t st);

void launch_vof_open(const VofArgs &V, const BedView &B, cudaStream_t st);
cudaError_t vof_interface_layer(const VofArgs &V, cudaStream_t st);
void launch_vof_height(const VofArgs &V, cudaStream_t st);
cudaError_t vof_sequence(const VofArgs &V, bool collapse_due, double *tree, cudaStream_t st);
void launch_vof_coalesce(const VofArgs &V, cudaStream_t st);
void launch_vof_exterior(const Dom &D, const int *dist, int32_t *out, cudaStream_t st);

// ---- device reductions of the harness metrics (lbm_diag.cuh)
struct DiagCellPart {
    unsigned long long max_key;   // (speed bits << 32) | (0xffffffff - cell): the first maximum wins ties
    long long active, tiny, excess_count;
    double fill_sum, mass_sum, excess_sum;
    float min_iface;
    int pad;
};
// masked sums of the slice: quantities p, p_hp, pt, pt_hp, v, v_hp over the
// wall band and over the free-surface band
struct DiagSlicePart {
    double s[2][6], s2[2][6];
    long long n[2];
};

struct DiagArgs {
    lbm_params P;
    int slot;
    Dom D;
    BedView bed;                 // geometry of the current step (no column cache)
    const float *rho, *ux, *uy, *uz, *fill, *mass, *excess, *fs_h;
    const int8_t *type, *type_prev;
    int types_are_prev;          // the pressure reference of the last step used the previous types
    int fs, vof;                 // free surface enabled, VOF tracking
    int slice_j;
    double rho_phys, gravity_phys;
    DiagCellPart *cellp;         // [gridDim of k_diag_cells]
    int ncellp;
    double *col_eta;             // [nx] sum over y of the surface height
    float *col_min, *col_max;    // [nx]
    double *sl_p, *sl_pt, *sl_v; // [nz][nx] slice fields
    uint8_t *sl_mask;            // [nz][nx] bit 0 inactive, bit 1 wall band, bit 2 free-surface band
    DiagSlicePart *slp;          // [2][nslp]: partials of the two passes of k_diag_slice_sum
    int nslp;
    double *slice_mean;          // [2][6] band means of the first pass
    lbm_diag *out;
};

constexpr int DIAG_THREADS = 256;
constexpr int DIAG_SLICE_THREADS = 128;   // 128 slice partials of 208 bytes fit static shared memory

void launch_diagnostics(const DiagArgs &G, cudaStream_t st);

// ---- ensembles stepped with one launch per phase and group (lbm_batch.cuh)
// One domain's 2-D bed state for the bed step of one parity.
struct BatchBed {
    lbm_params P;
    Dom D;
    const float *h_prev, *piecewise;
    float *h, *hmax, *uw, *vw, *ww;
    float *cg;                       // column cache of the slot (null without one)
};
// the bed phase of one group: one thread per column of its domains
struct BatchLaunch {
    const BatchBed *bed;             // [2][nall] by the parity of the bed step, whole ensemble
    int nall;                        // domains of the ensemble
    int d0;                          // ensemble index of the group's first domain
    const long long *col0;           // [ndom + 1] first column of each of the group's domains
    int ndom;
    long long ncols;
};
// Domains per launch of the step grids.  Their step arguments and the
// tensor maps of their source populations travel in the kernel's parameter
// space (read-only, at most 32,764 bytes), so that the shared bodies read
// them, indexed by the block's domain, as a domain's own kernel reads its
// arguments, without copies to shared memory or registers.
constexpr int BATCH_GROUP = 28;
struct BatchGroup {
    CUtensorMap tmap[BATCH_GROUP][2];  // interior tile-copy grid: boxes 24 and 20 wide (one map for 16-bit storage)
    const int4 *map;                 // general / stream blocks: (domain, bx, by, bz); interior grids: work
                                     // items (domain, tile x, tile y, z chunk); domain = index in a[]
    int nmap;
    int ndom;
    int *queue;                      // interior grids: next work item
    int pdl;                         // interior grids: the tile-copy grid follows the edge grid as a programmatic
                                     // dependent launch (the edge launch zeroes both counters)
    StepArgs a[BATCH_GROUP];         // step arguments of the launch (step number and flags included)
};
static_assert(sizeof(BatchGroup) <= 32764, "kernel parameter space");

// bed, 3x3 maximum and column cache of the group's domains at step m
void launch_batch_bed(const BatchLaunch &L, long long m, cudaStream_t st);
// one phase over one group (which = KER_PREPASS_*, KER_TILE_*, KER_TILE_TMA, KER_COLLIDE_*, KER_STREAM,
// KER_STREAM_INTERIOR); the group's domains share storage, LES and collision model; arith: the interior
// planes' policy (LBM_ARITH_*); tile_blocks: resident blocks of the interior grid
void launch_batch_group(int which, int storage, const BatchGroup &G, bool les, int collision, int arith,
                        int tile_blocks, cudaStream_t st);
// resident blocks of the interior grid (tma: the tile-copy grid) on this device (0: the shared memory is refused)
int batch_tile_blocks(int storage, bool les, int collision, int arith, bool tma = false);
// the fast-arithmetic interior grids of a group (lbm_fast.cu)
void launch_batch_tile_fast(int which, int storage, const BatchGroup &G, bool les, int collision, int tile_blocks,
                            cudaStream_t st);
int batch_tile_blocks_fast(int storage, bool les, int collision, bool tma);

}  // namespace lbm
