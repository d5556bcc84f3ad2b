/*
 * lbm_b200.h - C ABI of the B200-native D3Q19 step engine.
 *
 * This is the drop-in boundary for the per-timestep hot path of the
 * air-over-waves LES / free-surface solver
 * (reference: LBM_3D_LES_air_over_waves_CODEX.py).  The reference has no
 * FFI of its own: its interface is the Python module surface that
 * run_ab_case.py drives (module globals, Taichi fields, main()).  The
 * Python host layer of this project re-creates that module surface and
 * calls down into this ABI through ctypes.
 *
 * Conventions
 *   - Plain C types only; no C++ or torch types cross the boundary.
 *   - The library never allocates or frees state buffers: the caller owns
 *     every pointer in lbm_buffers (device pointers for the CUDA library,
 *     host pointers for the CPU oracle, which exports the same ABI).  The
 *     CUDA library owns only small scratch arrays, freed by lbm_destroy.
 *   - Every call returns an int status (LBM_OK or a negative LBM_ERR_*).
 *     No exceptions cross the ABI.  lbm_last_error() gives a message.
 *   - A context is bound to one stream and is not thread-safe.  Separate
 *     contexts may run concurrently on separate streams.
 *   - 3-D fields are [nz][ny][nx] with x fastest (the reference's Taichi
 *     field order (Nz, Ny, Nx), CODEX.py:531-620).  Populations are stored
 *     structure-of-arrays: f[q][nz][ny][nx], q in the D3Q19 order of
 *     lbm_lattice.py:3-43.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* status codes */
#define LBM_OK 0
#define LBM_ERR_BAD_ARG (-1)
#define LBM_ERR_CUDA (-2)
#define LBM_ERR_NOT_CONVERGED (-3)
#define LBM_ERR_NONFINITE (-4)
#define LBM_ERR_UNSUPPORTED (-5)
#define LBM_ERR_NOT_BOUND (-6)

/* enumerations (values mirror the reference's string options) */
enum { LBM_FS_NONE = 0, LBM_FS_HEIGHT_STATIC = 1, LBM_FS_HEIGHT_KINEMATIC = 2, LBM_FS_PRESCRIBED_SOLITARY = 3 };
enum { LBM_TRACK_HEIGHT = 0, LBM_TRACK_VOF = 1 };
enum { LBM_FSB_CELL = 0, LBM_FSB_HYDROSTATIC = 1 };
enum { LBM_REFILL_EQUILIBRIUM = 0, LBM_REFILL_NONEQ = 1, LBM_REFILL_DIRECTIONAL = 2 };
enum { LBM_FSINIT_FLAT = 0, LBM_FSINIT_SOLITARY = 1, LBM_FSINIT_GAUSSIAN = 2 };
enum { LBM_PRESSURE_TOTAL = 0, LBM_PRESSURE_HYDROSTATIC_BALANCED = 1, LBM_PRESSURE_VOF_COMPONENT_BALANCED = 2 };
enum { LBM_BED_MOVING_SINE = 0, LBM_BED_FLAT = 1, LBM_BED_PIECEWISE = 2 };
enum { LBM_COLLIDE_KBC = 0, LBM_COLLIDE_REGULARIZED = 1 };
enum { LBM_INITVEL_REFERENCE = 0, LBM_INITVEL_UNIFORM = 1 };
enum { LBM_SOLVEL_NONE = 0, LBM_SOLVEL_SHALLOW = 1, LBM_SOLVEL_SHALLOW_DIVFREE = 2 };
enum { LBM_STORE_F32 = 0, LBM_STORE_F16S = 1, LBM_STORE_BF16S = 2 };

/* free-surface cell states (CODEX.py:407-409) */
#define LBM_FS_GAS 0
#define LBM_FS_LIQUID 1
#define LBM_FS_INTERFACE 2
/* wall sources (CODEX.py:401-405) */
#define LBM_WALL_NONE 0
#define LBM_WALL_BED 1
#define LBM_WALL_CUBE 2
#define LBM_WALL_XMIN 3
#define LBM_WALL_XMAX 4

/*
 * Solver constants, exactly as the kernels use them.  The host layer
 * derives every value from the reference's LBM_* environment options
 * (CODEX.py:35-529) and rounds to float the way Taichi captures Python
 * constants into f32 kernels.
 */
typedef struct lbm_params {
    int32_t abi_version;
    int32_t nx, ny, nz;

    /* ---- modes (CODEX.py:49-208, 355-409, 481-528) ---- */
    int32_t physics_water;          /* LBM_PHYSICS_MODE: 0 air, 1 water */
    int32_t fs_mode;                /* LBM_FREE_SURFACE_MODE -> LBM_FS_* */
    int32_t fs_tracking;            /* LBM_FREE_SURFACE_TRACKING -> LBM_TRACK_* */
    int32_t fs_boundary;            /* LBM_FREE_SURFACE_BOUNDARY -> LBM_FSB_* */
    int32_t fs_refill;              /* LBM_FREE_SURFACE_REFILL -> LBM_REFILL_* */
    int32_t fs_initial;             /* LBM_FREE_SURFACE_INITIAL -> LBM_FSINIT_* */
    int32_t init_fs_populations;    /* LBM_INIT_FREE_SURFACE_POPULATIONS */
    int32_t vof_link_aperture;      /* LBM_VOF_LINK_APERTURE */
    int32_t vof_initial_block;      /* LBM_VOF_INITIAL_SHAPE == block */
    int32_t pressure_formulation;   /* LBM_PRESSURE_FORMULATION -> LBM_PRESSURE_* */
    int32_t use_hydrostatic_balanced_pressure;  /* CODEX.py:457-460 */
    int32_t use_component_balanced_pressure;    /* CODEX.py:454-456 */
    int32_t x_solid;                /* LBM_X_BOUNDARY == solid */
    int32_t use_phi_open_fraction;  /* LBM_BOUNDARY_GEOMETRY in (phi_fraction, phi) */
    int32_t use_phi_open_flags;     /* LBM_BOUNDARY_GEOMETRY == phi */
    int32_t use_link_wall_velocity; /* LBM_WALL_VELOCITY_SAMPLING == link */
    int32_t bed_profile;            /* LBM_BED_PROFILE -> LBM_BED_* */
    int32_t include_bed;            /* LBM_OBSTACLE_MODE in (bed, bed_cube) */
    int32_t include_cube;           /* LBM_OBSTACLE_MODE in (bed_cube, cube) */
    int32_t use_les;                /* LBM_USE_LES */
    int32_t collision;              /* LBM_COLLISION -> LBM_COLLIDE_* */
    int32_t enable_top_drive;       /* CODEX.py:526 */
    int32_t enable_x_fringe;        /* CODEX.py:527 */
    int32_t enable_top_sponge;      /* CODEX.py:528 */
    int32_t solitary_velocity_mode; /* LBM_SOLITARY_INITIAL_VELOCITY -> LBM_SOLVEL_* */
    /* extensions (not in the reference; defaults reproduce it) */
    int32_t top_free_slip;          /* specular top wall for air runs */
    int32_t init_velocity_mode;     /* LBM_INITVEL_*: reference log-law kick or uniform + noise */
    int32_t bed_orbital_velocity;   /* 1: reference u_s = c*eta/(h0+eta) terms; 0: u_s = 0 */
    int32_t pop_storage;            /* LBM_STORE_*: population storage precision */

    /* ---- VOF options (CODEX.py:101-154, 174-184) ---- */
    int32_t vof_orphan_search_radius;
    int32_t vof_orphan_max_weak_neighbors;
    int32_t vof_detached_advection;
    int32_t vof_detached_max_wet_neighbors;
    int32_t vof_detached_max_resolved_neighbors;
    int32_t vof_thin_gap_bridge;
    int32_t vof_collapse_enabled;
    int32_t vof_collapse_interval;
    int32_t vof_collapse_flood_sweeps;
    int32_t pad0;

    uint64_t seed;                  /* counter-based RNG key (backscatter) */

    /* ---- lattice / physical constants (f32 as the kernels use them) ---- */
    float dx;                       /* LBM_DX_M */
    float rho0;                     /* CODEX.py:414 */
    float tau0;                     /* CODEX.py:466 (or build override) */
    float nu0;                      /* CODEX.py:465 */
    float cs_delta_sq;              /* (Cs*Delta)**2, CODEX.py:3094 */
    float nu_t_max;                 /* CODEX.py:500 */
    float kappa;                    /* CODEX.py:516 */
    float z0_phys;                  /* CODEX.py:517 */
    float wall_dist_floor;          /* 0.001*dx, CODEX.py:3103 */
    float ti_kick;                  /* TI, CODEX.py:507 */
    float c_backscatter;            /* LBM_BACKSCATTER */
    float u_top_lb;                 /* CODEX.py:446 */
    float u_current_lb;             /* CODEX.py:448 */
    float g_lb;                     /* CODEX.py:449 */
    float g_body_lb;                /* CODEX.py:461-463 */
    float vel_scale;                /* CODEX.py:441 */
    float dt_phys_f;                /* dt_phys rounded to f32 (in-kernel use) */
    double dt_phys;                 /* dt_phys in double: t = (step+1)*dt_phys */

    /* bed kinematics (CODEX.py:1082-1162); the reference uses two
       harmonics: (amp, 0.5k, c) and (amp, k, 0.5c) */
    float bed_offset_m;
    float bed_amp1, bed_k1, bed_c1;
    float bed_amp2, bed_k2, bed_c2;
    float bed_ramp_time;            /* 2*wave_period (0 = no ramp) */
    float bed_h0;                   /* depth_swl_m */

    /* cube / prism obstacle (CODEX.py:369-400) */
    float cube_cx, cube_cy, cube_cz;
    float cube_hx, cube_hy, cube_hz;
    float cube_yaw_cos, cube_yaw_sin, cube_pitch_cos, cube_pitch_sin;

    /* free surface (CODEX.py:291-339) */
    float fs_base_m;
    float fs_depth_m;
    float solitary_amp_m, solitary_x0_m, solitary_direction, solitary_celerity, solitary_kappa_inv;
    float gaussian_amp_m, gaussian_center_x_m, gaussian_sigma_m;
    float vof_block_xmin, vof_block_xmax, vof_block_ymin, vof_block_ymax, vof_block_zmin, vof_block_zmax;

    /* VOF thresholds */
    float vof_empty_fill_threshold;
    float vof_orphan_empty_threshold;
    float vof_detached_residual_fill_threshold;
    float vof_thin_gap_bridge_strength;
    float vof_collapse_max_volume_m3;

    /* extension: uniform initial velocity (LBM_INITVEL_UNIFORM) */
    float init_u0x, init_u0y, init_u0z, init_noise_amp;

    /* Python-side constant folds the kernels use (Taichi evaluates pure
       Python sub-expressions in double and captures the result as f32) */
    float omega0;                   /* 1.0/tau0, CODEX.py:1047 */
    float half_inv_dx;              /* 0.5/dx, CODEX.py:2459 */
    float solitary_dir_cel;         /* direction*celerity, CODEX.py:1169 */
    float nu_lbm_init;              /* (tau0-0.5)/3, CODEX.py:2722 */
    float u_tau_init;               /* 0.1*u_top_lb, CODEX.py:2721 */
    float inv_kappa;                /* 1.0/kappa, CODEX.py:2731 */
    float one_third;                /* 1.0/3.0 as f32 */
    int32_t magic_end;              /* must equal LBM_PARAMS_MAGIC */
} lbm_params;

#define LBM_PARAMS_MAGIC 0x1B200D19

/*
 * Caller-owned buffers.  Pointers not needed by the configured mode may be
 * NULL (lbm_bind checks what the mode needs).  "n" = nz*ny*nx cells,
 * "a" = ny*nx columns.
 */
typedef struct lbm_buffers {
    void *f[2];              /* 19*n populations (float, or 16-bit shifted per pop_storage) */
    float *rho, *ux, *uy, *uz;   /* n each: moments (reference rho/ux/uy/uz) */
    float *omega;            /* n: persistent local relaxation rate (omegaLoc) */
    /* 2-D columns */
    float *water_h, *water_h_last;       /* a: bed height (reference name) */
    float *u_wave, *v_wave, *w_wave;     /* a: bed velocity, lattice units */
    float *fs_h, *fs_h_last;             /* a: free_surface_h / _last */
    float *fs_flux_x, *fs_flux_y;        /* a: column fluxes */
    float *piecewise_bed_z;              /* nx */
    float *u_inlet_profile;              /* nz */
    /* initialisation inputs */
    float *rho_initial;                  /* n */
    float *init_noise;                   /* 3*n uniform in [-1,1): kick / noise x,y,z */
    /* free surface 3-D state */
    float *fs_fill;                      /* n */
    int8_t *fs_type, *fs_type_prev;      /* n */
    float *fs_mass, *fs_mass_excess;     /* n */
    int8_t *fs_excess_dir;               /* n */
    /* diagnostics written only by lbm_export_diagnostics (may be NULL) */
    float *phi;                          /* n */
    int32_t *obstacle, *near_obstacle;   /* n */
    int8_t *lattice_open;                /* 19*n, [q][cell] */
    float *lattice_open_frac;            /* 19*n */
    int8_t *lattice_wall_type;           /* 19*n */
    float *pressure_reference_head, *gravity_body_fraction;  /* n */
    int32_t *vof_exterior_gas;           /* n: flood-fill labels of the last collapse pass */
} lbm_buffers;

/* Scalar diagnostics (reference CODEX.py:600-620). */
typedef struct lbm_counters {
    int32_t boundary_refill_count;
    int32_t free_surface_refill_count;
    int32_t free_surface_coalescence_repair_count;
    int32_t free_surface_thin_gap_bridge_count;
    int32_t free_surface_cut_link_count;
    int32_t free_surface_vof_excess_count;
    int32_t free_surface_vof_orphan_count;
    int32_t free_surface_vof_collapse_cell_count;
    int32_t free_surface_vof_detached_advect_count;
    int32_t free_surface_vof_detached_compress_count;
    int32_t boundary_cut_link_count;
    int32_t status_flags;                /* bit 0: non-finite density seen; bit 1: an interior-kernel
                                            precondition (cell far from the bed) failed; bit 2: a
                                            bounded wait for a tile copy gave up (that launch's
                                            results are incomplete) */
    float free_surface_vof_collapse_candidate_volume_m3;
    float free_surface_vof_collapse_applied_volume_m3;
    float free_surface_vof_collapse_removal_scale;
    float free_surface_vof_collapse_candidate_mass;
    float free_surface_vof_collapse_exterior_capacity;
    float free_surface_vof_detached_advect_mass;
    float free_surface_vof_detached_compress_mass;
    float pad;
    int64_t step;                        /* steps completed since init */
    int32_t current_f;                   /* index (0/1) of the buffer holding f */
    int32_t flood_sweeps_used;           /* last collapse pass: sweeps until the marks stopped changing */
} lbm_counters;

/* Inputs of lbm_diagnostics that are not solver constants. */
typedef struct lbm_diag_inputs {
    double rho_phys;        /* fluid density [kg/m^3]: pressures are reported in Pa */
    double gravity_phys;    /* [m/s^2] */
    int32_t slice_j;        /* y index of the xz slice (the reference uses Ny / 2) */
    int32_t pad;
} lbm_diag_inputs;

/* The per-plot metric row of run_ab_case.py (make_visualize,
   run_ab_case.py:283-679) and the health line of main() (CODEX.py:3930-3937),
   reduced on the device.  NaN (or -1 for counts) where the reference writes
   NaN / -1 for the mode.  Sums are FP64; the reference's float32 numpy sums
   agree to rounding. */
typedef struct lbm_diag {
    /* maximum speed over active cells (not solid, and not gas with a free surface) */
    double max_speed_lb;               /* lattice units (the health line's Max |U|) */
    double max_speed_phys;             /* m/s */
    double max_speed_x, max_speed_y, max_speed_z;   /* cell centre of the first maximum in C order */
    int32_t max_k, max_j, max_i;
    int32_t max_speed_fs_type;         /* free-surface state there (-1 without a free surface) */
    double max_speed_fs_fill;
    int32_t max_speed_wet_neighbors, max_speed_full_neighbors, max_speed_gas_neighbors;
    int32_t pad0;
    int64_t active_cells;
    /* volumes and VOF accounting (run_ab_case.py:299-347) */
    double water_volume;               /* m^3: fill summed over open cells times dx^3 */
    double vof_mass_total;
    double vof_min_interface_fill;
    int64_t vof_tiny_interface_count;
    double vof_pending_excess_mass;
    int64_t vof_pending_excess_count;
    /* free-surface line: mean over y of the surface elevation (run_ab_case.py:348-363) */
    double surface_min, surface_max;
    double surface_symmetry_l2, surface_eta_hp_rms, surface_left_max, surface_right_max;
    /* xz slice at slice_j: pressure [Pa] and vorticity statistics over the near-wall band
       0 < phi <= 10 dx and over the free-surface band (run_ab_case.py:431-596); the
       linear-wave residual columns are not computed here */
    double p_rms, p_hp_rms, p_total_rms, p_total_hp_rms, vort_rms, vort_hp_rms;
    double fs_p_rms, fs_p_hp_rms, fs_p_total_rms, fs_p_total_hp_rms, fs_vort_rms, fs_vort_hp_rms;
    int64_t band_cells, fs_band_cells;
} lbm_diag;

typedef struct lbm_ctx lbm_ctx;

/* Library identity: "cuda-sm100a" or "cpu-oracle". */
const char *lbm_backend_name(void);
int lbm_abi_version(void);
/* sizeof(lbm_params), sizeof(lbm_buffers), sizeof(lbm_counters),
   sizeof(lbm_diag), sizeof(lbm_diag_inputs) for which = 0 .. 4: lets a
   binding check its struct layout. */
int64_t lbm_struct_size(int32_t which);

/* Create a context from constants; replaces module import + field
   allocation (CODEX.py:35-620). */
int lbm_create(const lbm_params *params, lbm_ctx **out);

/* Bind caller-owned buffers (replaces the ti.field set, CODEX.py:531-620). */
int lbm_bind(lbm_ctx *ctx, const lbm_buffers *bufs);

/* Initialisation, phase 1: constants, bed at t=0, geometry, initial free
   surface height, classification, VOF block shape
   (CODEX.py:3776-3785 up to update_pressure_reference_fields).  After it
   the caller computes rho_initial on the host (prepare_initial_density_field,
   CODEX.py:743-818) from water_h and fs_h. */
int lbm_init_geometry(lbm_ctx *ctx, void *stream);

/* Initialisation, phase 2: init_fields, free-surface boundary populations,
   VOF mass from fill, interface layer, column height
   (CODEX.py:3787-3792).  Reads rho_initial and init_noise. */
int lbm_init_fields(lbm_ctx *ctx, void *stream);

/* Advance nsteps timesteps (the loop body CODEX.py:3873-3925). */
int lbm_step(lbm_ctx *ctx, int32_t nsteps, void *stream);

/* Write the derived per-cell fields the reference keeps resident (phi,
   obstacle, lattice_open*, near_obstacle, pressure reference) for the
   current step's geometry into the bound diagnostic buffers. */
int lbm_export_diagnostics(lbm_ctx *ctx, void *stream);

/* Copy scalar counters to the host (synchronises the stream). */
int lbm_read_counters(lbm_ctx *ctx, lbm_counters *out);

/* Device-side metrics of the current state, in place of the host reductions
   of run_ab_case.py:283-679 (its per-plot metric row) and of the health line
   (CODEX.py:3930-3937), which both pull whole fields to the host.  The
   reductions run on stream and only the lbm_diag record comes back; the call
   synchronises stream.  Obstacle and phi are recomputed from the current
   step's geometry, so no diagnostic buffer needs to be bound.  The first call
   allocates a small scratch (a few slice-sized arrays).  The CPU oracle
   returns LBM_ERR_UNSUPPORTED. */
int lbm_diagnostics(lbm_ctx *ctx, const lbm_diag_inputs *in, lbm_diag *out, void *stream);

/* Measurement hook (no counterpart in the reference): when enabled, the
   library brackets every launch of its dominant step kernel (the interior
   one-pass kernel) with CUDA events on the caller's stream.
   lbm_kernel_timing synchronises and returns the summed device time, the
   number of launches and the cells one launch updates.  The CPU oracle
   reports zeros. */
int lbm_set_kernel_timing(lbm_ctx *ctx, int32_t enable);
int lbm_kernel_timing(lbm_ctx *ctx, double *total_ms, int64_t *launches, int64_t *cells_per_launch);
/* Tuning hook (no counterpart in the reference): planes per thread block of
   the interior kernel, the work unit of its z march (0 restores the built-in
   choice).  lbm_b200.tuning picks it by timing candidates.  The CPU oracle
   accepts and ignores it. */
int lbm_set_tile_chunk(lbm_ctx *ctx, int32_t planes);
/* Arithmetic of the fused interior kernels (no counterpart in the reference).
   LBM_ARITH_EXACT evaluates every expression in the reference's operation
   order without multiply-add contraction, bit-equal to the CPU oracle.
   LBM_ARITH_FAST evaluates the same collision, LES rate and moments of the
   interior cells (every cell away from the bed and the top) in a reorganised
   form with contraction: the regularized and BGK collisions by opposite
   pairs of directions (shared equilibrium terms and Hermite projections).
   Its results differ from the
   exact ones by rounding; geometry, flags and every near-wall cell are
   computed exactly in both modes.  New contexts take LBM_B200_ARITH
   (fast or exact) from the environment, else exact.  Changing the mode drops
   captured step graphs.  The CPU oracle accepts and ignores it. */
#define LBM_ARITH_EXACT 0
#define LBM_ARITH_FAST 1
int lbm_set_arithmetic(lbm_ctx *ctx, int32_t mode);
int lbm_get_arithmetic(lbm_ctx *ctx, int32_t *mode);
/* Step graphs (no counterpart in the reference; the reference launches
   every kernel from its Python step loop): when enabled, each lbm_step call
   of the air path or of the kinematic height path runs as one CUDA graph
   launch.  The first call of a given
   step count, step parity and current population buffer is captured on the
   caller's stream (nothing runs during the capture) and kept; every later
   call of that shape replays it after one launch that writes the step
   number to a device clock, from which the captured kernels take the bed
   time and the random-kick key.  Results are those of the eager calls, bit
   for bit.  Graphs need a stream of the caller's (not the legacy default
   stream) and start after one eager call; they are dropped by lbm_bind,
   lbm_set_tile_chunk with a new value and lbm_destroy, and not used while
   kernel timing is on.  A refused capture turns the context back to eager
   calls.  The VOF path, the static height and the prescribed solitary
   height return LBM_ERR_UNSUPPORTED (the VOF step decides on the host; the
   prescribed height reads the host's step time).  The CPU oracle accepts
   and ignores it. */
int lbm_set_step_graphs(lbm_ctx *ctx, int32_t enable);

/* Measurement hook (no counterpart in the reference): number of kernels the
   library has launched in this process, over all contexts.  The CPU oracle
   reports 0. */
int lbm_launch_count(int64_t *count);

/* Allocation-free link geometry (no counterpart in the reference).
   Writes, for the bed height field bed_h ([ny][nx], device) and the grid
   and geometry options in params, the same per-cell link geometry that
   lbm_export_diagnostics writes after a step: phi, obstacle, near_obstacle
   ([nz][ny][nx]) and lattice_open, lattice_open_frac, lattice_wall_type
   ([19][nz][ny][nx]).  Any output pointer may be NULL.  It needs no
   context and allocates nothing.  It is meant for callers that must not
   call cudaMalloc but still want the open flags and fractions of a bed
   shape (a visualisation or analysis hook).  Examples: a serving process
   whose device memory is fully committed to population buffers by its
   admission budget; a host framework that owns all device memory through
   its own caching allocator, where a raw cudaMalloc would synchronise the
   device and fragment the pool.
   Scratch is a fixed device array of 9 floats per column, sized for at
   most LBM_NOALLOC_MAX_COLUMNS columns (nx*ny; 2.25 MiB, held by every
   GPU that loads the library until the process exits); larger grids are
   rejected with LBM_ERR_BAD_ARG.  Bed geometry only (no cube, no phi
   geometry, periodic x), else LBM_ERR_UNSUPPORTED.  Runs on the calling
   thread's current device, asynchronously on stream (which must belong to
   that device).  Outside stream capture every call looks up the array's
   device address afresh, so a device reset or a new driver context is
   picked up; a call made while stream is being captured uses the address
   of the last call on that device outside capture, so make one call
   before any capture (and again after a device reset).  All calls
   share the one array: calls that overlap on the GPU (other streams, other
   threads) race and must be serialised by the caller.  Each call rewrites
   every entry it reads, so nothing needs clearing between calls.  err (may
   be NULL) receives a message of at most err_len bytes on failure.  The
   CPU oracle returns LBM_ERR_UNSUPPORTED. */
#define LBM_NOALLOC_MAX_COLUMNS 65536
int lbm_link_geometry_noalloc(const lbm_params *params, const float *bed_h, float *phi, int32_t *obstacle,
                              int32_t *near_obstacle, int8_t *lattice_open, float *lattice_open_frac,
                              int8_t *lattice_wall_type, void *stream, char *err, size_t err_len);

int lbm_destroy(lbm_ctx *ctx);
const char *lbm_last_error(lbm_ctx *ctx);

/* Ensembles (no counterpart in the reference, which runs one domain per
   process; replaces running run_ab_case.py once per ensemble member):
   independent air contexts stepped together.  The contexts are ordered by
   collision model and split into groups of at most 28; each group runs one
   launch per phase of the step on a stream of the library's, joined to
   `stream` at the end of the call.  The interior planes of a group's
   domains form work queues of (domain, tile, z chunk) items taken by grids
   of resident blocks (tile copies for the tiles off each domain's edge,
   cp.async staging for the others), so domains of uneven size share the
   SMs; the planes next to the bed and the top, the bed and the final
   stream run as single grids over block maps of the group's domains.
   Results equal those of stepping each context with lbm_step, bit for bit,
   with the exact arithmetic (with the fast one, a domain of fewer than 3 x 3
   tiles differs by rounding: its own calls take the exact cp.async kernel
   for the interior).  Requirements: every context bound and
   initialised, air mode with bed-only geometry and periodic x, nx and ny
   multiples of 16, one population storage, one arithmetic
   (lbm_set_arithmetic), LES on for all or none, all at the same step; else LBM_ERR_UNSUPPORTED (message in lbm_last_error of the
   offending context).  lbm_batch_step advances every context by nsteps on
   stream (the contexts' own calls may be used between batch calls, keeping
   them at one step).  The CPU oracle returns LBM_ERR_UNSUPPORTED. */
typedef struct lbm_batch lbm_batch;
int lbm_batch_create(lbm_ctx *const *ctxs, int32_t n, lbm_batch **out);
int lbm_batch_step(lbm_batch *b, int32_t nsteps, void *stream);
int lbm_batch_destroy(lbm_batch *b);
const char *lbm_batch_last_error(lbm_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
