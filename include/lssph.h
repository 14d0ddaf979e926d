/*
 * lssph.h -- C ABI of the B200 LS-SPH engine.
 *
 * The engine replaces the time-step loop of the LS-SPH-Benchmarks Fortran solver
 * (source/main.f90:119-166): RK2/RK4 stages, LS-SPH type-A right-hand sides, cell-list
 * neighbour search, multi-layer ghost walls and the particle shifting technique all run
 * as sm_100a kernels on device-resident state.  Host code (the Fortran iso_c_binding
 * shim, the C++ driver, the Python ctypes wrapper) keeps the reference's config.h
 * parameter surface and its results/ file layout.
 *
 * Conventions
 *   - Every function returns an int status: 0 = OK, negative = LSSPH_E_*.  A message
 *     for the last failure is available from lssph_last_error() / lssph_handle_error().
 *   - Particle indices are 0-based (the Fortran shim adds 1).  Particle order is the
 *     reference order: interior (fluid) particles 0..num_int-1 in lattice scan order,
 *     then ghost wall particles num_int..num_total-1 (setup_closed_box_mod.f90:120-136).
 *   - All arrays are caller-owned host buffers, SoA, float64 unless noted.
 *   - A handle owns its device state and one CUDA stream.  A handle is not thread-safe;
 *     distinct handles are independent.
 */
#ifndef LSSPH_H
#define LSSPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSSPH_ABI_VERSION 2

/* ---- status codes ---------------------------------------------------------------- */
#define LSSPH_OK                 0
#define LSSPH_E_BAD_PARAM      (-1)  /* check_param_mod.f90 would `error stop` */
#define LSSPH_E_CUDA           (-2)  /* a CUDA runtime call failed */
#define LSSPH_E_CELL_OVERFLOW  (-3)  /* a cell holds more than its slot capacity */
#define LSSPH_E_OUT_OF_DOMAIN  (-4)  /* a particle left the cell grid */
#define LSSPH_E_NONFINITE      (-5)  /* a NaN/Inf appeared in the state */
#define LSSPH_E_SINGULAR       (-6)  /* a zero pivot in a moment-matrix solve */
#define LSSPH_E_IO             (-7)  /* file I/O failed */
#define LSSPH_E_CAPACITY       (-8)  /* an output buffer is too small / batch full */
#define LSSPH_E_TIMEOUT        (-9)  /* a bounded device wait gave up */
#define LSSPH_E_UNSUPPORTED    (-10) /* option combination not implemented */

/* ---- engine options (no counterpart in the reference) ----------------------------- */
#define LSSPH_PRECISION_FP64   0     /* plain FP64 path (reference arithmetic) */
#define LSSPH_PRECISION_MIXED  1     /* FP32 pair sums, FP64 solve */
#define LSSPH_PRECISION_MIXED_COMPENSATED 2  /* as MIXED, with Kahan-compensated FP32 pair sums
                                                and one refinement step of the FP64 solve */

/*
 * lssph_params -- mirrors Param_type (source/core/global_types.f90:22-73) plus the
 * compile-time macros of config.h that Param_type does not store (boundary codes, RK
 * order).  User fields come from config.h; derived fields are filled by
 * lssph_init_param() exactly as init_param_mod.f90:92-199 derives them.
 */
typedef struct lssph_params {
    /* ---- user-defined (config.h) ---- */
    int32_t target_problem;                                     /* TARGET_PROBLEM 1..4 */
    int32_t u_bc_top, u_bc_bottom, u_bc_left, u_bc_right;       /* U_BOUNDARY_*  1..3  */
    int32_t tem_bc_top, tem_bc_bottom, tem_bc_left, tem_bc_right; /* TEM_BOUNDARY_* 1..2 */
    double  u_top;
    double  tem_top, tem_bottom, tem_left, tem_right;
    char    save_name[256];
    char    read_name[256];
    int32_t omp_threads;
    int32_t rk;                                                 /* RK 2 or 4 */
    double  len_x, len_y;
    int32_t num_x, num_y;
    int32_t start_step, end_step, write_step;
    int32_t pad0_;
    double  threshold, coe_CFL, coe_dif, zeta_RSST, xi_VIM;
    double  rho_ref, vis_ref, K_ref, k_th_ref, cp_ref, alpha_ref;
    double  gravity, pos_pert;
    int32_t tg_a, tg_b;
    double  coe_h, PST_c, coe_delta_sph;
    int32_t kernel_type, sph_model, wall_model;
    /* ---- derived (init_param_mod.f90:92-199) ---- */
    int32_t total_step, num_WL;
    int32_t pad1_;
    double  dx, SP_mass, h, h_eff, W_ave, WL_thick;
    double  delta_tem, tem_ave;
    double  sound_speed, kinematic_vis, thermal_dif;
    double  Re, Ra, Pr;
    double  dt, dt_CFL, dt_vis, dt_th, dt_CFL_relax, dt_vis_relax;
    /* ---- engine options (no reference counterpart) ---- */
    int32_t  precision;   /* LSSPH_PRECISION_* */
    int32_t  lanes;       /* lanes per particle in neighbour loops: 1 = reference
                             summation order (bit-exact vs the oracle); 2, 4, 8 (mixed
                             precision 2, 4); 0 = auto: a q = 5 LS solve times 2 and 4 at
                             its first solo launch or batch join and keeps the faster
                             unless 4 is within 5 %, any other solve runs 4 */
    uint64_t seed;        /* POS_PERT jitter seed (the reference seeds from the clock,
                             impose_initial_conditions_mod.f90:43-51) */
    int32_t  periodic;    /* 1: periodic square [0, LEN_X)^2 without walls (problems 1, 2);
                             problem 1 then decays u = sin(2 pi x) sin(2 pi y) without the
                             source term.  0: the reference's closed box */
    int32_t  pad2_;
} lssph_params;

typedef struct lssph_handle lssph_handle;
typedef struct lssph_batch lssph_batch;

/* ---- library ------------------------------------------------------------------------ */
int         lssph_abi_version(void);
/* sizeof(lssph_params) as compiled into the library (FFI layout check). */
size_t      lssph_params_sizeof(void);
/* Last error message of the calling thread (for calls that have no handle). */
const char* lssph_last_error(void);
const char* lssph_status_string(int status);

/* ---- parameters (host only) ---------------------------------------------------------- */
/* Reference defaults: the values of the shipped config.h. */
int lssph_params_default(lssph_params* out);
/* Parse a config.h (`#define NAME value` lines), then lssph_init_param + lssph_check_param.
   Replaces init_param (init_param_mod.f90:24) + check_param (check_param_mod.f90:22). */
int lssph_params_from_config(const char* config_h_path, lssph_params* out);
/* Fill the derived fields of *p from its user fields (init_param_mod.f90:92-199). */
int lssph_init_param(lssph_params* p);
/* Validate user fields (check_param_mod.f90:22-284).  LSSPH_E_BAD_PARAM + message. */
int lssph_check_param(const lssph_params* p);

/* ---- particle setup (host only) ------------------------------------------------------ */
/* Particle counts of the closed box: num_total = (num_x+2 num_WL)(num_y+2 num_WL). */
int lssph_setup_counts(const lssph_params* p, int32_t* num_total, int32_t* num_int);
/* setup_closed_box (setup_closed_box_mod.f90:23-237) + impose_* initial conditions
   (impose_initial_conditions_mod.f90).  tem may be NULL unless target_problem == 4. */
int lssph_setup_particles(const lssph_params* p, int32_t num_total, int32_t* ptype,
                          double* x, double* y, double* u, double* v, double* rho,
                          double* pre, double* tem);

/* ---- simulation handle ---------------------------------------------------------------- */
/* Copy host state to the device and build the cell list (init_cell + update_cell,
   init_cell_mod.f90:23, update_cell_mod.f90:21) and the virtual markers
   (init_virtual_markers_mod.f90:23).  Ghost values are taken from the input; call
   lssph_ghost() for a fresh start (write_param_mod.f90:144 does it there).  tem may be
   NULL unless target_problem == 4.  Indices follow the reference order. */
int lssph_create(const lssph_params* p, int32_t num_total, int32_t num_int,
                 const int32_t* ptype, const double* x, const double* y, const double* u,
                 const double* v, const double* rho, const double* pre, const double* tem,
                 lssph_handle** out);
void        lssph_destroy(lssph_handle* h);
const char* lssph_handle_error(const lssph_handle* h);
int lssph_get_params(const lssph_handle* h, lssph_params* out);
int lssph_counts(const lssph_handle* h, int32_t* num_total, int32_t* num_int,
                 int32_t* num_ext, int32_t* num_cells);

/* One reference operator each (same names as the Fortran subroutines). */
int lssph_calculate_rhs(lssph_handle* h);            /* calculate_RHS_mod.f90:29 */
int lssph_update_cell(lssph_handle* h);              /* update_cell_mod.f90:21   */
int lssph_ghost(lssph_handle* h);                    /* ghost_mod.f90:43         */
int lssph_rk2(lssph_handle* h);                      /* RK2_mod.f90:30           */
int lssph_rk4(lssph_handle* h);                      /* RK4_mod.f90:30           */
int lssph_pst(lssph_handle* h);                      /* PST_mod.f90:28           */
int lssph_check_steady_state(lssph_handle* h, int32_t* is_steady); /* check_steady_state_mod.f90:23 */

/* The body of the time loop (main.f90:119-149) for nsteps steps, device-resident and
   graph-replayed: RK2/RK4, PST (problems 2-4), steady check (problem 1).  Stops early at
   a steady state; *steady_step_out (may be NULL) receives the 1-based step count within
   this call at which it was reached, or 0. */
int lssph_step(lssph_handle* h, int32_t nsteps, int32_t* steady_step_out);

/* Device memory (no counterpart in the reference), for admission control: the bytes a
   handle holds, and the bytes lssph_create would allocate for a fresh start with *p
   (host-only; both count requested bytes, before the allocator's rounding). */
int lssph_device_bytes(const lssph_handle* h, int64_t* bytes);
/* Free and total memory of the current device (cudaMemGetInfo). */
int lssph_mem_info(int64_t* free_bytes, int64_t* total_bytes);
int lssph_estimate_device_bytes(const lssph_params* p, int64_t* bytes);

/* Step budget (no counterpart in the reference): after nsteps more time steps the handle
   stops advancing, as it does at a steady state; later lssph_step / lssph_batch_step calls
   leave it where it stopped.  The stop takes effect exactly at the step boundary, also
   inside a batch.  nsteps = 0 removes the budget (and resumes a handle stopped by one). */
int lssph_set_step_budget(lssph_handle* h, int32_t nsteps);
/* Time steps completed since creation; *stopped = 0 running, 1 steady state, 2 step budget
   used up. */
int lssph_get_progress(lssph_handle* h, int32_t* steps_done, int32_t* stopped);

/* Host <-> device state (caller buffers of length num_total; tem may be NULL).  Both return
   after the transfer is complete, so the buffers may be reused at once.  Page-locked,
   mapped buffers (cudaHostAlloc, cudaMallocHost, cudaHostRegister) are read and written by
   one kernel over the bus; other host memory goes through one copy per field. */
int lssph_upload(lssph_handle* h, const double* x, const double* y, const double* u,
                 const double* v, const double* rho, const double* pre, const double* tem);
int lssph_download(lssph_handle* h, int32_t* ptype, double* x, double* y, double* u,
                   double* v, double* rho, double* pre, double* tem);
/* Upload the state from host arrays (as lssph_upload, positions included), run nsteps time
   steps (as lssph_step) and write the new state back into the same arrays (as
   lssph_download), queued back to back with one synchronisation: the call of a host that
   keeps the particle state in its own arrays between steps, as the reference's driver keeps
   SP%x..SP%tem (main.f90:119-166).  x..pre (and tem for problem 4) have num_total entries;
   page-locked mapped buffers are read and written in place by one kernel each way.  No
   reference counterpart as one call (it fuses the loop body with the copies). */
int lssph_advance_host(lssph_handle* h, int32_t nsteps, double* x, double* y, double* u,
                       double* v, double* rho, double* pre, double* tem, int32_t* steady_step);
/* RHS arrays of the last calculate_RHS (length num_int; rhs_tem may be NULL). */
int lssph_download_rhs(lssph_handle* h, double* rhs_u, double* rhs_v, double* rhs_rho,
                       double* rhs_tem);
/* Virtual markers (length num_ext): VM.dat content (write_param_mod.f90:147-159). */
int lssph_download_vm(lssph_handle* h, int32_t* ptype, double* x, double* y, double* u,
                      double* v, double* pre, double* tem);

/* In-radius neighbour sets (r^2 <= h_eff^2 among the 3x3 cells) as sorted CSR, for parity
   checks.  which = 0: interior particles over all particles (LSSPH_A_mod.f90:102-125);
   which = 1: virtual markers over fluid particles (interpolate_LSSPH_B_mod.f90:158-180).
   offsets has n+1 entries; *nnz_out receives the total. */
int lssph_neighbors_csr(lssph_handle* h, int32_t which, int32_t* offsets, int32_t* idx,
                        int64_t cap, int64_t* nnz_out);

/* results/ layout read by analysis/common/read_utils.py. */
int lssph_write_data(lssph_handle* h, const char* results_root, int32_t step);   /* write_data_mod.f90:22 */
int lssph_write_param(lssph_handle* h, const char* results_root, const char* config_h_path); /* write_param_mod.f90:27 */
/* parameters.csv alone (write_param_mod.f90:58-128), host only. */
int lssph_write_parameters(const lssph_params* p, int32_t num_total, int32_t num_int,
                           const char* path);
/* write_data without stopping the time loop (no counterpart in the reference, which writes
   synchronously): captures the current state with device-to-device copies on the handle's
   stream and returns; a copy to pinned host memory and the file write run in the
   background while later lssph_step calls proceed.  The file is the one lssph_write_data
   writes for the same state, byte for byte.  A write error is returned by the next call or
   by lssph_snapshot_wait, which waits for every pending snapshot of the handle;
   lssph_destroy waits as well. */
int lssph_write_data_async(lssph_handle* h, const char* results_root, int32_t step);
int lssph_snapshot_wait(lssph_handle* h);
/* Restart reader (restart_mod.f90:22-53): fills caller buffers of length num_total. */
int lssph_read_data(const char* path, int32_t num_total, int32_t with_tem, int32_t* ptype,
                    double* x, double* y, double* u, double* v, double* rho, double* pre,
                    double* tem);

/* Kernel configuration the handle runs (no counterpart in the reference): lanes per
   particle, and the register budget of the stage/PST kernels: 0 loose, 1 tight (512 threads
   per SM), 2 (640 threads per SM, q = 5 LS only), and for the pair kernel of the split shape
   also 3 (768) and 4 (1024), with the measured time of the fused kernels at the loose and
   tight budgets (SPH_MODEL 4-6: of the thread- and warp-per-particle mappings, one of which
   the measurement picks).  The measurement runs at the handle's first launch: whole time steps on
   the solve's own state, which is copied aside first and put back after each option (the
   RHS pass alone when the device has no room for the copy).  The lane count (lanes = 0),
   the shape and the budget are picked by it; the budget and shape never change a result. */
int lssph_get_tuning(const lssph_handle* h, int32_t* lanes, int32_t* tight, double* rhs_us_loose,
                     double* rhs_us_tight);
/* Shape of the q = 5 LS stage and PST kernels, FP64 or mixed precision (no counterpart in
   the reference): 1 split (a pair kernel over the cell tiles, FP64 or FP32, then an FP64
   solve-and-update kernel with one thread per particle), 0 fused (one kernel), as the
   handle's first-launch measurement picked it (LSSPH_KERNEL_SHAPE=fused|split fixes it).
   Solves at 1 or 8 lanes and the classical models run fused.  For the higher-order models
   (SPH_MODEL 4-6) the value is the mapping the measurement picked: 2 thread per particle
   over a cell tile, 3 warp per particle (LSSPH_HI_KERNEL=thread|warp fixes it).  Every
   shape and mapping computes identical results. */
int lssph_get_kernel_shape(const lssph_handle* h, int32_t* split);

/* Time-step schedule (no counterpart in the reference): cell tiles, the tiles whose halo
   holds no ghost particle, and whether lssph_step runs each ghost launch beside the next
   stage's interior tiles (1) or alone (0; LSSPH_OVERLAP=0 forces it).  Never changes a
   result. */
int lssph_get_schedule(const lssph_handle* h, int32_t* tiles, int32_t* interior_tiles, int32_t* overlapped);

/* Device time of the kernels launched by the last lssph_step call, in milliseconds
   (CUDA events on the handle's stream), and the number of kernel launches it made. */
int lssph_last_step_stats(const lssph_handle* h, double* device_ms, int64_t* kernel_launches);

/* Kernel kinds of a time step, for lssph_step_profiled. */
#define LSSPH_KIND_STAGE     0   /* RHS + RK stage update + cell scatter */
#define LSSPH_KIND_CELLSORT  1   /* cell list finish (update_cell) */
#define LSSPH_KIND_GHOST     2   /* virtual-marker interpolation + extrapolation */
#define LSSPH_KIND_PST       3   /* particle shifting */
#define LSSPH_KIND_OTHER     4   /* epilogue / reductions */
#define LSSPH_KIND_COUNT     5
/* The same launch sequence as lssph_step, issued without graph capture and with a
   CUDA event pair around every kernel: ms_by_kind[k] receives the summed device time of
   kind k, launches_by_kind[k] its launch count (arrays of LSSPH_KIND_COUNT). */
int lssph_step_profiled(lssph_handle* h, int32_t nsteps, double* ms_by_kind,
                        int64_t* launches_by_kind);

/* ---- batched time loop (no counterpart in the reference) ------------------------------ */
/* A batch advances many independent solves (handles) together: each kernel of a time
   step is launched once for all members of the same kind (same RHS width, RK order, wall
   model and lane count), members of different kinds run concurrently, and the whole step
   is one CUDA graph.  Every member computes exactly what lssph_step computes for it
   alone (bit-identical results), each stops at its own steady state or error, and
   members may join or leave between calls.  A handle belongs to at most one batch; it
   stays usable on its own between batch calls (its own lssph_step, uploads, downloads,
   files), and destroying it removes it from its batch.  Members are numbered in the
   order they were added; removal shifts later members down by one. */
int  lssph_batch_create(lssph_batch** out);
void lssph_batch_destroy(lssph_batch* b);
const char* lssph_batch_error(const lssph_batch* b);
int  lssph_batch_add(lssph_batch* b, lssph_handle* h);      /* LSSPH_E_BAD_PARAM if h is in a batch */
int  lssph_batch_remove(lssph_batch* b, lssph_handle* h);
int  lssph_batch_size(const lssph_batch* b);
/* nsteps time steps of every member.  status[i] (may be NULL) receives member i's status
   (LSSPH_OK or the code lssph_step would return), steady[i] (may be NULL) the 1-based step
   within this call at which member i reached a steady state, or 0, and steps_taken[i]
   (may be NULL) the steps member i actually advanced (fewer than nsteps once it stopped:
   steady state, step budget or error).  Returns LSSPH_OK, or the first member error, or
   LSSPH_E_CUDA for a failure of the batch itself. */
int  lssph_batch_step(lssph_batch* b, int32_t nsteps, int32_t* status, int32_t* steady,
                      int32_t* steps_taken);
/* lssph_batch_step in two halves, so that the host can prepare new solves while the GPU
   steps the batch: lssph_batch_launch enqueues the nsteps steps and returns; the batch
   and its members must not be used (no add/remove, no solo calls) until lssph_batch_wait
   has returned the same outputs as lssph_batch_step.  lssph_batch_step = launch + wait. */
int  lssph_batch_launch(lssph_batch* b, int32_t nsteps);
int  lssph_batch_wait(lssph_batch* b, int32_t* status, int32_t* steady, int32_t* steps_taken);
/* Device time and kernel launches of the last lssph_batch_step (all members). */
int  lssph_batch_last_step_stats(const lssph_batch* b, double* device_ms, int64_t* kernel_launches);

/* ---- post-processing interpolation (analysis/common/lssph_b.py:21-143) ---------------- */
/* LS-SPH type-B interpolation of one particle field at arbitrary points, the reference's
   analysis step `lssph_b.main(param, target_x, target_y, x_j, y_j, val_j, rho_j)`: for each
   point the value and the derivatives d/dx, d/dy from every particle within h_eff
   (normal equations with weights W_ij m / rho_j, basis size q = 3 / 6 / 10 / 15 / 21 from
   SPH_MODEL and TARGET_PROBLEM as in lssph_b.py:45-55).  out receives 3 doubles per point
   (value, d/dx, d/dy); a point with fewer than q particles in range, or a singular system,
   gets NaN, as in the reference.  Uses p->h, h_eff, kernel_type, sph_model,
   target_problem and SP_mass.  Host arrays in and out; the work runs on the GPU. */
int lssph_lsb_interpolate(const lssph_params* p, int32_t n, const double* x, const double* y,
                          const double* val, const double* rho, int32_t n_targets,
                          const double* tx, const double* ty, double* out);
/* The same on a solve's current device state (all num_total particles, ghosts included,
   as the analysis scripts read them from a .dat file).  Points are in the physical frame
   of the analysis scripts: particle positions minus WL_thick, so [0, LEN_X] x [0, LEN_Y]
   is the fluid box. */
#define LSSPH_FIELD_U   0
#define LSSPH_FIELD_V   1
#define LSSPH_FIELD_RHO 2
#define LSSPH_FIELD_PRE 3
#define LSSPH_FIELD_TEM 4
int lssph_interpolate(lssph_handle* h, int32_t field, int32_t n_targets, const double* tx,
                      const double* ty, double* out);

/* ---- allocation-free RHS (no counterpart in the reference) ---------------------------- */
/* One calculate_RHS pass (LS-SPH type A, problems 2-4, FP64, closed box) over a particle
   state that already lives in caller-owned device memory, writing the RHS arrays to
   caller-owned device memory, for callers that cannot allocate GPU memory at the point of
   the call (their memory is already committed to their own pool, or the call sits in a
   loop where a driver allocation is not acceptable).  It calls no cudaMalloc/cudaFree: its
   working set is one statically sized device array that every GPU loading this library
   reserves until the process exits.  Limits: num_total <= LSSPH_NOALLOC_MAX_PARTICLES,
   cell grid <= LSSPH_NOALLOC_MAX_CELLS cells, at most LSSPH_NOALLOC_CELL_CAP particles per
   cell; larger inputs return LSSPH_E_CAPACITY before any GPU work.  p->lanes picks the
   lanes per particle of the neighbour sums as for a handle: 1 (the reference summation
   order), 2 or 4 (0 means 4); other values, a periodic domain, problem 1 and mixed
   precision return LSSPH_E_UNSUPPORTED.  Every call looks up the array's device address on
   the current device.  The call runs on `stream` (NULL = default stream), waits for that
   stream, and returns the cell-overflow / out-of-domain errors its kernels recorded.  All
   calls share the one array and it keeps the last call's contents (each call clears what
   must start at zero): calls that overlap on the GPU (other threads or streams) race and
   give wrong results.  Inputs x..pre (and tem for problem 4) have num_total entries in the
   reference particle order; rhs_* have num_int entries (rhs_tem only for problem 4). */
#define LSSPH_NOALLOC_MAX_PARTICLES 262144
#define LSSPH_NOALLOC_MAX_CELLS     32768
#define LSSPH_NOALLOC_CELL_CAP      32
int lssph_rhs_noalloc(const lssph_params* p, int32_t num_total, int32_t num_int,
                      const double* x, const double* y, const double* u, const double* v,
                      const double* rho, const double* pre, const double* tem,
                      double* rhs_u, double* rhs_v, double* rhs_rho, double* rhs_tem,
                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LSSPH_H */
