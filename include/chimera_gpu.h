/*
 * chimera_gpu.h -- C-ABI of the B200 (sm_100a) drop-in for CHIMERA's per-step
 * hot path: one SSP-RK3 step of the 2-D ideal-MHD finite-volume solver.
 *
 * The reference has no C-ABI: the path is the body of the Fortran time loop
 * (src/main.f90:65-303) calling module subroutines on whole arrays.  Each entry
 * point below names the reference code it replaces.  Plain C types only: a
 * Fortran iso_c_binding interface, ctypes, or C/C++ can bind it directly.
 *
 * Arrays: real(8) (ld, ny) column-major with x fastest -- the Fortran layout of
 * Mass, Momx, Momy, Energy (cell centred, multiplied by the cell volume) and the
 * staggered face fields b_x (x face i+1/2) and b_y (y face j+1/2)
 * (src/mhd_init.f90:44-47).  ld >= nx is the leading dimension in elements.
 *
 * Errors: every call returns CHIMERA_OK (0) or a negative CHIMERA_ERR_*.
 * Nothing on this path prints, exits, traps or aborts.
 * Threading: a handle owns one CUDA stream and is not thread safe; distinct
 * handles are independent.  Calls are asynchronous on the handle's stream
 * except *_get_state, *_diag and chimera_advance, which synchronise it.
 */
#ifndef CHIMERA_GPU_H
#define CHIMERA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Switch values are the reference's code numbering (src/mhd_config.f90:27-43). */
#define CHIMERA_RIEMANN_RUSANOV 1
#define CHIMERA_RIEMANN_HLLE 2
#define CHIMERA_RIEMANN_HLLD 3
#define CHIMERA_LIMITER_VAN_LEER 1
#define CHIMERA_LIMITER_MC 2
#define CHIMERA_BC_PERIODIC 1
#define CHIMERA_BC_FIXED 2    /* behaves as outflow on this path (src/main.f90:349-354) */
#define CHIMERA_BC_OUTFLOW 3
#define CHIMERA_BC_INFLOW 4   /* behaves as outflow on this path */

#define CHIMERA_FP64 0        /* plain FP64, bit-compatible with the reference expressions */
#define CHIMERA_FP32_BULK 1   /* FP32 storage/arithmetic, FP64 pressure recovery, dt and sums */
#define CHIMERA_FP32_MIXED 2  /* FP64 storage; FP32 reconstruction, limiter, MOOD and Riemann
                                 arithmetic; FP64 pressure recovery, cell and face-B updates,
                                 floors, RK blends, dt and sums */

#define CHIMERA_HOST 0        /* pointer arguments are host memory */
#define CHIMERA_DEVICE 1      /* pointer arguments are device memory */

#define CHIMERA_OK 0
#define CHIMERA_ERR_BAD_ARG -1       /* invalid argument (dims, switches, null pointer, ld) */
#define CHIMERA_ERR_CUDA -2          /* a CUDA runtime call failed */
#define CHIMERA_ERR_NONFINITE -3     /* the device status word reports a non-finite state */
#define CHIMERA_ERR_TIMEOUT -4       /* a bounded device wait gave up */
#define CHIMERA_ERR_UNSUPPORTED -5   /* valid in the reference but not on this path */
#define CHIMERA_ERR_NO_DEVICE -6     /* no usable sm_100 device */
#define CHIMERA_ERR_NOMEM -7         /* device allocation failed */
#define CHIMERA_ERR_TOO_LARGE -8     /* size exceeds a fixed capacity */

/* Build-time switches of src/mhd_config.f90:16-62, passed through so the
 * Fortran program's own parameters are honoured. */
typedef struct chimera_cfg {
  int nx, ny;              /* N, N in the reference (nx == ny there) */
  double dx, dy;           /* dx = boxsize/N (src/main.f90:34); dy == dx in the reference */
  double gamma;
  double courant;          /* courant_fac (0.3) */
  double t_out;            /* tOut (0.01): dt is clipped to the next output time */
  double t_end;            /* tEnd: steps stop once t >= t_end */
  int bc_xlo, bc_xhi, bc_ylo, bc_yhi;   /* BC_xlo.. (src/mhd_config.f90:48-49) */
  int riemann;             /* riemann_solver */
  int limiter;             /* slope_limiter */
  int use_slope_limiting;  /* useSlopeLimiting */
  int mood;                /* fallback_2_MOOD */
  int precision;           /* CHIMERA_FP64, CHIMERA_FP32_BULK or CHIMERA_FP32_MIXED */
} chimera_cfg;

typedef struct chimera_diag_out {
  double t;                /* simulation time after the last step */
  double dt;               /* time step the next step will use (CFL + tOut clip) */
  int output_count;        /* outputCount of src/main.f90:62,291 */
  int active;              /* t < t_end */
  unsigned long long steps;
  double divb_max;         /* max |divB| over cells (compute_divB, src/mhd_field_ops.f90:60-117) */
  double divb_mean;        /* sum |divB| / (nx ny), the reference's printed monitor (src/main.f90:299) */
  double bmax;             /* max |B| of the cell-centred field */
  double divb_rel;         /* max|divB| * min(dx,dy) / max|B| */
  double mass;             /* sum of Mass (FP64) */
  double energy;           /* sum of Energy (FP64) */
  double cfl_speed;        /* max(c_f + |v|) */
  unsigned long long mood_resets;  /* faces with a MOOD reset (if counters on) */
  unsigned long long floor_hits;   /* cells with a conserved floor hit (if counters on) */
  unsigned status;         /* device status word (0 = clean) */
} chimera_diag_out;

typedef struct chimera_handle chimera_handle;

/* ---- single grid --------------------------------------------------------- */

/* Create a solver for one grid.  stream: a cudaStream_t, or NULL to create one.
 * Each side takes its own boundary flag, as src/mhd_bc.f90:45-100 does (a
 * periodic side may face a non-periodic one, in every precision form).
 * Replaces the allocations of src/mhd_init.f90:99-164 for the path's arrays. */
int chimera_create(const chimera_cfg* cfg, void* stream, chimera_handle** out);

/* Copy a conserved state in (host or device arrays); marks dt stale.  Host
 * arrays have been read completely when the call returns (it synchronises);
 * device arrays are read in order on the handle's stream.
 * Replaces the module globals Mass..b_y (src/mhd_init.f90:44-47). */
int chimera_set_state(chimera_handle* h, const double* Mass, const double* Momx,
                      const double* Momy, const double* Energy, const double* b_x,
                      const double* b_y, int ld, int where);

/* Copy the conserved state out (synchronises).  Returns CHIMERA_ERR_NONFINITE
 * if the device status word is set (the arrays are still copied). */
int chimera_get_state(chimera_handle* h, double* Mass, double* Momx, double* Momy,
                      double* Energy, double* b_x, double* b_y, int ld, int where);

/* One RK3 step on HOST arrays: in[6] (Mass, Momx, Momy, Energy, b_x, b_y,
 * pitch ld doubles) is copied in, advanced one step (CFL dt of the new state,
 * tOut clip, three stages) and copied out to out[6] (which may be in).  For a
 * single-grid FP64 handle the stages run over chunks of rows, and the
 * device-to-host copy of each chunk starts as soon as stage 3 has written it,
 * overlapping the later chunks' compute; pinned host memory is needed for that
 * overlap.  Synchronises.  Replaces, for a
 * caller that keeps its state in host arrays, one pass of the loop body of
 * src/main.f90:65-303 between the module arrays. */
int chimera_step_host(chimera_handle* h, const double* const* in, double* const* out, int ld);

/* Set t and outputCount (src/main.f90:61-62); marks dt stale. */
int chimera_set_time(chimera_handle* h, double t, int output_count);

/* Advance nsteps SSP-RK3 steps: the loop body of src/main.f90:65-303 (CFL dt,
 * tOut clip, three stages, t += dt, div B monitor, outputCount).  Steps stop
 * early, on the device, once t >= t_end. */
int chimera_step(chimera_handle* h, int nsteps);

/* Run until t >= t_end or max_steps steps (do while (t < tEnd),
 * src/main.f90:65); *steps_taken receives the count.  Synchronises. */
int chimera_advance(chimera_handle* h, int max_steps, int* steps_taken);

/* As chimera_advance, but every member also stops right after the step whose
 * t reaches its next output time (t >= outputCount*tOut or t >= tEnd, the
 * condition under which src/main.f90:279-292 writes a snapshot and advances
 * outputCount): the time loop and its stop test stay on the device (graph
 * replay, no host round trip per step), and the call returns with the state
 * of the snapshot.  The snapshot cadence of the reference's loop is one call
 * per output.  In a batch, members that stop early wait for the others.
 * *steps_taken receives the largest step count of a member.  Synchronises. */
int chimera_advance_output(chimera_handle* h, int max_steps, int* steps_taken);

/* One RK stage k (1..3) with a given dt on the handle's stage buffers
 * (src/main.f90:107-149, 155-208, 214-267): stage 1 reads U^n, writes U1;
 * stage 2 reads U1 and U^n, writes U2; stage 3 reads U2 and U^n, writes U^n.
 * For stage-level parity tests. */
int chimera_stage(chimera_handle* h, int k, double dt);

/* Read stage buffer b (0 = U^n, 1 = U1, 2 = U2), synchronising. */
int chimera_get_stage_buffer(chimera_handle* h, int b, double* Mass, double* Momx,
                             double* Momy, double* Energy, double* b_x, double* b_y,
                             int ld, int where);

/* Diagnostics of the last step or CFL evaluation (synchronises). */
int chimera_diag(chimera_handle* h, chimera_diag_out* out);

/* Count MOOD resets and floor hits on the device (off by default). */
int chimera_set_counters(chimera_handle* h, int on);

/* Time every kernel launch of the eager (non-graph) path with CUDA events on
 * the handle's stream (no counterpart in the reference, which has no timers). */
int chimera_set_profiling(chimera_handle* h, int on);

/* Accumulated device time in ms and launch counts of [CFL, stage 1, stage 2,
 * stage 3] since the last reset (synchronises). */
int chimera_get_profile(chimera_handle* h, double* ms, long long* launches, int reset);

/* The handle's stream (a cudaStream_t). */
void* chimera_stream(chimera_handle* h);

void chimera_destroy(chimera_handle* h);

/* ---- batched ensembles (one persistent launch per stage over all members) -- */

/* A batch of independent grids of uneven sizes.  All members share riemann,
 * limiter, use_slope_limiting, mood and precision; sizes, spacing, gamma and
 * boundary conditions are per member.  Replaces the sequential ensemble loop
 * of scripts/run_mhd_MC.py:62-73. */
int chimera_batch_create(int n_members, const chimera_cfg* cfgs, void* stream,
                         chimera_handle** out);
int chimera_batch_set_state(chimera_handle* h, int member, const double* Mass,
                            const double* Momx, const double* Momy, const double* Energy,
                            const double* b_x, const double* b_y, int ld, int where);
int chimera_batch_get_state(chimera_handle* h, int member, double* Mass, double* Momx,
                            double* Momy, double* Energy, double* b_x, double* b_y, int ld,
                            int where);
int chimera_batch_set_time(chimera_handle* h, int member, double t, int output_count);
int chimera_batch_diag(chimera_handle* h, int member, chimera_diag_out* out);
int chimera_batch_size(chimera_handle* h);

/* Capture nsteps steps into a CUDA graph once and replay it on every
 * chimera_step(h, nsteps) call with the same count (0 disables). */
int chimera_set_graph_steps(chimera_handle* h, int nsteps);

/* ---- tile-shape autotuner (no counterpart in the reference) --------------------
 * Each precision is compiled in several tile shapes / occupancy targets.  The
 * autotuner times reps dry RK3 steps of every variant on the handle's current
 * state (scratch buffers only; the state and time-loop counters are untouched)
 * and keeps the fastest; the choice is cached per problem shape for the process. */
int chimera_autotune(chimera_handle* h, int reps, int* chosen, double* best_ms_per_step);
int chimera_variant_count(chimera_handle* h);
int chimera_set_variant(chimera_handle* h, int variant);
int chimera_get_variant(chimera_handle* h, int* variant, int* tile_x, int* tile_y, int* threads);

/* ---- one grid split into y-slabs across ranks (no counterpart in the reference) --
 * The reference advances one grid in one process (src/main.f90:65-303).  A
 * slab handle holds its rows of the grid plus `rows` ghost rows on each side
 * that has a neighbour.  Once per step the caller (i) packs the interior rows
 * its neighbours need, (ii) moves them (NCCL send / recv, or a copy when the
 * slabs share a GPU), (iii) unpacks the received ghost rows, (iv) fetches the
 * slab's CFL dt into a device double (the previous step's stage 3 computed it
 * over the slab's own rows, which the exchange leaves unchanged), (v) takes
 * the minimum over the slabs (an all-reduce) and (vi) writes it back before
 * chimera_step(h, 1).  Seven
 * ghost rows make every interior cell of the step identical to the undivided
 * grid's: each RK3 stage reaches two rows, and the lowest ghost row is wrong
 * before the first stage (its cell-centred B averages a face below it that
 * the slab does not hold), so 1 + 3 x 2 rows at the bottom (6 at the top).
 * Single-member handles only; the per-step calls are asynchronous on the
 * handle's stream.
 *   - pack:   lo <- state rows [rows, 2 rows), hi <- rows [ny - 2 rows, ny - rows)
 *   - unpack: state rows [0, rows) <- lo, rows [ny - rows, ny) <- hi
 * lo / hi are device buffers of 6 * rows * nx elements (field-major, Mass..b_y),
 * 8-byte elements for CHIMERA_FP64 and CHIMERA_FP32_MIXED, 4-byte ones for
 * CHIMERA_FP32_BULK; a
 * null side is skipped.  Requires 2 * rows <= ny. */
int chimera_halo_pack(chimera_handle* h, int rows, void* lo, void* hi);
int chimera_halo_unpack(chimera_handle* h, int rows, const void* lo, const void* hi);
/* Declare the ghost rows (bottom, top) of a slab handle: the CFL dt and the
 * diagnostics (of the stage-3 epilogue, the CFL pass and chimera_diag) cover
 * only the slab's own rows, so that the minimum / maximum / sum over the
 * slabs is the grid's.  Synchronises. */
int chimera_slab_ghost_rows(chimera_handle* h, int ghost_lo, int ghost_hi);
/* Recompute the CFL dt of the current state (src/main.f90:69-83, with the
 * tOut clip; a CFL kernel launch) into d_dt[member] (device memory; null:
 * only the handle's own copy), with the diagnostics of chimera_diag. */
int chimera_refresh_dt(chimera_handle* h, double* d_dt);
/* The dt the next step will use into d_dt[member] (device memory): the one
 * the last stage 3 or CFL pass computed, or a CFL pass if the state changed
 * since (a ghost-row unpack within chimera_slab_ghost_rows' rows does not
 * count as a change). */
int chimera_get_dt_device(chimera_handle* h, double* d_dt);
/* Set every member's dt from d_dt[member] (device memory) for the next step. */
int chimera_set_dt_device(chimera_handle* h, const double* d_dt);

/* ---- discrete adjoint of one RK3 step (FP64, periodic or outflow sides) ----
 * No counterpart in the reference.  lambda_n = (dU_{n+1}/dU_n)^T lambda_{n+1}
 * for the step U_n -> U_{n+1} with a given (frozen) dt: the MOOD, floor and
 * thermal-check decisions are the forward's, and at a kink the derivative is
 * that of the branch the forward took.  Pointer arguments are arrays of six
 * device pointers (Mass, Momx, Momy, Energy, b_x, b_y), each a dense (nx, ny)
 * array.  Boundaries: every non-periodic kind acts as outflow, each side on
 * its own (a periodic side may face a non-periodic one).  All calls
 * synchronise the adjoint's stream. */
typedef struct chimera_adjoint chimera_adjoint;
int chimera_adjoint_create(const chimera_cfg* cfg, void* stream, chimera_adjoint** out);
int chimera_adjoint_step(chimera_adjoint* a, const double* const* U_n, double dt,
                         const double* const* lambda_next, double* const* lambda_n);
/* The same step forward with a given dt (bit-identical to chimera_step's FP64
 * stage kernels): recomputation from checkpoints and frozen-dt replays. */
int chimera_adjoint_forward_step(chimera_adjoint* a, const double* const* U_n, double dt,
                                 double* const* U_next);
void chimera_adjoint_destroy(chimera_adjoint* a);

/* ---- one step without device allocation ---------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc --
 * a host code whose device memory is all owned by its own allocator, a time
 * loop that must not pay cudaMalloc's implicit device synchronisation, or a
 * program that forbids allocation after initialisation -- this advances a
 * caller-owned FP64 state by one SSP-RK3 step (CFL dt with the tOut clip, the
 * three stages, t += dt, outputCount) exactly as chimera_step does, without
 * allocating anything: its stage buffers and reductions live in one fixed
 * file-scope device array (about 6.5 MB) that every GPU which loads the
 * library holds until the process exits.
 *   - Mass..b_y: device pointers to dense (nx, ny) arrays, x fastest, updated
 *     in place; cfg->precision must be CHIMERA_FP64.
 *   - nx*ny above CHIMERA_NOALLOC_MAX_CELLS returns CHIMERA_ERR_TOO_LARGE;
 *     cfg->t_end must be > 0 (CHIMERA_ERR_BAD_ARG otherwise).
 *   - *t and *output_count are read and advanced; *dt_next (optional) receives
 *     the dt the next step will take.  The call synchronises the stream, on
 *     its error paths too.
 *   - With *t >= cfg->t_end the run is over: the call launches nothing and
 *     returns CHIMERA_OK with the arrays, *t, *output_count and *dt_next
 *     untouched (as chimera_step leaves an inactive state).
 *   - stream (null = the current device's legacy stream) must belong to the
 *     current device, whose scratch the call uses; CHIMERA_ERR_BAD_ARG if not.
 *   - FP64 only, and each pair of opposite sides alike (a periodic side facing
 *     a non-periodic one: CHIMERA_ERR_UNSUPPORTED; chimera_create takes it).
 *   - The first call on a device looks up the scratch's device address; make
 *     that first call before any stream capture.
 *   - Every call shares the one scratch array of its device, which keeps the
 *     last call's contents (each call clears the parts that must start at
 *     zero).  Two calls whose GPU work overlapped would race on it, so calls
 *     from several host threads of one process are serialised per device
 *     inside the library (a call holds a lock until its stream has drained);
 *     calls from other processes use their own copy. */
#define CHIMERA_NOALLOC_MAX_CELLS 65536
int chimera_rk3_step_noalloc(const chimera_cfg* cfg, double* Mass, double* Momx, double* Momy,
                             double* Energy, double* b_x, double* b_y, double* t,
                             int* output_count, double* dt_next, void* stream);

/* ---- the reference's module routines, one kernel each ----------------------------
 * Same names, argument meaning and per-side boundary handling as the Fortran
 * routines; dense (nx, ny) device arrays (x fastest), cfg gives nx, ny, dx, dy,
 * gamma, the BC flags, riemann, limiter and mood; asynchronous on `stream`. */
int chimera_op_average_face_to_cell_B(const chimera_cfg* cfg, const double* b_x, const double* b_y,
                                      double* Bx, double* By, void* stream);   /* src/mhd_field_ops.f90:120-156 */
int chimera_op_get_primitive(const chimera_cfg* cfg, const double* Mass, const double* Momx,
                             const double* Momy, const double* Energy, const double* Bx,
                             const double* By, double* rho, double* vx, double* vy, double* P,
                             void* stream);                                   /* src/mhd_change_states.f90:61-113 */
int chimera_op_get_conserved(const chimera_cfg* cfg, const double* rho, const double* vx,
                             const double* vy, const double* P, const double* Bx, const double* By,
                             double* Mass, double* Momx, double* Momy, double* Energy,
                             void* stream);                                   /* src/mhd_change_states.f90:16-58 */
int chimera_op_apply_conserved_floors(const chimera_cfg* cfg, double* Mass, double* Momx, double* Momy,
                                      double* Energy, const double* Bx, const double* By,
                                      void* stream);                          /* src/mhd_change_states.f90:116-166 */
int chimera_op_fill_ghost_cells(const chimera_cfg* cfg, const double* f, double* f_pad,
                                void* stream);            /* src/mhd_bc.f90:36-170; f_pad is (nx+2, ny+2) */
int chimera_op_compute_gradients(const chimera_cfg* cfg, const double* f_pad, double* f_dx, double* f_dy,
                                 void* stream);                               /* src/mhd_derivatives.f90:15-47 */
int chimera_op_apply_slope_limiter(const chimera_cfg* cfg, const double* f_pad, double* f_dx,
                                   double* f_dy, void* stream);               /* src/mhd_derivatives.f90:50-127 */
int chimera_op_reconstruction(const chimera_cfg* cfg, const double* f, const double* f_dx,
                              const double* f_dy, double* f_XL, double* f_XR, double* f_YL,
                              double* f_YR, int rho_or_p, void* stream);      /* src/mhd_derivatives.f90:130-229 */
/* faces24[s*6+q]: slot s in (XL, XR, YL, YR), field q in (P, Bx, By, rho, vx, vy); cell6 likewise */
int chimera_op_thermal_pressure_check(const chimera_cfg* cfg, double* const* faces24,
                                      const double* const* cell6, void* stream); /* src/mhd_derivatives.f90:232-293 */
/* in12: rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R (normal first);
 * out5: mass, normal momentum, tangential momentum, energy, tangential B */
int chimera_op_compute_fluxes(const chimera_cfg* cfg, const double* const* in12, double* const* out5,
                              void* stream);                                  /* src/mhd_flux.f90:139-779 */
int chimera_op_update_conserved(const chimera_cfg* cfg, double* F, const double* flux_X,
                                const double* flux_Y, double dt, void* stream); /* src/mhd_flux.f90:20-76 */
/* scratch: one caller-owned (nx, ny) array */
int chimera_op_constrained_transport(const chimera_cfg* cfg, double* b_x, double* b_y,
                                     const double* flux_By_X, const double* flux_Bx_Y, double dt,
                                     double* scratch, void* stream);          /* src/mhd_flux.f90:79-136 */
int chimera_op_compute_curl_2d(const chimera_cfg* cfg, const double* Az, double* b_x, double* b_y,
                               void* stream);                                 /* src/mhd_field_ops.f90:15-57 */
int chimera_op_compute_divB(const chimera_cfg* cfg, const double* b_x, const double* b_y, double* divB,
                            void* stream);                                    /* src/mhd_field_ops.f90:60-117 */

/* ---- misc ------------------------------------------------------------------ */
const char* chimera_strerror(int code);
int chimera_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CHIMERA_GPU_H */
