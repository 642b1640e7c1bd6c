/*
 * aeromhd.h -- C ABI of libaeromhd.so, the B200 (sm_100a) implementation of
 * the AeroMHD-CUDA solver hot path: one SSP-RK3 step of 2-D ideal MHD
 * (van Leer / minmod MUSCL, HLLD fluxes in x and y, GLM + Powell source,
 * CFL dt), plus the batched-ensemble driver.
 *
 * Conventions
 *   - Every entry point returns int: AMHD_OK (0) or a negative AMHD_ERR_*
 *     (amhd_march_pack and amhd_march_items return a count, or a negative
 *     AMHD_ERR_*); amhd_last_error() gives a message for the calling thread.
 *   - All array pointers are DEVICE pointers owned by the caller unless the
 *     name says _host.  The library never allocates device memory on a step.
 *   - `stream` is a cudaStream_t passed as void*; calls are asynchronous on
 *     it, except those that return host scalars (they synchronise it).
 *   - A state array holds 10 planes (conserved slots rho, mx, my, mz, Bx, By,
 *     Bz, E, psi, rho*C; reference config.py:13-16).  Element (v, i, j) with
 *     i the x index and j the y index, ghosts included (i in [0, nx+4),
 *     j in [0, ny+4)), lives at  base[v*var_stride + i*pitch + j].
 *     The reference's contiguous U[10, nx+4, ny+4] (solver.py:83) is the case
 *     pitch = ny+4, var_stride = (nx+4)*(ny+4).
 *   - dtype AMHD_F64: double everywhere; AMHD_F32: float state and fluxes,
 *     double pressure recovery, dt reduction and diagnostics.
 *
 * Each declaration cites the reference routine it replaces (file:line of the
 * reference project).
 */
#ifndef AEROMHD_H
#define AEROMHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AMHD_OK 0
#define AMHD_ERR_ARG (-1)
#define AMHD_ERR_CUDA (-2)
#define AMHD_ERR_NONFINITE (-3)
#define AMHD_ERR_TIMEOUT (-4)
#define AMHD_ERR_UNSUPPORTED (-5)

#define AMHD_F64 0
#define AMHD_F32 1

#define AMHD_BC_PERIODIC 0
#define AMHD_BC_EXTRAPOLATION 1
#define AMHD_BC_CHARACTERISTIC 2

#define AMHD_LIMITER_VANLEER 0
#define AMHD_LIMITER_MINMOD 1

/* flags set in amhd_control.flags by the kernels */
#define AMHD_FLAG_NONFINITE 1   /* a non-finite value was written by a step */
#define AMHD_FLAG_DT_TINY 2     /* dt <= 1e-16 stopped the loop (solver.py:479) */
#define AMHD_FLAG_PAUSED 4      /* loop paused at a snapshot time (amhd_control.snap_t) */
#define AMHD_FLAG_TIMEOUT 8     /* a bounded device wait (TMA completion) expired; finalize
                                   stops the loop on this flag and on AMHD_FLAG_NONFINITE */

/* Grid and physics parameters of one instance (reference Config,
 * config.py:47-89, flattened; dx, dy precomputed as config.py:78-84 does). */
typedef struct amhd_grid {
    int32_t nx, ny;          /* interior cells                                  */
    int32_t pitch;           /* elements between x-rows, >= ny + 4              */
    int32_t dtype;           /* AMHD_F64 or AMHD_F32                            */
    int64_t var_stride;      /* elements between planes, >= (nx + 4) * pitch    */
    double dx, dy;
    double gamma, cfl, glm_alpha;
    int32_t bc_x, bc_y;      /* AMHD_BC_*; y knows periodic / extrapolation     */
    int32_t powell;          /* 1: add the Powell source (solver.py:304-306)    */
    int32_t limiter;         /* AMHD_LIMITER_*                                  */
} amhd_grid;

/* Per-instance time-stepping state kept in DEVICE memory, so that a loop of
 * steps (and a CUDA graph of it) needs no host round trip.  Fields mirror the
 * reference solver's attributes: t, dt, step (solver.py:84-86),
 * cfg.glm_ch (solver.py:215), _glm_ch_frozen (:87),
 * _cumulative_boundary_energy (:103).  Allocate sizeof(amhd_control) bytes of
 * device memory per instance and initialise it with amhd_control_init. */
typedef struct amhd_control {
    double t;            /* simulation time                                    */
    double t_end;        /* loop stops at t >= t_end                           */
    double dt;           /* dt of the next step = min(dt_cfl, t_end - t)       */
    double dt_cfl;       /* last CFL dt (solver.py:206-223)                    */
    double ch;           /* cfg.glm_ch set by the last dt computation          */
    double decay;        /* psi damping factor of the next step (:331-333)    */
    double e_bnd;        /* cumulative boundary energy flux x dt (:316-317)   */
    double last_dt;      /* dt of the last step taken                          */
    int64_t step;        /* steps taken                                        */
    int64_t max_steps;   /* loop stops at step >= max_steps                    */
    int32_t active;      /* 1 while the loop should continue                   */
    int32_t flags;       /* AMHD_FLAG_*                                        */
    uint64_t red[4];     /* dt reduction accumulators (bit patterns of         */
                         /* non-negative doubles): max cf^2, max(|vx|+|vy|),   */
                         /* max |vx|, max |vy|                                 */
    int32_t queue[2];    /* work queue of a persistent marching grid over this  */
                         /* single grid: {next item, warps finished}, zero     */
                         /* between launches (amhd_control_init zeroes it)     */
    double snap_t;       /* pause the loop after the step that brings t within */
                         /* 1.5 dt of snap_t (run(), solver.py:487-490);       */
                         /* +inf or NaN: never                                 */
    double scratch;      /* device scratch of amhd_boundary_energy_flux          */
    double e_bnd_next;   /* boundary energy flux x dt of the step the loop takes */
                         /* next; added to e_bnd once that step is taken, so    */
                         /* e_bnd counts the steps taken (solver.py:316-317)    */
    double reserved;
} amhd_control;

/* ---- library ---------------------------------------------------------- */
const char *amhd_version(void);
const char *amhd_last_error(void);
/* Configure every kernel of the library on the current device (shared
 * memory limits); idempotent.  Call once before capturing a CUDA graph. */
int amhd_init(void);
/* element counts of the padded layout the fused step kernels require:
 * pitch and rows per plane (multiples the kernels' tiles need). */
int amhd_padded_layout(int32_t nx, int32_t ny, int32_t dtype, int32_t *pitch, int32_t *rows);
size_t amhd_control_size(void);
/* Stage kernel and its work shape for single-grid calls.  tile_x 4, 8 or 16:
 * the tiled kernel, tile_x x 32 cells per CTA staged in shared memory;
 * tile_x from -1024 to -4: the warp-marching kernel, one warp per item of
 * -tile_x rows x 28 columns, walking the rows with the x-slopes and x-face
 * fluxes carried from row to row (no CTA barriers).  ctas_per_sm: 0 = one CTA
 * per tile (tiled) / per 4 items (marching), otherwise a persistent grid of
 * ctas_per_sm x SM-count CTAs.  Both kernels compute the same arithmetic
 * (identical float64 results).  0 restores the default: -24 for float32 grids, -16
 * for float64 grids.  Process-wide; chosen by the autotuner.  The
 * same nonzero tile_x values are accepted by amhd_stage_info and
 * amhd_ensemble_advance.  No counterpart in the reference. */
int amhd_set_tiling(int32_t tile_x, int32_t ctas_per_sm);
/* TMA staging (cp.async.bulk.tensor) per stage kernel, as a bit mask: bit 0
 * the tiled kernel's tile + halo (else 128-bit loads), bit 1 the marching
 * kernel's rows, one box of 32 columns x 10 planes per row for the warp
 * (else per-lane cp.async).  Results are identical either way.  Default 1.
 * Process-wide.  No counterpart in the reference. */
int amhd_set_tma(int32_t mode);
/* shared memory per CTA and resident CTAs per SM of the stage kernel of this geometry */
int amhd_stage_info(int32_t dtype, int32_t tile_x, int32_t *smem_bytes, int32_t *ctas_per_sm, int32_t *sm_count);

/* ---- physics.py ------------------------------------------------------- */
/* cons_to_prim, physics.py:284-301 (all cells, ghosts included) */
int amhd_cons_to_prim(const amhd_grid *g, const void *U, void *W, void *stream);
/* prim_to_cons, physics.py:304-320 */
int amhd_prim_to_cons(const amhd_grid *g, const void *W, void *U, void *stream);
/* muscl_x / muscl_y, physics.py:323-350.  axis 0: WL, WR are contiguous
 * [10][nx+1][ny+4]; axis 1: [10][nx+4][ny+1]. */
int amhd_muscl(const amhd_grid *g, int32_t axis, const void *W, void *WL, void *WR, void *stream);
/* hlld_flux_x / hlld_flux_y, physics.py:353-379 (kernel physics.py:43-276).
 * axis 0: x faces; axis 1: y faces (components rotated as physics.py:376-379).
 * WL, WR, F: contiguous [10][n_faces]; smax: [n_faces] per-face signal speed
 * (may be NULL). */
int amhd_hlld_flux(int32_t axis, int32_t dtype, const void *WL, const void *WR, void *F, void *smax, int64_t n_faces,
                   double gamma, double ch, void *stream);

/* ---- solver.py: MHDSolver -------------------------------------------- */
/* apply_bc, solver.py:158-197 (in place) */
int amhd_apply_bc(const amhd_grid *g, void *U, void *stream);
/* enforce_scalar_bounds, solver.py:199-204 (in place, all cells) */
int amhd_enforce_scalar_bounds(const amhd_grid *g, void *U, void *stream);
/* compute_dt, solver.py:206-223, from primitive W (all cells, ghosts
 * included).  Writes dt_cfl and ch (the new cfg.glm_ch) into *ctl and leaves
 * the loop fields alone.  If dt_host / ch_host are not NULL the call
 * synchronises and stores them. */
int amhd_compute_dt(const amhd_grid *g, const void *W, amhd_control *ctl, double *dt_host, double *ch_host,
                    void *stream);
/* the same from conserved U (cons_to_prim fused in) */
int amhd_compute_dt_cons(const amhd_grid *g, const void *U, amhd_control *ctl, double *dt_host, double *ch_host,
                         void *stream);
/* _compute_boundary_energy_flux, solver.py:225-240 (0 for periodic x).
 * ctl is used as device scratch (its scratch field receives the flux, nothing
 * else changes); synchronises. */
int amhd_boundary_energy_flux(const amhd_grid *g, const void *U, amhd_control *ctl, double *out_host, void *stream);
/* _compute_powell_source, solver.py:242-266: S from primitive W (same layout
 * as W); zero on the outermost ring, as the reference. */
int amhd_powell_source(const amhd_grid *g, const void *W, void *S, void *stream);
/* compute_rhs, solver.py:268-308: fills U's ghosts in place, then R (same
 * layout as U; zero outside the interior). */
int amhd_compute_rhs(const amhd_grid *g, void *U, void *R, double ch, void *stream);
/* step_ssprk3, solver.py:310-333, with the step's dt, frozen ch and psi
 * damping factor given by the host.  U is advanced in place; U1, U2 are
 * scratch states of the same layout.  Needs the padded layout
 * (amhd_padded_layout).  If ctl is not NULL: ctl->e_bnd accumulates the
 * boundary energy flux x dt (solver.py:316-317) and ctl->flags records a
 * non-finite result. */
int amhd_step_ssprk3(const amhd_grid *g, void *U, void *U1, void *U2, double dt, double ch, double decay,
                     amhd_control *ctl, void *stream);
/* one RK stage (1, 2 or 3) of step_ssprk3 (solver.py:319-329) on states that
 * already hold their ghost cells: stage 1: Uout = U0 + dt L(U0); stage 2:
 * Uout = 3/4 U0 + 1/4 (Uin + dt L(Uin)); stage 3: 1/3 U0 + 2/3 (Uin + dt
 * L(Uin)), psi damped; each followed by the scalar clamp and the boundary
 * conditions.  Padded layout. */
int amhd_rk_stage(const amhd_grid *g, int32_t stage, const void *Uin, const void *U0, void *Uout, double dt,
                  double ch, double decay, void *stream);
/* Initialise *ctl (device) for a run from state U: t, t_end, step,
 * max_steps; computes dt/ch from U exactly as run() does before its first
 * step (solver.py:476-479).  Asynchronous. */
int amhd_control_init(const amhd_grid *g, const void *U, amhd_control *ctl, double t, double t_end, int64_t step,
                      int64_t max_steps, void *stream);
/* Set the snapshot time at which the device loop pauses next (snap_t, +inf
 * for none) for n controls, and resume those paused at the previous one.
 * Asynchronous; no counterpart in the reference (its loop is on the host). */
int amhd_control_resume(amhd_control *ctl, int32_t n, double snap_t, void *stream);
/* The run loop (solver.py:475-482 / main.py:66-73) for n_steps iterations on
 * the device: each iteration is one SSP-RK3 step with dt, ch and the psi
 * damping taken from *ctl, the CFL reduction of the new state fused into the
 * last stage, then t += dt, step += 1, boundary-energy bookkeeping and the
 * next dt.  Iterations after the stop condition (t >= t_end, step >=
 * max_steps, dt <= 1e-16) do nothing.  No host synchronisation; capturable
 * in a CUDA graph.  With the marching kernel every stage reads the ghost
 * cells of its input from the interior cells they copy, and U's ghost cells
 * are filled once, after the last iteration (every stream-ordered reader of
 * U sees a complete state); the launches of the loop are programmatic
 * dependents of one another (each waits for the one before on the device). */
int amhd_advance(const amhd_grid *g, void *U, void *U1, void *U2, amhd_control *ctl, int32_t n_steps,
                 void *stream);
/* amhd_advance for a float32 state accumulated with compensation: U_lo (same
 * padded layout and dtype as U) holds the low part of the base state, U_hi +
 * U_lo.  Stage 3 adds the step's increment to hi + lo and splits the sum into
 * the stored float32 U and its exact rounding error (TwoSum), the new U_lo,
 * so that the rounding of the stored state does not accumulate from step to
 * step; stages 1 and 2 read U (the increment they feed is exact either way).
 * Zero U_lo whenever U is set or changed outside this loop.  Marching kernel
 * only.  No counterpart in the reference (float64 there). */
int amhd_advance_compensated(const amhd_grid *g, void *U, void *U_lo, void *U1, void *U2, amhd_control *ctl,
                             int32_t n_steps, void *stream);
/* The run loop taken apart, for drivers that act between its pieces (a grid
 * split over GPUs by x rows exchanges ghost rows after every stage and
 * max-reduces the CFL maxima ctl->red[4] across GPUs before the dt):
 *   amhd_control_init_split -- as amhd_control_init, but stops after
 *     accumulating the state's CFL maxima into ctl->red (no dt yet) and
 *     filling U's ghost cells;
 *   amhd_advance_stage -- stage 1 (U -> U1), 2 (U1 -> U2, base U) or 3
 *     (U2 -> U, base U, CFL maxima of the new state into ctl->red) with dt,
 *     ch and the psi damping from ctl, ghost cells of the output filled;
 *   amhd_advance_finish -- advance = 1: t += dt, step += 1 (as at the end of
 *     an amhd_advance iteration), then in both cases dt / ch / damping / the
 *     stop flags from ctl->red, which is cleared, and the boundary energy of
 *     the block's physical x sides into ctl->e_bnd (non-periodic x;
 *     solver.py:225-240, :316-317).  cut_x marks the sides that are cuts
 *     between blocks and carry no boundary flux: bit 0 the block's first
 *     row, bit 1 its last row (0 for a whole grid).  The whole grid's
 *     boundary energy is the sum of the blocks' e_bnd.
 * amhd_advance(n) == n x (stage 1, 2, 3, finish(1)).  Asynchronous.  No
 * counterpart in the reference. */
int amhd_control_init_split(const amhd_grid *g, void *U, amhd_control *ctl, double t, double t_end, int64_t step,
                            int64_t max_steps, void *stream);
int amhd_advance_stage(const amhd_grid *g, int32_t stage, void *U, void *U1, void *U2, amhd_control *ctl,
                       void *stream);
int amhd_advance_finish(const amhd_grid *g, void *U, amhd_control *ctl, int32_t advance, int32_t cut_x,
                        void *stream);
/* amhd_advance with a CUDA event recorded after every launch: ms_out[0..3]
 * receive the summed device time of the stage-1, stage-2, stage-3 and
 * finalize launches, ms_out[4] the whole interval.  Synchronises.  For
 * profiling; no counterpart in the reference. */
int amhd_advance_profile(const amhd_grid *g, void *U, void *U1, void *U2, amhd_control *ctl, int32_t n_steps,
                         double *ms_out, void *stream);
/* One iteration of the run loop (solver.py:476-482) on a HOST state: copies
 * U_host (pinned or pageable, contiguous [10][nx+4][ny+4] of the grid's
 * dtype) to the device, computes dt from it (CFL, capped at t_end - t),
 * advances one SSP-RK3 step, and copies the new state back into U_host.
 * out_host (may be NULL) receives {t + dt, dt, glm_ch, boundary energy
 * flux x dt}.  dev_U/dev_U1/dev_U2 and ctl are caller device buffers (padded
 * layout).  Returns AMHD_ERR_NONFINITE if the new state holds a NaN/Inf,
 * AMHD_ERR_TIMEOUT if a bounded device wait gave up (tiles not updated).
 * Synchronises. */
int amhd_step_host(const amhd_grid *g, void *U_host, void *dev_U, void *dev_U1, void *dev_U2, amhd_control *ctl,
                   double t, double t_end, double *out_host, void *stream);
/* n_steps iterations of amhd_step_host in one call, the same bits: every step
 * copies its input from U_host and its result back into U_host, plane by
 * plane on two copy streams of the library (one per direction), so that a
 * plane of step k+1 travels to the device as soon as step k's result for that
 * plane is back, while the other planes of step k are still travelling the
 * other way (with pinned U_host both PCIe directions are busy at once).
 * out_host receives {t, dt of the last step, glm_ch, boundary energy flux x dt
 * summed over the n steps}.  Synchronises; calls on one device from several
 * threads run one after the other. */
int amhd_step_host_n(const amhd_grid *g, void *U_host, void *dev_U, void *dev_U1, void *dev_U2, amhd_control *ctl,
                     double t, double t_end, int32_t n_steps, double *out_host, void *stream);
/* compute_diagnostics, solver.py:335-444 (the conserved-quantity part):
 * out_dev receives (float64) [0] mass = sum(rho) dx dy, [1] energy = sum(E)
 * dx dy (solver.py:430), [2] max|divB|, [3] sqrt(mean divB^2) (:419-428),
 * [4] integral mixing width (:353-356), [5] peak stagnation pressure (:415-417),
 * [6] global enstrophy mean(rho w^2) (:399-402).
 * rows_dev: 7*nx doubles, left holding the per-row sums of clip(C), rho, E,
 * divB^2, rho w^2 and the per-row maxima of |divB| and the stagnation
 * pressure (in that order).  Asynchronous. */
int amhd_diagnostics(const amhd_grid *g, const void *U, double x0, double *out_dev, double *rows_dev, void *stream);
/* The colour-field part of compute_diagnostics (solver.py:358-383) that needs a
 * second pass over the field, after amhd_diagnostics filled rows_dev:
 * cp2_dev[nx] = per-row sum over y of (clip(C) - Cbar)^2 (C_prime_sq x ny,
 * :360); pos_dev[ny] = per-column interface position, the |dC/dx|-weighted
 * mean of x within 10 rows of the first maximum of |dC/dx| (numpy.gradient
 * along x; numpy's pairwise sums), NaN where the reference leaves NaN
 * (:369-378).  The threshold mixing width, mixedness, perturbation modes and
 * local enstrophy follow on the host from these nx + ny values and rows_dev.
 * Asynchronous. */
int amhd_diagnostics_colour(const amhd_grid *g, const void *U, double x0, const double *rows_dev, double *cp2_dev,
                            double *pos_dev, void *stream);

/* The same diagnostics for callers that cannot allocate device memory: a
 * host framework that owns every device allocation and hands its plugins
 * only their inputs and outputs, or a loop with a strict time budget that
 * must not risk an allocation synchronising the device.  No counterpart in
 * the reference.  The row scratch is a fixed device array compiled into this
 * library (room for nx <= AMHD_NOALLOC_MAX_NX interior rows; larger grids
 * get AMHD_ERR_ARG); it is resident on every GPU that loads the library until
 * the process exits.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and must be made with that device current and
 * before any stream capture that contains later calls; the address is kept
 * per device ordinal for the life of the process, so after a
 * cudaDeviceReset of that device this entry point must not be called again.
 * All calls share the one array: calls whose kernels may overlap on the GPU
 * (different streams without ordering) race on it.  out_dev: 7 doubles as
 * for amhd_diagnostics.  Asynchronous. */
#define AMHD_NOALLOC_MAX_NX 16384
int amhd_diagnostics_noalloc(const amhd_grid *g, const void *U, double x0, double *out_dev, void *stream);

/* ---- batched ensemble -------------------------------------------------- */
/* One entry per instance of the packed ensemble; offsets are element offsets
 * of each instance's state in the three packed state buffers. */
typedef struct amhd_instance {
    amhd_grid grid;
    int64_t offset;          /* element offset of plane 0, row 0, col 0          */
    int32_t first_tile;      /* index of the instance's first tile in the list   */
    int32_t tiles_x, tiles_y;/* tiles of this instance (tile_x rows x 32 cols)   */
    int32_t cut_x;           /* x sides that are cuts, not boundaries (bit 0 the
                                first row, bit 1 the last): excluded from the
                                boundary energy; 0 for a whole grid             */
    int32_t pack;            /* marching kernel without TMA staging: row chunks
                                of the last column strip that share one work
                                item, amhd_march_pack(grid.ny); 0 or 1: none
                                (any other value is taken as none)              */
    int32_t reserved;        /* zero                                            */
} amhd_instance;

/* Work items of the warp-marching kernel (tile_x < 0: -tile_x rows x 28
 * columns per warp).  An instance's last column strip holds ny mod 28
 * columns; when they and their 2-column halo on each side fit 8 lanes (up to
 * 4 columns) or 16 lanes (up to 12), amhd_march_pack returns 4 or 2 and that
 * many row chunks of the strip share one warp, one segment of lanes each;
 * otherwise 1.  amhd_march_items: the instance's work items with that pack
 * value -- (chunks x strips) for pack 1, else (strips - 1) x chunks plus
 * ceil(full-height chunks / pack) plus 1 for a short last chunk.  The packed
 * items are numbered first, then the full-width strips' items chunk-major.
 * Both return a count; amhd_march_items returns AMHD_ERR_ARG for a
 * non-positive size or a pack other than 0, 1 or amhd_march_pack(ny).  A
 * work list with more items than this count has the extra ones skipped. */
int amhd_march_pack(int32_t ny);
int amhd_march_items(int32_t nx, int32_t ny, int32_t rows, int32_t pack);
/* Switch the packing of single-grid calls (1, the default) off (0) or on;
 * ensembles set amhd_instance.pack themselves.  Results do not depend on it. */
int amhd_set_march_pack(int32_t on);

/* Advance every active instance of a packed ensemble by n_steps run-loop
 * steps: one persistent launch per RK stage over the (instance, tile) work
 * list, per-instance dt/ch/t in ctl[n_inst].  U, U1, U2 are the packed
 * buffers; inst and ctl are device arrays.  Tiles are numbered per instance
 * from inst[k].first_tile (tile_x rows x 32 columns, y fastest);
 * tile_inst[tile] is the instance of each tile; tile_order (may be NULL for
 * the identity) is the order in which work positions are taken.  ctas is the
 * grid size (0: resident CTAs per SM x SM count).  Without a queue, CTA /
 * warp b takes positions b, b + ctas (warps), ...  queue_dev (marching
 * kernel; may be NULL): two device int32 that are zero before the first call
 * and between launches -- each warp of a persistent grid then takes the next
 * free position as it finishes an item, and the last warp of a launch resets
 * the pair; one pair per stream of calls.  tmaps_dev: device copy of
 * amhd_ensemble_tensormaps for this tile_x (NULL: 128-bit loads instead of
 * TMA).  Capturable in a CUDA graph.
 * No counterpart in the reference (one grid per solver there). */
int amhd_ensemble_advance(const amhd_instance *inst_dev, int32_t n_inst, const int32_t *tile_inst_dev,
                          const int32_t *tile_order_dev, int32_t n_tiles, int32_t dtype, int32_t tile_x, void *U,
                          void *U1, void *U2, amhd_control *ctl_dev, int32_t n_steps, int32_t ctas,
                          const void *tmaps_dev, int32_t *queue_dev, void *stream);
/* Continue every instance from its current t and step to a new t_end: dt,
 * ch and the loop flags are recomputed from the current states (as
 * amhd_ensemble_init does, but keeping t, step, flags and the boundary
 * energy).  Asynchronous.  No counterpart in the reference. */
int amhd_ensemble_continue(const amhd_instance *inst_host, const amhd_instance *inst_dev, int32_t n_inst,
                           int32_t dtype, void *U, amhd_control *ctl_dev, double t_end, void *stream);
/* Fill maps_host (3 * n_inst CUtensorMap of 128 bytes: U, U1, U2 per
 * instance) for amhd_ensemble_advance; copy it to device memory (64-byte
 * aligned) before use.  No counterpart in the reference. */
int amhd_ensemble_tensormaps(const amhd_instance *inst_host, int32_t n_inst, int32_t dtype, int32_t tile_x,
                             const void *U, const void *U1, const void *U2, void *maps_host);
/* amhd_control_init for every instance of the ensemble (inst_host: a host
 * copy of the instance table).  Asynchronous. */
int amhd_ensemble_init(const amhd_instance *inst_host, const amhd_instance *inst_dev, int32_t n_inst,
                       int32_t dtype, void *U, amhd_control *ctl_dev, double t_end, int64_t max_steps,
                       void *stream);

/* ---- learned coarse-grid corrector ------------------------------------- */
/* Kernels of the convolutional corrector's training and inference; none has a
 * counterpart in the reference.  Activations are float32 [C][B*H*W]
 * (channel-major), GEMM operands bfloat16, accumulation float32. */
const char *amhd_nn_last_error(void);
/* C[M][N] = alpha op(A) op(B) + beta C on the BF16 tensor cores (FP32
 * accumulate; mma.sync m16n8k16 or tcgen05, amhd_nn_set_gemm_path).  op(A) = A ([M][K], lda) or, transA, A^T (A
 * stored [K][M]); op(B) = B ([K][N]) or, transB, B^T (B stored [N][K]).
 * splits > 1 divides K over CTAs and accumulates atomically. */
/* The same contract on the 5th-generation tensor cores (tcgen05.mma, FP32
 * accumulator in tensor memory).  Operands whose base is 16-byte aligned and
 * whose ld is a multiple of 8 are loaded by TMA (128-byte swizzle), 128 x 64
 * output tiles: without split-K by a persistent kernel (one CTA per SM, an
 * 8-stage load ring, two TMEM accumulators so that a tile's epilogue overlaps
 * the next tile's loads and MMAs; amhd_nn_set_gemm_persistent(0) takes the
 * one-tile-per-CTA kernel instead), with splits > 1 (which may be raised to
 * fill the GPU) one tile per CTA and a 3-stage ring; others are staged by the
 * CTA's threads (128 x 128 tiles).
 * amhd_nn_gemm_status returns (and clears) 1 if a load or MMA completion wait
 * gave up since the last call, else 0; amhd_nn_gemm_tc_paths counts the
 * launches of either path since the library was loaded. */
int amhd_nn_gemm_tc(int32_t transA, int32_t transB, int32_t M, int32_t N, int32_t K, const void *A, int32_t lda,
                    const void *B, int32_t ldb, float *C, int32_t ldc, float alpha, float beta, int32_t splits,
                    void *stream);
int amhd_nn_gemm_status(int32_t *flag);
int amhd_nn_gemm_tc_paths(int64_t *tma, int64_t *staged);
/* Which kernel amhd_nn_gemm runs (process-wide): 0 (default) the tcgen05
 * TMA pipeline on the shapes where it is faster on B200 -- N >= 64 or
 * K >= 4096 -- when the operands qualify, mma.sync otherwise; 1 always
 * mma.sync; 2 always amhd_nn_gemm_tc. */
int amhd_nn_set_gemm_path(int32_t mode);
/* 1 (default): unsplit TMA GEMMs run the persistent kernel; 0: one tile per CTA
 * (process-wide; for measurement) */
int amhd_nn_set_gemm_persistent(int32_t on);

/* Self-test of the bounded device waits every kernel of this library uses on
 * an mbarrier (TMA staging, tensor-core completion; no counterpart in the
 * reference).  One thread waits on a shared-memory mbarrier after arriving on
 * it itself (arrive != 0: the wait must succeed) or with nothing arriving (the
 * wait must give up after limit_ns, 0 < limit_ns <= 2e9, and say so):
 * *timed_out = 1 when it gave up, *waited_us = how long it waited.  The
 * context stays usable either way.  Synchronous. */
int amhd_selftest_wait(int32_t arrive, int64_t limit_ns, int32_t *timed_out, int32_t *waited_us);
int amhd_nn_gemm(int32_t transA, int32_t transB, int32_t M, int32_t N, int32_t K, const void *A, int32_t lda,
                 const void *B, int32_t ldb, float *C, int32_t ldc, float alpha, float beta, int32_t splits,
                 void *stream);
/* 3x3 zero-padded convolution columns: col[c*9+tap][b,h,w] (BF16) of X[c][b][h][w] */
int amhd_nn_im2col3(const float *X, int32_t C, int32_t B, int32_t H, int32_t W, void *col, void *stream);
/* adjoint of im2col3: dX[c][b][h][w] = sum over taps of dcol (gather, fixed order) */
int amhd_nn_col2im3(const float *dcol, int32_t C, int32_t B, int32_t H, int32_t W, float *dX, void *stream);
/* the 3x3 weights w[co][ci*9+tap] (BF16) for the input gradient:
 * wt[ci][co*9+t] = w[co][ci*9+8-t], columns cout*9 .. ldo-1 zero; then
 * dX = wt x im2col3(dY) (the adjoint of a zero-padded 3x3 convolution) */
int amhd_nn_flip3(const void *w, int32_t cout, int32_t cin, int32_t ldo, void *wt, void *stream);
/* rows x cols BF16 values into rows x ldo, columns cols .. ldo-1 zero (a GEMM
 * operand whose row pitch is a multiple of 8 values, as the TMA path needs) */
int amhd_nn_pad_cols(const void *w, int32_t rows, int32_t cols, int32_t ldo, void *out, void *stream);
int amhd_nn_cast_bf16(const float *x, void *y, int64_t n, void *stream);
/* Y[c][n] = act(Y[c][n] + bias[c]), act = ReLU if relu else identity */
int amhd_nn_bias_act(float *Y, const float *bias, int32_t C, int64_t N, int32_t relu, void *stream);
/* dY *= (Y > 0) */
int amhd_nn_relu_bwd(float *dY, const float *Y, int64_t n, void *stream);
/* db[c] = sum_n dY[c][n] */
int amhd_nn_bias_grad(const float *dY, int32_t C, int64_t N, float *db, void *stream);
/* 2x2 average pooling of [CB][H][W] (backward: its adjoint into [CB][H][W]) */
int amhd_nn_pool2(const float *X, int32_t CB, int32_t H, int32_t W, float *Y, int32_t backward, void *stream);
/* nearest 2x upsampling of [CB][h][w] (backward: its adjoint into [CB][h][w]) */
int amhd_nn_up2(const float *X, int32_t CB, int32_t h, int32_t w, float *Y, int32_t backward, void *stream);
/* y += a x */
int amhd_nn_axpy(float *y, const float *x, float a, int64_t n, void *stream);
/* grad = 2 (pred - target) / n (if grad), *loss += mean squared error (if loss) */
int amhd_nn_mse(const float *pred, const float *target, int64_t n, float *grad, float *loss, void *stream);
/* Adam with bias correction (step t >= 1) and decoupled-into-gradient weight
 * decay; refreshes the BF16 copy w_bf16 (may be NULL) */
int amhd_nn_adam(float *w, const float *g, float *m, float *v, void *w_bf16, int64_t n, float lr, float beta1,
                 float beta2, float eps, int32_t t, float weight_decay, void *stream);
/* One parameter tensor of amhd_nn_adam_multi (device pointers). */
typedef struct amhd_nn_tensor {
    float *w;             /* float32 master weights                          */
    const float *g;       /* gradient                                        */
    float *m, *v;         /* Adam moments                                    */
    void *w_bf16;         /* bfloat16 copy refreshed after the step, or NULL */
    int64_t n;            /* elements                                        */
    float weight_decay;
    int32_t pad_;
} amhd_nn_tensor;
/* The Adam step of amhd_nn_adam on n_tensors tensors in one launch, with the
 * step's scalars read from device memory -- hyper_dev = {lr, beta1, beta2,
 * eps, 1/(1 - beta1^t), 1/(1 - beta2^t)} -- so that the launch can be part of
 * a captured CUDA graph replayed every step.  tensors_dev: the records in
 * device memory; max_n: the largest n among them.  Same arithmetic as
 * amhd_nn_adam.  No counterpart in the reference. */
int amhd_nn_adam_multi(const amhd_nn_tensor *tensors_dev, int32_t n_tensors, int64_t max_n, const float *hyper_dev,
                       void *stream);
/* factor x factor block average of a fine state's interior (float64 sums)
 * into sample b of out[10][B][nx/f][ny/f] (plane stride out_vs) */
int amhd_nn_restrict(const amhd_grid *fine, const void *Uf, int32_t factor, float *out, int64_t out_vs, int32_t b,
                     int32_t B, void *stream);
/* network input: x[v][b][i][j] = (U_interior - mean[v]) * istd[v] */
int amhd_nn_pack(const amhd_grid *g, const void *U, const float *mean, const float *istd, float *x, int64_t x_vs,
                 int32_t b, void *stream);
/* corrector output applied: U_interior[v] += scale[v] * y[v][b][i][j]
 * (ghost cells are left to amhd_apply_bc) */
int amhd_nn_apply(const amhd_grid *g, void *U, const float *scale, const float *y, int64_t y_vs, int32_t b,
                  void *stream);
/* the same, per cell and kept admissible: U_cell += alpha * scale[v] * y[v]
 * only if the corrected cell is finite and keeps >= min_ratio of its density
 * and of its pressure (float64); rejected cells keep their state and are
 * counted into *rejected_dev (may be NULL).  scalar_mode: 0 the correction as
 * is; 1 the passive scalar's correction scaled by 4 C (1 - C) of the cell;
 * 2 no scalar correction; 3 every variable's correction scaled by 4 C (1 - C)
 * (corrections confined to the mixing layer).  Ghost cells are left to
 * amhd_apply_bc. */
int amhd_nn_apply_guarded(const amhd_grid *g, void *U, const float *scale, const float *y, int64_t y_vs, int32_t b,
                          float alpha, float min_ratio, int32_t scalar_mode, int32_t *rejected_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AEROMHD_H */
