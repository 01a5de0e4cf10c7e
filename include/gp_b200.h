/*
 * gp_b200.h -- C ABI of the B200 grand-potential explicit step.
 *
 * Drop-in replacement for the explicit-Euler loop of MicroSim's
 * Grand_potential_Finite_difference_2D solver (serial twin, 2D, isothermal,
 * Function_F = 1 quadratic free energies).  Plain C types only: handles,
 * pointers, sizes.  Every function returns 0 or a negative GP_E* code.
 *
 * The reference exposes its path as process-global state plus function-pointer
 * "plugins" (functions/global_vars.h:384-415, bound in
 * solverloop/initialize_functions_solverloop.h:4-58) and three step entry
 * points called from main (microsim_gp.c:103-106):
 *     solverloop_phasefield(start, end)      solverloop/solverloop.h:21
 *     apply_boundary_conditions(0)           solverloop/boundary_serial.h:176
 *     solverloop_concentration(start, end)   solverloop/solverloop.h:35
 * Here the same step is one call on an opaque context; the plugin choices
 * (Function_W, Function_anisotropy, BINARY/TERNARY/DILUTE) are fields of
 * gp_model.  Paths below are relative to Grand_potential_Finite_difference_2D_serial/.
 *
 * Field layout at this boundary: interior cells only, structure of arrays,
 * double precision, plane-major: phi[a][x][y] with y fastest (the reference's
 * index y + x*rows_y with the three ghost layers removed), then
 * mu[k][x][y].  Ghost layers are never stored: the Neumann and periodic copies
 * of the reference are applied as index maps when a kernel reads past an edge.
 */
#ifndef GP_B200_H_
#define GP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GP_MAX_PHASES 6 /* NUMPHASES supported by the kernels               */
#define GP_MAX_K1 3     /* NUMCOMPONENTS-1 supported by the kernels         */
#define GP_NAME_LEN 52  /* Phases/Components names (reference: 51 chars)    */

/* error codes */
#define GP_OK 0
#define GP_E_ARG -1         /* bad argument / NULL pointer                          */
#define GP_E_IO -2          /* file could not be opened / read / written            */
#define GP_E_PARSE -3       /* Input.in / Filling.in content not understood        */
#define GP_E_UNSUPPORTED -4 /* input asks for a feature outside this path          */
#define GP_E_CUDA -5        /* CUDA runtime error                                  */
#define GP_E_NONFINITE -6   /* NaN/Inf found in the fields (stability watchdog)    */
#define GP_E_NOMEM -7       /* host or device allocation failed                    */
#define GP_E_TIMEOUT -8     /* a bounded device wait gave up                        */
#define GP_E_SIZE -9        /* request exceeds a documented size limit              */

/* mu-update solver, calculate_divergence_concentration.h:238-270 */
#define GP_MU_BINARY 0  /* BINARY = 1: 1/x                         */
#define GP_MU_TERNARY 1 /* TERNARY = 1: closed-form 2x2 inverse    */
#define GP_MU_DILUTE 2  /* DILUTE = 1: diagonal                    */
#define GP_MU_LU 3      /* none set: the reference's LU inverse    */

/* precision of a device context */
#define GP_FP64 0 /* plain form: FP64 storage and arithmetic, bit-faithful to the reference */
#define GP_FP32 1 /* chosen form: FP32 storage/update, FP64 reductions                       */

/* boundary types, functions/utility_functions.h:471-653 */
#define GP_BC_NEUMANN 1
#define GP_BC_PERIODIC 3

/*
 * Model constants of one simulation instance, all derived on the host with
 * the reference's own operation order (functions/functionF_01.h:169-230
 * init_propertymatrices, functions/matrix.h:50 matinvnew,
 * functions/utility_functions.h:700 populate_rotation_matrix) so that the
 * device step reproduces the reference's doubles.
 */
typedef struct gp_model {
  int32_t N;  /* NUMPHASES (last phase = liquid)      */
  int32_t K1; /* NUMCOMPONENTS - 1                     */
  int64_t mesh_x, mesh_y;
  double dx, dy, dt;
  double epsilon, tau; /* interface width; FunctionTau fallback */
  double T, Teq;
  int32_t obstacle;   /* 1: Function_W=1 obstacle, 0: Function_W=2 well */
  int32_t anisotropy; /* Function_anisotropy (4-fold cubic when 1)      */
  int32_t mu_solver;  /* GP_MU_*                                        */
  int32_t bc_phi[4];  /* boundary[0..3] for phi: x-lo, x-hi, y-hi, y-lo */
  int32_t bc_mu[4];   /* same for mu                                    */
  int32_t pad0;
  double Gamma[GP_MAX_PHASES][GP_MAX_PHASES];
  double Gamma_abc[GP_MAX_PHASES][GP_MAX_PHASES][GP_MAX_PHASES];
  double tau_ab[GP_MAX_PHASES][GP_MAX_PHASES];
  double dab[GP_MAX_PHASES][GP_MAX_PHASES];
  double R[GP_MAX_PHASES][GP_MAX_PHASES][2][2];    /* Rotation_matrix, 2x2 block     */
  double Rinv[GP_MAX_PHASES][GP_MAX_PHASES][2][2]; /* Inv_Rotation_matrix, 2x2 block */
  double cmu[GP_MAX_PHASES][GP_MAX_K1][GP_MAX_K1];  /* (d mu/dc)^-1                  */
  double A[GP_MAX_PHASES][GP_MAX_K1][GP_MAX_K1];
  double Beff[GP_MAX_PHASES][GP_MAX_K1]; /* Beq + dBbdT*(T - Teq) (c_mu, Mu at T)     */
  double Bfill[GP_MAX_PHASES][GP_MAX_K1]; /* Beq + dBbdT*(Teq - Teq) (filling)        */
  double B[GP_MAX_PHASES][GP_MAX_K1];    /* B(T) of free_energy                        */
  double C[GP_MAX_PHASES];               /* C(T) of free_energy                        */
  double Diff[GP_MAX_PHASES][GP_MAX_K1][GP_MAX_K1];
  /* constants folded on the host exactly as the reference evaluates them */
  double inv_eps;     /* 1.0/epsilon                                */
  double w_obstacle;  /* 16.0/(M_PI*M_PI)                           */
  double jat_obst;    /* -0.25*M_PI*epsilon                         */
  double jat_well;    /* -1.0*epsilon                               */
  double s_well;      /* 0.5/sqrt(2.0)                              */
  /* mu of the liquid rows a moving-frame shift appends: Mu(cfill of the liquid)
   * at Filling_temperature (functions/shift.h:24-37) */
  double mu_shift[GP_MAX_K1];
  /* Non-isothermal frozen gradient (ISOTHERMAL = 0: Tempgrady; microsim_gp.c:77-82, 108-113,
   * functions/Temperature_gradient.h:4-29): after every step the temperature of ghost-padded row gy
   * is T = temp_bottom + gy * GRADIENT, GRADIENT = DeltaT * dy / Distance, temp_bottom = base_temp -
   * BASE_POS * GRADIENT, BASE_POS = gradient_OFFSET / dy + (velocity / dy) * (t * dt).  The cell's T
   * enters c(mu, T) and mu(c, T) through Beq + dBbdT (T - Teq), and B(T), C(T) of the free energies
   * (functions/functionF_01.h:62-104, with the constants below). */
  int32_t nonisothermal; /* 1: ISOTHERMAL = 0 (T above is then only the filling's) */
  int32_t bc_T[4];       /* boundary copy of T (x-lo, x-hi, y-hi, y-lo): 1 Neumann, 3 periodic, 0 none (ghosts keep the linear T) */
  int32_t pad1;
  double tg_base, tg_deltaT, tg_distance, tg_offset, tg_velocity; /* Tempgrady = {base_temp, DeltaT, Distance, gradient_OFFSET, velocity} */
  double Beq[GP_MAX_PHASES][GP_MAX_K1];   /* B(Teq)                                         */
  double dBbdT[GP_MAX_PHASES][GP_MAX_K1]; /* dB/dT                                          */
  double ceq_s[GP_MAX_PHASES][GP_MAX_K1]; /* ceq[a][a][k]                                   */
  double ceq_l[GP_MAX_PHASES][GP_MAX_K1]; /* ceq[a][N-1][k]                                 */
  double dC[GP_MAX_PHASES][GP_MAX_K1];    /* DELTA_C[a][k]                                  */
  double dT_s[GP_MAX_PHASES], dT_l[GP_MAX_PHASES]; /* DELTA_T[a][a], DELTA_T[a][N-1]        */
} gp_model;

/* Parsed Input.in (+ its BOUNDARY lines) and Filling.in. */
typedef struct gp_input gp_input;

/* Running statistics, microsim_gp.c:139-148 (interior cells; FP64). */
typedef struct gp_stats {
  double phi_max[GP_MAX_PHASES], phi_min[GP_MAX_PHASES], rel_change_phi[GP_MAX_PHASES];
  double mu_max[GP_MAX_K1], mu_min[GP_MAX_K1], rel_change_mu[GP_MAX_K1];
  double solute[GP_MAX_K1]; /* sum over cells of sum_a c_a(mu, T) h_a(phi) (file_writer.h:203-235 integrand; T the
                               cell's current one under a frozen gradient) */
  double phase_fraction[GP_MAX_PHASES]; /* sum over cells of phi_a                                      */
  int64_t nonfinite;  /* number of non-finite phi/mu values found                                         */
  /* Energies of the current state, FP64 sums over the interior cells times dx*dy.  The reference
   * has no global energy output; these are the functional whose variational derivatives its phase-field
   * step uses (solverloop/calculate_divergence_phasefield.h:24-26), with cell-centred gradients
   * (the gradphi_c of solverloop/calculate_gradients.h:92-131) and ghost cells by the boundary map:
   *   gradient   eps * sum_{a<b} Gamma_ab a_c(R_ab q_ab)^2 |q_ab|^2,  q_ab = phi_a grad phi_b - phi_b grad phi_a
   *              (functions/function_A_00.h:4-23, function_A_01.h, anisotropy_01.h:30-48; a_c = 1 isotropic)
   *   potential  (1/eps) * [16/pi^2 sum_{a<b} Gamma_ab |phi_a phi_b|       (obstacle, functionW_01.h:6-39)
   *                         or 9 sum_{a<b} Gamma_ab phi_a^2 phi_b^2       (well, functionW_02.h:4-33)
   *                         + sum_{a<b<c} Gamma_abc |phi_a phi_b phi_c|]
   *   chemical   sum_a h_a(phi) f_a(c_a(mu))        (functionF_01.h:5-18, functionH.h:24-37, c_mu :30-40)
   *   grand_potential = gradient + potential + sum_a h_a(phi) (f_a(c_a) - mu . c_a)   (the psi of functionF_01.h:41-57)
   * The free energy is gradient + potential + chemical. */
  double energy_gradient, energy_potential, energy_chemical, grand_potential;
} gp_stats;

/* ---------------- host side: files (reference L3/L4) ---------------- */

/* Parse Input.in with the reference's line grammar and key order rules
 * (functions/reading_input_parameters.h:1-308, read_boundary_conditions.h:4-57).
 * filling_in may be NULL (no FILL* lines). */
int gp_input_read(const char *input_in, const char *filling_in, gp_input **out);
void gp_input_free(gp_input *in);
/* Simple scalar queries on a parsed input (NTIMESTEPS, SAVET, ...). Returns
 * GP_E_ARG for an unknown key. */
int gp_input_get_long(const gp_input *in, const char *key, int64_t *value);
int gp_input_get_double(const gp_input *in, const char *key, double *value);
/* Phase (which = 0) or component (which = 1) name, verbatim (leading blanks kept). */
int gp_input_name(const gp_input *in, int which, int index, char *buf, size_t len);

/* Derive the model constants (initialize_variables.h:4-28, init_propertymatrices). */
int gp_model_from_input(const gp_input *in, gp_model *out);

/* Initial fields from the FILL* lines (functions/fill_domain.h:4-151,
 * functions/filling.h:6-270): phi[N][mx][my], mu[K1][mx][my], interior only. */
int gp_fill(const gp_input *in, const gp_model *m, double *phi, double *mu);

/* Write DATA/<out>_<t>.vtk (solverloop/file_writer.h:23-255), BINARY or ASCII
 * as Input.in's WRITEFORMAT says; Composition_* fields when Writecomposition. */
int gp_write_vtk(const gp_input *in, const gp_model *m, const char *path, const double *phi, const double *mu);
/* The same after time step tstep: for a non-isothermal model the Temperature field (and the
 * Composition fields) use the frozen gradient's temperature after that step. */
int gp_write_vtk_t(const gp_input *in, const gp_model *m, const char *path, const double *phi, const double *mu,
                   int64_t tstep);
/* Read fields back (solverloop/file_writer.h:256-386, restart). */
int gp_read_vtk(const gp_input *in, const gp_model *m, const char *path, double *phi, double *mu);

/* ---------------- device side: the step (reference L2 + L1) ---------------- */

typedef struct gp_ctx gp_ctx;

/* Allocate device state for one instance on the current CUDA device.
 * precision: GP_FP64 (plain) or GP_FP32 (chosen form). */
int gp_create(const gp_model *m, int precision, gp_ctx **out);
int gp_destroy(gp_ctx *ctx);
/* Host <-> device copies of the interior fields (double on the host side). */
int gp_upload(gp_ctx *ctx, const double *phi, const double *mu);
int gp_download(gp_ctx *ctx, double *phi, double *mu);
/* nsteps explicit steps: phase-field half step, ghost fill, concentration
 * half step, ghost fill -- microsim_gp.c:102-106 for t = 1..nsteps.
 * Asynchronous on the context's stream; errors of earlier launches surface here
 * or in gp_sync.  An isothermal FP64 context replays runs of eight steps from a
 * CUDA graph captured on the first such run from each of its two buffers (the
 * same kernels and arguments as direct launches, one host launch instead of 16). */
int gp_step(gp_ctx *ctx, int64_t nsteps);
/* The context's step count (the frozen temperature gradient's clock: step t uses the temperature
 * the reference sets after step t - 1).  Starts at 0 on creation; gp_step advances it. */
int gp_set_time_step(gp_ctx *ctx, int64_t t);
/* FP32 only (no counterpart in the reference, whose step is FP64): compensated
 * accumulation.  The net face flux of every cell's concentration update, the
 * interface source sum and the bulk and pure-phase increments of mu are summed
 * with error-free transforms (TwoSum, TwoProduct on the fused multiply-add), their
 * rounding errors carried apart and added once, so the update keeps the
 * increments that plain FP32 sums lose against mu's scale.  Off by default; a
 * step costs more arithmetic and no extra memory traffic.  GP_E_ARG on an FP64
 * context. */
int gp_set_compensated(gp_ctx *ctx, int on);
int gp_get_compensated(gp_ctx *ctx);
/* nsteps smoothing pre-steps (the reference runs NSMOOTH - 1 of them before its
 * time loop, microsim_gp.c:97-100; solverloop.h:72-90): the phase-field step
 * without the driving force and with isotropic gradient energy, the
 * concentration step without antitrapping current and source, ghost fill.
 * FP32 contexts run them in FP64 on a copy of their FP32-stored state; the
 * bit-exact route is an FP64 context (the CLI driver smooths the filled doubles
 * in FP64 before an FP32 time loop). */
int gp_smooth(gp_ctx *ctx, int64_t nsteps);
/* Moving frame (Shift = 1; microsim_gp.c:115-125, functions/shift.h):
 * gp_interface_y gives the highest row where the liquid fraction crosses 0.5
 * upwards, in the reference's ghost-padded row index (interior row + 3; 0 when
 * there is none), as check_SHIFT scans it; gp_shift_y moves the window d rows
 * along +y, appending liquid rows (mu = gp_model.mu_shift).  The reference
 * shifts its ghost rows too, and its next phase-field half step reads them
 * before the boundary copy refreshes them: FP64 contexts keep those rows and
 * reproduce it bit for bit; FP32 contexts read the boundary map of the shifted
 * interior. */
int gp_interface_y(gp_ctx *ctx, int64_t *pos);
int gp_shift_y(gp_ctx *ctx, int64_t d);
int gp_sync(gp_ctx *ctx);
/* FP64 statistics of the current state (max/min/rel-change of the last step,
 * solute and phase sums, NaN watchdog). Synchronous. */
int gp_get_stats(gp_ctx *ctx, gp_stats *out);
/* Delta-phi of the most recent phase-field half step on the interior plus one
 * ring, dphi[N][mx+2][my+2] (FP64 context only; for tests). */
int gp_download_dphi(gp_ctx *ctx, double *dphi);
/* The CUDA stream (cudaStream_t) the context launches on. */
void *gp_stream(gp_ctx *ctx);
/* The current state buffers on the device (valid until the next step, smooth
 * or shift): phi [N][mesh_x][pitch], mu [K1][mesh_x][pitch], plane = elements
 * per plane, esize = 8 (FP64) or 4 (FP32).  For callers that exchange rows
 * between contexts (halo rows of a grid split across GPUs); after writing into
 * them, call gp_state_changed. */
int gp_state_device(gp_ctx *ctx, void **phi, void **mu, int64_t *pitch, int64_t *plane, int *esize);
int gp_state_changed(gp_ctx *ctx);
/* Number of kernel launches this context issued since creation. */
int64_t gp_launch_count(const gp_ctx *ctx);
/* ---------------- batches: many independent instances, FP32 chosen form ---------------- */

/* A batch of n instances (uneven sizes and parameters allowed; they must share
 * N and K1; isotropic and anisotropic instances mix: the batch then runs the
 * anisotropic kernels, with no anisotropy for the isotropic instances, whose
 * results then differ from an isotropic batch's by FP32 rounding).  One
 * kernel launch per time step covers
 * every tile of every instance; gp_batch_step replays the launches from a
 * captured CUDA graph.  No counterpart in the reference (one process = one
 * simulation there). */
typedef struct gp_batch gp_batch;
int gp_batch_create(const gp_model *models, int n, gp_batch **out);
int gp_batch_destroy(gp_batch *b);
int gp_batch_upload(gp_batch *b, int i, const double *phi, const double *mu);
int gp_batch_download(gp_batch *b, int i, double *phi, double *mu);
/* As gp_batch_upload / gp_batch_download, but queued on the batch's stream
 * without waiting: the host arrays must stay untouched (and, for a download,
 * unread) until gp_batch_sync or a call that waits.  Copies of consecutive
 * instances then run back to back instead of one host round trip per instance.
 * Page-locked host arrays (cudaHostAlloc, cudaHostRegister, torch pin_memory)
 * are read or written by the FP64 <-> FP32 conversion kernel itself across the
 * link, with no staging copy; they must then hold the instance's whole state
 * (N, resp. K-1, planes of mesh_x * mesh_y doubles). */
int gp_batch_upload_async(gp_batch *b, int i, const double *phi, const double *mu);
int gp_batch_download_async(gp_batch *b, int i, double *phi, double *mu);
/* Every instance at once (phi[i], mu[i] for i < n), queued like the _async
 * calls: page-locked arrays move in one conversion launch over all instances,
 * pageable ones through the staging copies.  gp_batch_sync waits. */
int gp_batch_upload_all(gp_batch *b, const double *const *phi, const double *const *mu);
int gp_batch_download_all(gp_batch *b, double *const *phi, double *const *mu);
int gp_batch_step(gp_batch *b, int64_t nsteps);
/* Capture the step graphs of both buffer parities now, without stepping (the
 * first gp_batch_step would otherwise capture them). */
int gp_batch_prepare(gp_batch *b);
int gp_batch_sync(gp_batch *b);
int gp_batch_get_stats(gp_batch *b, int i, gp_stats *out);
/* gp_batch_get_stats queued on the batch's stream without waiting: the
 * GP_STAT_VALUES reduced FP64 values of instance i land in raw (page-locked host
 * memory of GP_STAT_VALUES doubles, left untouched until gp_batch_sync or a call
 * that waits) when the stream gets there, so a loop can read every step's
 * statistics back without holding the GPU at each step.  gp_batch_stats_from_raw
 * then fills a gp_stats from them, with gp_batch_get_stats's return codes
 * (GP_E_NONFINITE, GP_E_TIMEOUT). */
#define GP_STAT_VALUES 64
int gp_batch_get_stats_async(gp_batch *b, int i, double *raw);
int gp_batch_stats_from_raw(gp_batch *b, int i, const double *raw, gp_stats *out);
/* Tile shape of the fused kernel (tx along x, ty along y): 16x32, 8x32, 32x32, 16x64. */
int gp_batch_set_tile(gp_batch *b, int tx, int ty);
/* Narrow band (on by default): tiles whose cells and two-cell ring were one
 * pure phase after the previous step (per-tile purity words written by every
 * step) take a lean diffusion-only kernel, the rest the full kernel, both
 * launched concurrently; the results are bit-identical with it off. */
int gp_batch_set_narrowband(gp_batch *b, int on);
/* Tiles the next step sends to the lean kernel, all tiles of the batch, and
 * the interior cells of those lean tiles (diagnostics; synchronises the
 * batch's stream). */
int gp_batch_lean_tiles(gp_batch *b, int64_t *lean, int64_t *total, int64_t *lean_cells);
/* Blocks per SM of the two persistent grids (lean kernel, full kernel); 0 =
 * as many as fit.  The kernels run concurrently, so a lean grid below its
 * occupancy leaves every SM room for full-kernel blocks beside it.
 * gp_batch_get_grids also reports the occupancies. */
int gp_batch_set_grids(gp_batch *b, int lean_per_sm, int general_per_sm);
/* Threads per full-kernel block (one interface tile per block): 256, or 512
 * for binary alloys (shorter chains per thread, half the resident blocks:
 * faster when few tiles hold an interface).  The autotuner chooses it too. */
int gp_batch_set_block(gp_batch *b, int threads);
int gp_batch_get_block(gp_batch *b);
/* How the full kernel finds the tiles the lean kernel rejects: 0 = a list
 * kernel collects them into a queue (best with many interface tiles), 1 = each
 * full-kernel block scans its own interleaved share of the tiles (one launch
 * fewer per step, best with few).  The autotuner chooses it too. */
int gp_batch_set_scan(gp_batch *b, int on);
int gp_batch_get_scan(gp_batch *b);
/* Temporal blocking: depth 1 = one launch set per step; depth 2 = blocked
 * pairs.  In a pair the lean tiles (pure on the tile and its two-cell ring)
 * take two diffusion steps from one staged mu box -- half the state traffic per
 * step -- while the full kernel updates the other tiles twice through an
 * intermediate buffer, which the lean tiles bordering them fill with their
 * first step.  The results are bit-identical to single steps.  Needs the narrow
 * band and the list mode (scan off); the autotuner chooses it.  After a pair,
 * rel_change_* of gp_batch_get_stats covers the pair's two steps. */
int gp_batch_set_depth(gp_batch *b, int depth);
int gp_batch_get_depth(gp_batch *b);
/* The frozen temperature gradient's clock of a batch (gp_set_time_step for a
 * context): the number of steps taken, which the next step's temperature
 * depends on (microsim_gp.c:108-113).  Counted by gp_batch_step; set it when
 * resuming a run. */
int gp_batch_set_time_step(gp_batch *b, int64_t t);
/* Compensated accumulation for every instance of the batch (gp_set_compensated). */
int gp_batch_set_compensated(gp_batch *b, int on);
int gp_batch_get_compensated(gp_batch *b);
/* Failure-detection test (no counterpart in the reference): the next step's
 * lean kernel leaves one staged tile box unissued; its wait gives up after one
 * second, the kernel returns, and the next gp_batch_get_stats reports GP_E_TIMEOUT.
 * The batch's results are invalid from then on. */
int gp_batch_test_lose_box(gp_batch *b);
int gp_batch_get_grids(gp_batch *b, int *lean_per_sm, int *general_per_sm, int *occ_lean, int *occ_general);
/* Per-kernel timing (diagnostics): while on, steps launch directly (no graph
 * replay), their kernels one after the other on the batch's stream, and record
 * CUDA events around each kernel; gp_batch_kernel_ms gives
 * the mean milliseconds per step of the lean kernel, the list kernel and the
 * full kernel (ms3[0..2]) over the steps since timing was switched on. */
int gp_batch_set_timing(gp_batch *b, int on);
int gp_batch_kernel_ms(gp_batch *b, double *ms3, int64_t *steps);
/* Measured sweep over the tile shapes, each with full-kernel blocks of 256
 * and (binary alloys) 512 threads, the list or scan way of finding the
 * interface tiles, depth 1 or 2 (list mode), the lean grid at its occupancy,
 * one block per SM below it or half of it, and the full kernel's grid at its
 * occupancy or one block per SM below it, on the batch's own state (restored
 * afterwards); the winner is applied and cached in cache_path (may be NULL)
 * per batch signature (phases, components, anisotropy, cells, instances and the
 * accumulation mode), read back on the next call. */
int gp_batch_autotune(gp_batch *b, const char *cache_path, int *tx, int *ty);
void *gp_batch_stream(gp_batch *b);
/* The current state buffers of instance i on the device (FP32: esize 4), as
 * gp_state_device; after writing into them (halo rows of a grid split across
 * GPUs), call gp_batch_state_changed, which is ordered on the batch's stream. */
int gp_batch_state_device(gp_batch *b, int i, void **phi, void **mu, int64_t *pitch, int64_t *plane, int *esize);
int gp_batch_state_changed(gp_batch *b);
int64_t gp_batch_launch_count(const gp_batch *b);
int64_t gp_batch_cells(const gp_batch *b);

/* One plain (FP64) step that allocates nothing.  No counterpart in the
 * reference: it exists for callers that own their device buffers and cannot
 * allocate device memory (a framework pool that owns the whole GPU, a fixed
 * start-up memory budget).  phi/mu (inputs) and phi_out/mu_out (outputs) are
 * device buffers in this header's layout with the given row pitch (elements,
 * >= mesh_y; plane stride mesh_x*pitch); no output byte may overlap an input
 * or the other output (GP_E_ARG).  The buffers and the stream must belong to
 * this library's current device -- the one gp_set_device chose, device 0 by
 * default, not the host program's own choice -- or the call returns GP_E_ARG.  The
 * Delta-phi ring between the step's two kernels lives in a fixed device array of
 * GP_NOALLOC_SCRATCH_BYTES per GPU, held until the process exits and shared by
 * every call (contents of the last call kept; calls that overlap on the GPU
 * race on it).  Grids needing more than N*(mesh_x+2)*round_up(mesh_y+2,32)
 * doubles of it get GP_E_SIZE.  The first call on a device looks up the array's
 * address and should come before any stream capture.  stream: a cudaStream_t
 * (NULL = legacy default stream); the call is asynchronous on it. */
#define GP_NOALLOC_SCRATCH_BYTES (8u << 20)
int gp_step_f64_noalloc(const gp_model *m, const double *phi, const double *mu, double *phi_out, double *mu_out,
                        int64_t pitch, void *stream);
/* The GPU that contexts, batches and adjoints created next on this thread use.
 * The library carries its own CUDA runtime, so the host program's own choice of
 * device (e.g. torch.cuda.set_device) does not reach it; one process per GPU
 * calls this once with its local rank. */
int gp_set_device(int device);
/* sizeof(gp_model) as compiled into the library (binding layout check). */
size_t gp_model_sizeof(void);
/* Text of the last error on this thread. */
const char *gp_last_error(void);

/* ---- adjoint of the explicit step (binary alloys: N = 2, K-1 = 1) ----------
 * No counterpart in the reference (it has no adjoint).  A hand-written reverse
 * of the plain step's model in FP32 (GP_FP32) or FP64 (GP_FP64), with
 * checkpointing: gp_adj_forward runs nsteps steps from (phi0, mu0), keeping
 * every checkpoint_every-th state (0: ceil(sqrt(nsteps))), and returns the final
 * state; gp_adj_backward takes the adjoint of a loss with respect to that final
 * state (lam_phi [2][mesh_x][mesh_y], lam_mu [mesh_x][mesh_y] or NULL for 0)
 * and returns the gradient with respect to the GP_ADJ_NPARAM parameters
 *   grad[0]  mobility M = 1/tau_ab[0][1] (tau scaled with it)
 *   grad[1]  anisotropy strength dab[0][1]
 *   grad[2]  interface energy Gamma[0][1]
 *   grad[3]  liquid diffusivity Diff[1][0][0]
 * and, when lam_phi0 / lam_mu0 are not NULL, with respect to the initial state.
 * The segment of checkpoint_every steps is recomputed before it is reversed, so
 * ceil(nsteps / checkpoint_every) + checkpoint_every states are stored. */
#define GP_ADJ_NPARAM 4
typedef struct gp_adj gp_adj;
int gp_adj_create(const gp_model *m, int precision, gp_adj **out);
int gp_adj_forward(gp_adj *a, const double *phi0, const double *mu0, int64_t nsteps, int64_t checkpoint_every,
                   double *phi_out, double *mu_out);
int gp_adj_backward(gp_adj *a, const double *lam_phi, const double *lam_mu, double *grad, double *lam_phi0,
                    double *lam_mu0);
int gp_adj_stored_states(const gp_adj *a, int64_t *states);
int gp_adj_destroy(gp_adj *a);

#ifdef __cplusplus
}
#endif
#endif
