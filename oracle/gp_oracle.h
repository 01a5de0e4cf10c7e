/*
 * gp_oracle.h -- CPU restatement of the MicroSim grand-potential explicit step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product never links or calls it.
 *
 * It restates Grand_potential_Finite_difference_2D_serial (2D, isothermal,
 * Function_F = 1) in plain C: same ghost-padded layout (index = y + x*rows_y,
 * rows = MESH + 6), same arithmetic order, no FMA, so that the interior cells
 * match the reference bit for bit.  Parity of this restatement against the
 * reference itself is pinned by tests/golden (fixtures produced by running the
 * reference, compiled from its own sources, through oracle/ref_harness.c).
 */
#ifndef GP_ORACLE_H_
#define GP_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int N;            /* NUMPHASES; the last phase is the liquid                 */
  int K1;           /* NUMCOMPONENTS-1 (independent chemical potentials)       */
  long mesh_x, mesh_y;
  double dx, dy, dt;
  double epsilon;   /* interface width                                         */
  double tau;       /* fallback relaxation constant (FunctionTau)              */
  double T, Teq;
  int obstacle;     /* 1: Function_W = 1 (obstacle), 0: Function_W = 2 (well)  */
  int anisotropy;   /* Function_anisotropy (0 or 1, 4-fold cubic)              */
  int binary, ternary, dilute;  /* mu-solve selection, as in the Input.in keys */
  int bc_phi[4];    /* boundary[0..3] types for phi: x-lo, x-hi, y-hi, y-lo    */
  int bc_mu[4];     /* same for mu (1 = Neumann, 3 = periodic)                 */
  const double *Gamma;      /* [N][N]                                        */
  const double *Gamma_abc;  /* [N][N][N] (may be NULL when N < 3)            */
  const double *tau_ab;     /* [N][N]                                        */
  const double *dab;        /* [N][N] (anisotropy only)                      */
  const double *R;          /* [N][N][3][3] rotation matrices                */
  const double *Rinv;       /* [N][N][3][3] their LU inverses                */
  const double *cmu;        /* [N][K1][K1] = inverse of d(mu)/dc             */
  const double *A;          /* [N][K1][K1]                                   */
  const double *Beq;        /* [N][K1]                                       */
  const double *dBbdT;      /* [N][K1]                                       */
  const double *B;          /* [N][K1] at T                                  */
  const double *C;          /* [N]     at T                                  */
  const double *Diff;       /* [N][K1][K1] diffusivities                     */
} gpo_params;

typedef struct {
  double phi_max[8], phi_min[8], rel_change_phi[8];
  double mu_max[8], mu_min[8], rel_change_mu[8];
} gpo_stats;

/* Ghost fill, Neumann (type 1) and periodic (type 3) copies
 * (solverloop/boundary_serial.h:176-203 with the index tables of
 * functions/utility_functions.h:471-653). */
void gpo_apply_bc(const gpo_params *p, double *phi, double *mu);

/* Advance nsteps explicit steps in place on ghost-padded SoA planes
 * phi[N][rows_x*rows_y], mu[K1][rows_x*rows_y].  If dphi_first is not NULL it
 * receives Delta-phi of the first step on the ring [2, rows-3]^2.
 * Stats (if not NULL) follow microsim_gp.c's running max/min and the last
 * step's sum of squared changes, over interior cells.  Returns 0, or -1 for
 * unsupported parameters. */
/* nsteps smoothing pre-steps (the reference runs NSMOOTH - 1 of them before
 * the time loop), each followed by the boundary copy. */
int gpo_smooth(const gpo_params *p, double *phi, double *mu, long nsteps);
int gpo_step(const gpo_params *p, double *phi, double *mu, long nsteps, double *dphi_first,
             gpo_stats *st);

#ifdef __cplusplus
}
#endif
#endif
