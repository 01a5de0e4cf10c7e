/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (oracle side).
 *
 * Drives the reference serial grand-potential solver, compiled from its own
 * sources, and dumps its state so the oracle restatement and the CUDA path can
 * be checked against the reference itself.  Nothing in the product links this.
 *
 * The reference is one translation unit: microsim_gp.c #includes every header
 * that holds the function bodies (Grand_potential_Finite_difference_2D_serial/
 * microsim_gp.c:1-39).  We compile that file unchanged, with its `main`
 * renamed, and call its functions in the order its main does
 * (microsim_gp.c:41-106):
 *
 *   reading_input_parameters -> initialize_variables -> serialinfo_xy ->
 *   initialize_functions_solverloop -> read_boundary_conditions ->
 *   fill_domain -> apply_boundary_conditions -> [smooth x (NSMOOTH-1)] ->
 *   for t: solverloop_phasefield; BC; solverloop_concentration; BC
 *
 * Usage:
 *   gp_ref_harness Input.in Filling.in Out DUMPDIR NSTEPS [dump steps...]
 *     writes DUMPDIR/consts.txt, DUMPDIR/state_<t>.bin for t=0 and each
 *     listed step, DUMPDIR/dphi_1.bin (Delta-phi after the phi half-step of
 *     step 1), DATA/<Out>_0.vtk through the reference's own VTK writer, and
 *     prints "loop_seconds=<s> steps=<n>" on stdout.
 *   gp_ref_harness Input.in Filling.in Out - NSTEPS
 *     timing only (no dumps).
 *
 * With ISOTHERMAL = 0 the frozen temperature gradient is set after the
 * filling and after every step exactly as the reference main does
 * (microsim_gp.c:77-82, 108-113; no moving frame with it).
 */
#define main microsim_reference_main
#include "microsim_gp.c"
#undef main

#include <time.h>

static void dump_state(const char *dir, const char *tag, long tstep, int with_dphi) {
  char name[1200];
  long n = rows_x * rows_y;
  long idx, a2, k2;
  FILE *fp;
  if (with_dphi) {
    sprintf(name, "%s/dphi_%ld.bin", dir, tstep);
  } else {
    sprintf(name, "%s/%s_%ld.bin", dir, tag, tstep);
  }
  fp = fopen(name, "wb");
  if (!fp) { fprintf(stderr, "cannot open %s\n", name); exit(2); }
  {
    long hdr[4];
    hdr[0] = rows_x; hdr[1] = rows_y; hdr[2] = NUMPHASES; hdr[3] = NUMCOMPONENTS;
    fwrite(hdr, sizeof(long), 4, fp);
  }
  if (with_dphi) {
    for (a2 = 0; a2 < NUMPHASES; a2++)
      for (idx = 0; idx < n; idx++) fwrite(&gridinfo[idx].deltaphi[a2], sizeof(double), 1, fp);
  } else {
    for (a2 = 0; a2 < NUMPHASES; a2++)
      for (idx = 0; idx < n; idx++) fwrite(&gridinfo[idx].phia[a2], sizeof(double), 1, fp);
    for (k2 = 0; k2 < NUMCOMPONENTS - 1; k2++)
      for (idx = 0; idx < n; idx++) fwrite(&gridinfo[idx].compi[k2], sizeof(double), 1, fp);
  }
  fclose(fp);
}

static void put_scalar(FILE *fp, const char *name, double v) { fprintf(fp, "%s 1 %.17g\n", name, v); }

static void put_vec(FILE *fp, const char *name, const double *v, long m) {
  long i;
  fprintf(fp, "%s %ld", name, m);
  for (i = 0; i < m; i++) fprintf(fp, " %.17g", v[i]);
  fprintf(fp, "\n");
}

static void dump_consts(const char *dir) {
  char name[1200];
  long a2, b2, c2, i, j;
  long N = NUMPHASES, K1 = NUMCOMPONENTS - 1;
  FILE *fp;
  sprintf(name, "%s/consts.txt", dir);
  fp = fopen(name, "w");
  put_scalar(fp, "NUMPHASES", N);
  put_scalar(fp, "NUMCOMPONENTS", NUMCOMPONENTS);
  put_scalar(fp, "MESH_X", MESH_X);
  put_scalar(fp, "MESH_Y", MESH_Y);
  put_scalar(fp, "deltax", deltax);
  put_scalar(fp, "deltay", deltay);
  put_scalar(fp, "deltat", deltat);
  put_scalar(fp, "epsilon", epsilon);
  put_scalar(fp, "tau", tau);
  put_scalar(fp, "T", T);
  put_scalar(fp, "Teq", Teq);
  put_scalar(fp, "OBSTACLE", OBSTACLE);
  put_scalar(fp, "WELL", WELL);
  put_scalar(fp, "ANISOTROPY", ANISOTROPY);
  put_scalar(fp, "BINARY", BINARY);
  put_scalar(fp, "TERNARY", TERNARY);
  put_scalar(fp, "DILUTE", DILUTE);
  {
    double bt[4];
    bt[0] = boundary[0][0].type; bt[1] = boundary[1][0].type;
    bt[2] = boundary[2][0].type; bt[3] = boundary[3][0].type;
    put_vec(fp, "bc_phi", bt, 4);
    bt[0] = boundary[0][1].type; bt[1] = boundary[1][1].type;
    bt[2] = boundary[2][1].type; bt[3] = boundary[3][1].type;
    put_vec(fp, "bc_mu", bt, 4);
  }
  /* model matrices, flattened row-major */
  {
    double *buf = (double *)malloc(sizeof(double) * (N * N * N * 9 + N * K1 * K1 + 64));
    long m;
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) for (j = 0; j < K1; j++) buf[m++] = cmu[a2][i][j];
    put_vec(fp, "cmu", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) for (j = 0; j < K1; j++) buf[m++] = A[a2][i][j];
    put_vec(fp, "A", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) for (j = 0; j < K1; j++) buf[m++] = Diffusivity[a2][i][j];
    put_vec(fp, "Diffusivity", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) buf[m++] = Beq[a2][i];
    put_vec(fp, "Beq", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) buf[m++] = dBbdT[a2][i];
    put_vec(fp, "dBbdT", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (i = 0; i < K1; i++) buf[m++] = B[a2][i];
    put_vec(fp, "B", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) buf[m++] = C[a2];
    put_vec(fp, "C", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) buf[m++] = Gamma[a2][b2];
    put_vec(fp, "Gamma", buf, m);
    m = 0; for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) buf[m++] = tau_ab[a2][b2];
    put_vec(fp, "tau_ab", buf, m);
    if (ANISOTROPY) {
      m = 0; for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) buf[m++] = dab[a2][b2];
      put_vec(fp, "dab", buf, m);
      m = 0;
      for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) for (i = 0; i < 3; i++) for (j = 0; j < 3; j++)
        buf[m++] = (a2 == b2) ? 0.0 : Rotation_matrix[a2][b2][i][j];
      put_vec(fp, "Rotation_matrix", buf, m);
      m = 0;
      for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) for (i = 0; i < 3; i++) for (j = 0; j < 3; j++)
        buf[m++] = (a2 == b2) ? 0.0 : Inv_Rotation_matrix[a2][b2][i][j];
      put_vec(fp, "Inv_Rotation_matrix", buf, m);
    }
    if (N >= 3) {
      m = 0;
      for (a2 = 0; a2 < N; a2++) for (b2 = 0; b2 < N; b2++) for (c2 = 0; c2 < N; c2++) {
        int distinct = (a2 != b2) && (b2 != c2) && (a2 != c2);
        buf[m++] = distinct ? Gamma_abc[a2][b2][c2] : 0.0;
      }
      put_vec(fp, "Gamma_abc", buf, m);
    }
    free(buf);
  }
  fclose(fp);
}

int main(int argc, char *argv[]) {
  const char *dumpdir;
  long nsteps, i;
  long *dump_at = NULL;
  long ndump = 0;
  struct timespec t0, t1;
  int dumping;

  if (argc < 6) {
    fprintf(stderr, "usage: %s Input.in Filling.in Out DUMPDIR|- NSTEPS [dump steps...]\n", argv[0]);
    return 2;
  }
  dumpdir = argv[4];
  nsteps = atol(argv[5]);
  dumping = strcmp(dumpdir, "-") != 0;
  ndump = argc - 6;
  if (ndump > 0) {
    dump_at = (long *)malloc(sizeof(long) * ndump);
    for (i = 0; i < ndump; i++) dump_at[i] = atol(argv[6 + i]);
  }

  /* microsim_gp.c:42-49 and :84 (fresh start only) */
  mkdir("DATA", 0777);
  reading_input_parameters(argv);
  initialize_variables();
  serialinfo_xy();
  initialize_functions_solverloop();
  read_boundary_conditions(argv);
  fill_domain(argv);
  /* microsim_gp.c:77-82 */
  if (TEMPGRADY) {
    BASE_POS    = (temperature_gradientY.gradient_OFFSET/deltay) - shift_OFFSET;
    GRADIENT    = (temperature_gradientY.DeltaT)*deltay/(temperature_gradientY.Distance);
    temp_bottom = temperature_gradientY.base_temp - BASE_POS*GRADIENT;
    apply_temperature_gradientY(gridinfo, shift_OFFSET, 0);
  }
  apply_boundary_conditions(0);

  if (dumping) {
    dump_consts(dumpdir);
    dump_state(dumpdir, "state", 0, 0);
    /* the reference's own VTK writer (solverloop/file_writer.h:23-46) */
    if (ASCII == 0) writetofile_serial2D_binary(gridinfo, argv, 0);
    else writetofile_serial2D(gridinfo, argv, 0);
  }
  /* microsim_gp.c:97-100 (pre-conditioning) */
  for (t = 1; t < nsmooth; t++) {
    smooth(start, end);
    apply_boundary_conditions(0);
  }
  if (dumping && nsmooth > 1) dump_state(dumpdir, "smoothed", 0, 0);

  clock_gettime(CLOCK_MONOTONIC, &t0);
  /* microsim_gp.c:102-106 */
  for (t = 1; t <= nsteps; t++) {
    solverloop_phasefield(start, end);
    apply_boundary_conditions(0);
    if (dumping && t == 1) dump_state(dumpdir, "dphi", 1, 1);
    solverloop_concentration(start, end);
    apply_boundary_conditions(0);
    /* microsim_gp.c:108-113: the frozen gradient after the step */
    if (TEMPGRADY) {
      BASE_POS    = (temperature_gradientY.gradient_OFFSET/deltay) - shift_OFFSET + ((temperature_gradientY.velocity/deltay)*(t*deltat));
      GRADIENT    = (temperature_gradientY.DeltaT)*deltay/(temperature_gradientY.Distance);
      temp_bottom = temperature_gradientY.base_temp - BASE_POS*GRADIENT;
      apply_temperature_gradientY(gridinfo, shift_OFFSET, t);
    }
    /* microsim_gp.c:115-125: the moving frame, every 100 steps */
    if (t % 100 == 0 && SHIFT) {
      if (MAX_INTERFACE_POS > shiftj) shift_ON = 1;
      if (shift_ON) {
        apply_shiftY(gridinfo, MAX_INTERFACE_POS);
        shift_OFFSET += (MAX_INTERFACE_POS - shiftj);
        shift_ON = 0;
      }
      printf("shift %ld %ld %ld\n", (long)t, (long)MAX_INTERFACE_POS, (long)shift_OFFSET);
    }
    if (dumping) {
      for (i = 0; i < ndump; i++) {
        if (dump_at[i] == t) dump_state(dumpdir, "state", t, 0);
      }
    }
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  printf("loop_seconds=%.9f steps=%ld cells=%ld\n",
         (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec), nsteps, MESH_X * MESH_Y);
  {
    long b2, k2;
    for (b2 = 0; b2 < NUMPHASES; b2++)
      printf("stat phi %ld %.17g %.17g %.17g\n", b2, global_max_min.phi_max[b2], global_max_min.phi_min[b2],
             global_max_min.rel_change_phi[b2]);
    for (k2 = 0; k2 < NUMCOMPONENTS - 1; k2++)
      printf("stat mu %ld %.17g %.17g %.17g\n", k2, global_max_min.mu_max[k2], global_max_min.mu_min[k2],
             global_max_min.rel_change_mu[k2]);
  }
  return 0;
}
