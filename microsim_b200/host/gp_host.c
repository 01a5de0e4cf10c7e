/*
 * gp_host.c -- host side of the drop-in: Input.in / Filling.in parsing, model
 * constants, initial filling and VTK files, with the reference's semantics.
 *
 * Reference paths are relative to Grand_potential_Finite_difference_2D_serial/.
 * Built with -ffp-contract=off: the constants here must come out as the
 * reference's doubles (x86-64 gcc without -march never fuses a*b+c).
 */
#include "gp_b200.h"

#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PMAX 16 /* phases the parser accepts (kernels: GP_MAX_PHASES) */
#define KMAX 8  /* components the parser accepts                      */
#define MAXFILL 4096

#include <stdarg.h>

/* last error text, per thread */
static __thread char g_err[512];

void gp_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

const char *gp_last_error(void) { return g_err; }

enum { FILL_CUBE = 1, FILL_CYLINDER, FILL_SPHERE, FILL_ELLIPSE };

typedef struct {
  int kind;
  long phase;
  long v[6];
  double r;
} fill_op;

struct gp_input {
  int DIMENSION;
  long MESH_X, MESH_Y, MESH_Z;
  double deltax, deltay, deltaz, deltat;
  int NUMPHASES, NUMCOMPONENTS;
  long ntimesteps, saveT, nsmooth, STARTTIME, RESTART;
  double R, V;
  int ASCII;
  long time_output;
  double TEMPERATURE_SCALE, Teq, Tfill, T, tilt_angle, Rtheta;
  char Components[KMAX][GP_NAME_LEN];
  char Phases[PMAX][GP_NAME_LEN];
  int FUNCTION_ANISOTROPY, FOLD, OBSTACLE, FUNCTION_W, FUNCTION_F, ISOTHERMAL, TEMPGRADY;
  double tempgrady[5];
  int SHIFT;
  long shiftj;
  int BINARY, TERNARY, DILUTE, WRITECOMPOSITION, NOISE_PHASEFIELD;
  double AMP_NOISE_PHASE;
  double epsilon, tau;
  int have_gamma, have_tau, have_dab, have_gabc;
  double Gamma[PMAX][PMAX], tau_ab[PMAX][PMAX], dab[PMAX][PMAX];
  double Gamma_abc[PMAX][PMAX][PMAX];
  double Diffusivity[PMAX][KMAX][KMAX];
  double ceq[PMAX][PMAX][KMAX], cfill[PMAX][PMAX][KMAX], slopes[PMAX][PMAX][KMAX];
  double A[PMAX][KMAX][KMAX];
  double Rot[PMAX][PMAX][3][3], RotInv[PMAX][PMAX][3][3];
  int have_rot[PMAX][PMAX];
  int bc_type[6][3];       /* boundary[i][j].type, j: 0 phi, 1 mu, 2 T           */
  int bc_proxy_type[6][3]; /* type seen when BOUNDARY_VALUE assigned the proxies */
  int nfill;
  fill_op fill[MAXFILL];
  int n_unknown;
};

/* ------------------------------------------------------------------------- */
/* small linear algebra, ported from functions/matrix.h                      */
/* ------------------------------------------------------------------------- */

/* matinvnew (functions/matrix.h:50-114): LU with the reference's signed
 * pivot, forward/back substitution with pow(x,-1), then the input matrix is
 * rebuilt from L*U with rows swapped back -- the reference leaves that rebuilt
 * matrix in place of its input, and later reads it (Rotation_matrix). */
static void host_matinv(double *m, double *inv, int n) {
  double fac[KMAX * KMAX], inv1[KMAX * KMAX], prod[KMAX * KMAX];
  int tag[KMAX], i, j, k;
  for (k = 0; k < n; k++) tag[k] = k;
  for (i = 0; i < n * n; i++) fac[i] = 0.0;
  for (k = 0; k < n; k++) {
    /* pivot(), matrix.h:161-191 -- `big` keeps the signed entry */
    double big = fabs(m[k * n + k]);
    int t1 = k, ts;
    for (i = k + 1; i < n; i++)
      if (fabs(m[i * n + k]) > big) { t1 = i; big = m[i * n + k]; }
    ts = tag[k]; tag[k] = tag[t1]; tag[t1] = ts;
    for (i = 0; i < n; i++) { double s = m[k * n + i]; m[k * n + i] = m[t1 * n + i]; m[t1 * n + i] = s; }
    for (i = 0; i < k; i++) { double s = fac[k * n + i]; fac[k * n + i] = fac[t1 * n + i]; fac[t1 * n + i] = s; }
    for (i = k + 1; i < n; i++) {
      double f = -m[i * n + k] / m[k * n + k];
      fac[i * n + k] = -f;
      for (j = k; j <= n - 1; j++) m[i * n + j] = f * m[k * n + j] + m[i * n + j];
    }
  }
  for (i = 0; i < n; i++)
    for (j = 0; j < n; j++) {
      if (i == j) fac[i * n + j] = 1;
      if (j > i) fac[i * n + j] = 0;
    }
  for (i = 0; i < n; i++) {
    double v1[KMAX], v[KMAX];
    /* substitutef, matrix.h:132-149 */
    v1[0] = (i == 0) ? 1.0 : 0.0;
    for (k = 1; k < n; k++) {
      double s = 0;
      for (j = 0; j < k; j++) s = s - fac[k * n + j] * v1[j];
      v1[k] = ((k == i) ? 1.0 : 0.0) + s;
    }
    /* substituteb, matrix.h:117-129 */
    v[n - 1] = v1[n - 1] * pow(m[(n - 1) * n + (n - 1)], -1);
    for (k = n - 2; k >= 0; k--) {
      double s = 0;
      for (j = k + 1; j < n; j++) s = s - m[k * n + j] * v[j];
      v[k] = (v1[k] + s) * pow(m[k * n + k], -1);
    }
    for (j = 0; j < n; j++) inv1[j * n + i] = v[j];
  }
  /* colswap, matrix.h:193-204 */
  for (j = 0; j < n; j++)
    for (k = 0; k < n; k++) inv[k * n + tag[j]] = inv1[k * n + j];
  /* multiply2d(factor, coeffmatrix) then rowswap back, matrix.h:105-106 */
  for (k = 0; k < n; k++)
    for (i = 0; i < n; i++) {
      double s = 0;
      for (j = 0; j < n; j++) s = s + fac[k * n + j] * m[j * n + i];
      prod[k * n + i] = s;
    }
  for (j = 0; j < n; j++)
    for (k = 0; k < n; k++) m[tag[j] * n + k] = prod[j * n + k];
}

/* multiply2d, functions/matrix.h:35-48 */
static void host_mul3(const double a[3][3], const double b[3][3], double out[3][3]) {
  int k, i, j;
  for (k = 0; k < 3; k++)
    for (i = 0; i < 3; i++) {
      double s = 0;
      for (j = 0; j < 3; j++) s = s + a[k][j] * b[j][i];
      out[k][i] = s;
    }
}

/* get_Rotation_Matrix, functions/utility_functions.h:655-699 */
static void rotation_axis(double R[3][3], double theta, int axis) {
  double c = cos(theta * M_PI / 180.0);
  double s = sin(theta * M_PI / 180.0);
  memset(R, 0, sizeof(double) * 9);
  if (axis == 0) {
    R[0][0] = 1.0; R[1][1] = c; R[1][2] = -s; R[2][1] = s; R[2][2] = c;
  } else if (axis == 1) {
    R[0][0] = c; R[0][2] = s; R[2][0] = -s; R[1][1] = 1.0; R[2][2] = c;
  } else {
    R[0][0] = c; R[0][1] = -s; R[1][0] = s; R[1][1] = c; R[2][2] = 1.0;
  }
}

/* ------------------------------------------------------------------------- */
/* Input.in grammar                                                          */
/* ------------------------------------------------------------------------- */

/* Tokens of "{a, b, c}" split on "{,}" like strtok_r (empty tokens dropped,
 * blanks kept: atof/atol skip them, names keep them). */
static int tokenize(const char *s, char tok[][GP_NAME_LEN], int maxtok) {
  int n = 0;
  const char *p = s;
  while (*p) {
    while (*p && strchr("{,}", *p)) p++;
    if (!*p) break;
    const char *q = p;
    while (*q && !strchr("{,}", *q)) q++;
    if (n < maxtok) {
      size_t len = (size_t)(q - p);
      if (len >= GP_NAME_LEN) len = GP_NAME_LEN - 1;
      memcpy(tok[n], p, len);
      tok[n][len] = 0;
    }
    n++;
    p = q;
  }
  return n;
}

#define MAXTOK 64

static int parse_pairs(double M[PMAX][PMAX], int N, const char *val) {
  char tok[MAXTOK][GP_NAME_LEN];
  int nt = tokenize(val, tok, MAXTOK), i, j, k = 0;
  /* populate_matrix, functions/utility_functions.h:84-117 */
  for (i = 0; i < N; i++)
    for (j = i + 1; j < N; j++) {
      M[i][i] = 0.0;
      if (k >= nt) return GP_E_PARSE;
      M[i][j] = atof(tok[k]);
      M[j][i] = M[i][j];
      k++;
    }
  return GP_OK;
}

int gp_input_read(const char *input_in, const char *filling_in, gp_input **out) {
  FILE *fr;
  char line[1000], key[101], val[101];
  gp_input *in;
  if (!input_in || !out) { gp_set_error("gp_input_read: NULL argument"); return GP_E_ARG; }
  fr = fopen(input_in, "rt");
  if (!fr) { gp_set_error("file %s not found", input_in); return GP_E_IO; }
  in = (gp_input *)calloc(1, sizeof(gp_input));
  if (!in) { fclose(fr); return GP_E_NOMEM; }
  /* defaults of functions/global_vars.h */
  in->FUNCTION_W = 1;
  in->FUNCTION_ANISOTROPY = 1;
  in->FUNCTION_F = 1;
  int rc = GP_OK;
  /* first pass: reading_input_parameters.h:24-307 */
  while (fgets(line, sizeof line, fr)) {
    key[0] = val[0] = 0;
    /* A line that is not "KEY = VALUE;" is skipped.  (The reference's sscanf
     * leaves its buffers untouched on such a line and re-applies the previous
     * key to a strtok-mangled value; nothing sensible depends on that.) */
    if (sscanf(line, "%100s = %100[^;];", key, val) < 1) continue;
    if (key[0] == '#') continue;
    int N = in->NUMPHASES, K1 = in->NUMCOMPONENTS - 1;
    int mats = (N > 0) && (K1 > 0);
    char tok[MAXTOK][GP_NAME_LEN];
    int nt, i, j;
    if (!strcmp(key, "DIMENSION")) in->DIMENSION = atoi(val);
    else if (!strcmp(key, "MESH_X")) in->MESH_X = atol(val);
    else if (!strcmp(key, "MESH_Y")) in->MESH_Y = atol(val);
    else if (!strcmp(key, "MESH_Z")) in->MESH_Z = atol(val);
    else if (!strcmp(key, "DELTA_X")) in->deltax = atof(val);
    else if (!strcmp(key, "DELTA_Y")) in->deltay = atof(val);
    else if (!strcmp(key, "DELTA_Z")) in->deltaz = atof(val);
    else if (!strcmp(key, "DELTA_t")) in->deltat = atof(val);
    else if (!strcmp(key, "NUMPHASES")) {
      in->NUMPHASES = atoi(val);
      if (in->NUMPHASES < 1 || in->NUMPHASES > PMAX) { rc = GP_E_UNSUPPORTED; gp_set_error("NUMPHASES=%d outside 1..%d", in->NUMPHASES, PMAX); break; }
    } else if (!strcmp(key, "NUMCOMPONENTS")) {
      in->NUMCOMPONENTS = atoi(val);
      if (in->NUMCOMPONENTS < 2 || in->NUMCOMPONENTS > KMAX + 1) { rc = GP_E_UNSUPPORTED; gp_set_error("NUMCOMPONENTS=%d outside 2..%d", in->NUMCOMPONENTS, KMAX + 1); break; }
    } else if (!strcmp(key, "epsilon")) in->epsilon = atof(val);
    else if (!strcmp(key, "tau")) in->tau = atof(val);
    else if (!strcmp(key, "NTIMESTEPS")) in->ntimesteps = atol(val);
    else if (!strcmp(key, "SAVET")) in->saveT = atol(val);
    else if (!strcmp(key, "NSMOOTH")) in->nsmooth = atol(val);
    else if (!strcmp(key, "STARTTIME")) in->STARTTIME = atol(val);
    else if (!strcmp(key, "RESTART")) in->RESTART = atol(val);
    else if (!strcmp(key, "R")) in->R = atof(val);
    else if (!strcmp(key, "V")) in->V = atof(val);
    else if (!strcmp(key, "WRITEFORMAT")) {
      if (!strcmp(val, "ASCII")) in->ASCII = 1;
      else if (!strcmp(val, "BINARY")) in->ASCII = 0;
    } else if (!strcmp(key, "TRACK_PROGRESS")) in->time_output = atol(val);
    else if (!strcmp(key, "TEMPERATURE_SCALE")) in->TEMPERATURE_SCALE = atof(val);
    else if (!strcmp(key, "Equilibrium_temperature")) in->Teq = atof(val);
    else if (!strcmp(key, "Filling_temperature")) in->Tfill = atof(val);
    else if (!strcmp(key, "T")) in->T = atof(val);
    else if (!strcmp(key, "tilt_angle")) in->tilt_angle = atof(val);
    else if (!strcmp(key, "Rtheta")) in->Rtheta = atof(val);
    else if (!strcmp(key, "COMPONENTS")) {
      nt = tokenize(val, tok, MAXTOK);
      for (i = 0; i < nt && i < KMAX; i++) strcpy(in->Components[i], tok[i]);
    } else if (!strcmp(key, "PHASES")) {
      nt = tokenize(val, tok, MAXTOK);
      for (i = 0; i < nt && i < PMAX; i++) strcpy(in->Phases[i], tok[i]);
    } else if (!strcmp(key, "Function_anisotropy") && mats) in->FUNCTION_ANISOTROPY = atoi(val);
    else if (!strcmp(key, "Anisotropy_type") && in->FUNCTION_ANISOTROPY != 0) in->FOLD = atoi(val);
    else if (!strcmp(key, "Rotation_matrix") && in->FUNCTION_ANISOTROPY != 0) {
      /* populate_rotation_matrix, functions/utility_functions.h:700-774 */
      double Rx[3][3], Ry[3][3], Rz[3][3], mult[3][3], M[3][3], Mi[3][3];
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 5 || N < 1) { rc = GP_E_PARSE; gp_set_error("Rotation_matrix needs 5 entries after NUMPHASES"); break; }
      long p1 = atol(tok[0]), p2 = atol(tok[1]);
      if (p1 < 0 || p2 < 0 || p1 >= N || p2 >= N) { rc = GP_E_PARSE; gp_set_error("Rotation_matrix phase out of range"); break; }
      rotation_axis(Rx, atof(tok[2]), 0);
      rotation_axis(Ry, atof(tok[3]), 1);
      rotation_axis(Rz, atof(tok[4]), 2);
      host_mul3((const double(*)[3])Rx, (const double(*)[3])Ry, mult);
      host_mul3((const double(*)[3])mult, (const double(*)[3])Rz, M);
      host_matinv(&M[0][0], &Mi[0][0], 3);
      memcpy(in->Rot[p1][p2], M, sizeof M);
      memcpy(in->RotInv[p1][p2], Mi, sizeof Mi);
      memcpy(in->Rot[p2][p1], M, sizeof M);
      memcpy(in->RotInv[p2][p1], Mi, sizeof Mi);
      in->have_rot[p1][p2] = in->have_rot[p2][p1] = 1;
    } else if (!strcmp(key, "OBSTACLE")) in->OBSTACLE = atoi(val);
    else if (!strcmp(key, "Function_W") && mats) in->FUNCTION_W = atoi(val);
    else if (!strcmp(key, "ISOTHERMAL")) {
      in->ISOTHERMAL = atoi(val);
      if (!in->ISOTHERMAL) in->TEMPGRADY = 1;
    } else if (!strcmp(key, "Tempgrady") && in->TEMPGRADY) {
      nt = tokenize(val, tok, MAXTOK);
      for (i = 0; i < 5 && i < nt; i++) in->tempgrady[i] = atof(tok[i]);
    } else if (!strcmp(key, "Shift")) in->SHIFT = atoi(val);
    else if (!strcmp(key, "Shiftj")) {
      if (in->SHIFT) in->shiftj = atol(val);
    } else if (!strcmp(key, "BINARY")) { in->BINARY = atoi(val); in->TERNARY = 0; in->DILUTE = 0; }
    else if (!strcmp(key, "TERNARY")) { in->TERNARY = atoi(val); in->BINARY = 0; in->DILUTE = 0; }
    else if (!strcmp(key, "DILUTE")) { in->DILUTE = atoi(val); in->BINARY = 0; in->TERNARY = 0; }
    else if (!strcmp(key, "Writecomposition")) in->WRITECOMPOSITION = atoi(val);
    else if (!strcmp(key, "Noise_phasefield")) in->NOISE_PHASEFIELD = atoi(val);
    else if (!strcmp(key, "Amp_Noise_Phase")) {
      if (in->NOISE_PHASEFIELD) in->AMP_NOISE_PHASE = atof(val);
    } else if (!strcmp(key, "GAMMA") && N > 0) {
      if ((rc = parse_pairs(in->Gamma, N, val)) != GP_OK) { gp_set_error("GAMMA needs N(N-1)/2 entries"); break; }
      in->have_gamma = 1;
    } else if (!strcmp(key, "Tau") && N > 0) {
      if ((rc = parse_pairs(in->tau_ab, N, val)) != GP_OK) { gp_set_error("Tau needs N(N-1)/2 entries"); break; }
      in->have_tau = 1;
    } else if (!strcmp(key, "dab") && N > 0) {
      if ((rc = parse_pairs(in->dab, N, val)) != GP_OK) { gp_set_error("dab needs N(N-1)/2 entries"); break; }
      in->have_dab = 1;
    } else if ((!strcmp(key, "ec") || !strcmp(key, "e2") || !strcmp(key, "e4") || !strcmp(key, "beta")) && N > 0) {
      /* parsed by the reference, used by no path of the solver */
    } else if (!strcmp(key, "Gamma_abc") && N > 0) {
      /* populate_matrix3M, functions/utility_functions.h:119-162 */
      int l = 0, k;
      nt = tokenize(val, tok, MAXTOK);
      for (i = 0; i < N; i++)
        for (j = i + 1; j < N; j++)
          for (k = j + 1; k < N; k++) {
            if (l >= nt) { rc = GP_E_PARSE; break; }
            double g = atof(tok[l++]);
            in->Gamma_abc[i][j][k] = in->Gamma_abc[i][k][j] = in->Gamma_abc[j][i][k] = g;
            in->Gamma_abc[j][k][i] = in->Gamma_abc[k][i][j] = in->Gamma_abc[k][j][i] = g;
          }
      if (rc != GP_OK) { gp_set_error("Gamma_abc needs N(N-1)(N-2)/6 entries"); break; }
      in->have_gabc = 1;
    } else if (!strcmp(key, "DIFFUSIVITY") && mats) {
      /* populate_diffusivity_matrix, functions/utility_functions.h:163-218 */
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 2 + K1) { rc = GP_E_PARSE; gp_set_error("DIFFUSIVITY too short"); break; }
      long ph = atol(tok[1]);
      if (ph < 0 || ph >= N) { rc = GP_E_PARSE; gp_set_error("DIFFUSIVITY phase out of range"); break; }
      int l = 1;
      for (i = 0; i < K1; i++) { in->Diffusivity[ph][i][i] = atof(tok[1 + l]); l++; }
      if (!strcmp(tok[0], "1")) {
        for (i = 0; i < K1; i++)
          for (j = i + 1; j < K1; j++) in->Diffusivity[ph][i][j] = in->Diffusivity[ph][j][i] = 0.0;
      } else {
        if (nt < 2 + K1 + K1 * K1) { rc = GP_E_PARSE; gp_set_error("DIFFUSIVITY (full) too short"); break; }
        for (i = 0; i < K1; i++)
          for (j = 0; j < K1; j++) { in->Diffusivity[ph][i][j] = atof(tok[1 + l]); l++; }
      }
    } else if ((!strcmp(key, "ceq") || !strcmp(key, "cfill") || !strcmp(key, "slopes")) && mats) {
      /* populate_thermodynamic_matrix, functions/utility_functions.h:259-292 */
      double(*M)[PMAX][KMAX] = !strcmp(key, "ceq") ? in->ceq : (!strcmp(key, "cfill") ? in->cfill : in->slopes);
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 2 + K1) { rc = GP_E_PARSE; gp_set_error("%s too short", key); break; }
      int p1 = atoi(tok[0]), p2 = atoi(tok[1]);
      if (p1 < 0 || p2 < 0 || p1 >= N || p2 >= N) { rc = GP_E_PARSE; gp_set_error("%s phase out of range", key); break; }
      for (i = 0; i < K1; i++) M[p1][p2][i] = atof(tok[2 + i]);
    } else if (!strcmp(key, "Function_F") && mats) in->FUNCTION_F = atoi(val);
    else if (!strcmp(key, "A") && mats) {
      /* populate_A_matrix, functions/utility_functions.h:219-257 */
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 1 + K1 + K1 * (K1 - 1) / 2) { rc = GP_E_PARSE; gp_set_error("A too short"); break; }
      long ph = atol(tok[0]);
      if (ph < 0 || ph >= N) { rc = GP_E_PARSE; gp_set_error("A phase out of range"); break; }
      int l = 1;
      for (i = 0; i < K1; i++) { in->A[ph][i][i] = atof(tok[l]); l++; }
      for (i = 0; i < K1; i++)
        for (j = i + 1; j < K1; j++) { in->A[ph][i][j] = in->A[ph][j][i] = atof(tok[l]); l++; }
    } else if ((!strcmp(key, "EIGEN_STRAIN") || !strcmp(key, "VOIGT_ISOTROPIC")) && N > 0) {
      /* elasticity inputs: parsed by the reference, unused by this solver */
    } else if (!strcmp(key, "BOUNDARY") || !strcmp(key, "BOUNDARY_VALUE")) {
      /* second pass below (read_boundary_conditions.h); the reference's first
       * pass reports them as unrecognised */
      in->n_unknown++;
    } else {
      in->n_unknown++;
    }
  }
  fclose(fr);
  if (rc != GP_OK) { free(in); return rc; }

  /* second pass: read_boundary_conditions.h:29-41 */
  fr = fopen(input_in, "rt");
  if (!fr) { free(in); return GP_E_IO; }
  while (fgets(line, sizeof line, fr)) {
    key[0] = val[0] = 0;
    if (sscanf(line, "%100s = %100[^;];", key, val) < 1) continue;
    if (key[0] == '#' || in->NUMPHASES <= 0) continue;
    char tok[MAXTOK][GP_NAME_LEN];
    int nt, j = -1;
    if (!strcmp(key, "BOUNDARY")) {
      /* initialize_boundary_conditions + assign_buffer_points_conditions,
       * utility_functions.h:376-421, 471-542: note LEFT = tmp[2], RIGHT = tmp[1] */
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 7) { rc = GP_E_PARSE; gp_set_error("BOUNDARY needs 7 entries"); break; }
      if (!strcmp(tok[0], "phi")) j = 0;
      else if (!strcmp(tok[0], "mu")) j = 1;
      else if (!strcmp(tok[0], "T")) j = 2;
      if (j < 0) continue;
      int t[6];
      t[0] = atoi(tok[2]); t[1] = atoi(tok[1]); t[2] = atoi(tok[3]);
      t[3] = atoi(tok[4]); t[4] = atoi(tok[5]); t[5] = atoi(tok[6]);
      if (t[0] == 3 || t[1] == 3) t[0] = t[1] = 3;
      if (t[2] == 3 || t[3] == 3) t[2] = t[3] = 3;
      if (t[4] == 3 || t[5] == 3) t[4] = t[5] = 3;
      if (in->DIMENSION == 2) t[4] = t[5] = 0;
      int s;
      for (s = 0; s < 6; s++) in->bc_type[s][j] = t[s];
    } else if (!strcmp(key, "BOUNDARY_VALUE")) {
      /* assign_boundary_points_values sets the copy proxies for the types of
       * the BOUNDARY lines read so far (utility_functions.h:544-654) */
      nt = tokenize(val, tok, MAXTOK);
      if (nt < 1) continue;
      if (!strcmp(tok[0], "phi")) j = 0;
      else if (!strcmp(tok[0], "mu")) j = 1;
      else if (!strcmp(tok[0], "T")) j = 2;
      if (j < 0) continue;
      int s;
      for (s = 0; s < 6; s++) in->bc_proxy_type[s][j] = in->bc_type[s][j];
    }
  }
  fclose(fr);
  if (rc != GP_OK) { free(in); return rc; }

  /* Filling.in: functions/fill_domain.h:4-151 */
  if (filling_in) {
    fr = fopen(filling_in, "rt");
    if (!fr) { gp_set_error("file %s not found", filling_in); free(in); return GP_E_IO; }
    while (fgets(line, sizeof line, fr)) {
      key[0] = val[0] = 0;
      if (sscanf(line, "%100s = %100[^;];", key, val) < 1) continue;
      if (key[0] == '#') continue;
      if (!(in->NUMPHASES > 0 && in->NUMCOMPONENTS - 1 > 0)) continue;
      char tok[MAXTOK][GP_NAME_LEN];
      int nt = tokenize(val, tok, MAXTOK), i;
      fill_op op;
      memset(&op, 0, sizeof op);
      if (!strcmp(key, "FILLCUBE")) { op.kind = FILL_CUBE; if (nt < 7) rc = GP_E_PARSE; }
      else if (!strcmp(key, "FILLCYLINDER")) { op.kind = FILL_CYLINDER; if (nt < 6) rc = GP_E_PARSE; }
      else if (!strcmp(key, "FILLSPHERE")) { op.kind = FILL_SPHERE; if (nt < 5) rc = GP_E_PARSE; }
      else if (!strcmp(key, "FILLELLIPSE")) { op.kind = FILL_ELLIPSE; if (nt < 7) rc = GP_E_PARSE; }
      else continue;
      if (rc != GP_OK) { gp_set_error("%s: too few entries", key); break; }
      if (in->nfill >= MAXFILL) { rc = GP_E_SIZE; gp_set_error("more than %d FILL lines", MAXFILL); break; }
      op.phase = atol(tok[0]);
      if (op.phase < 0 || op.phase >= in->NUMPHASES) { rc = GP_E_PARSE; gp_set_error("%s phase out of range", key); break; }
      if (op.kind == FILL_CYLINDER) {
        for (i = 0; i < 4; i++) op.v[i] = atol(tok[1 + i]);
        op.r = atof(tok[5]);
      } else if (op.kind == FILL_SPHERE) {
        for (i = 0; i < 3; i++) op.v[i] = atol(tok[1 + i]);
        op.r = atof(tok[4]);
      } else {
        for (i = 0; i < 6; i++) op.v[i] = atol(tok[1 + i]);
      }
      in->fill[in->nfill++] = op;
    }
    fclose(fr);
    if (rc != GP_OK) { free(in); return rc; }
  }
  *out = in;
  return GP_OK;
}

void gp_input_free(gp_input *in) { free(in); }

int gp_input_get_long(const gp_input *in, const char *key, int64_t *v) {
  if (!in || !key || !v) return GP_E_ARG;
  if (!strcmp(key, "MESH_X")) *v = in->MESH_X;
  else if (!strcmp(key, "MESH_Y")) *v = in->MESH_Y;
  else if (!strcmp(key, "NUMPHASES")) *v = in->NUMPHASES;
  else if (!strcmp(key, "NUMCOMPONENTS")) *v = in->NUMCOMPONENTS;
  else if (!strcmp(key, "NTIMESTEPS")) *v = in->ntimesteps;
  else if (!strcmp(key, "SAVET")) *v = in->saveT;
  else if (!strcmp(key, "NSMOOTH")) *v = in->nsmooth;
  else if (!strcmp(key, "STARTTIME")) *v = in->STARTTIME;
  else if (!strcmp(key, "RESTART")) *v = in->RESTART;
  else if (!strcmp(key, "TRACK_PROGRESS")) *v = in->time_output;
  else if (!strcmp(key, "Shift")) *v = in->SHIFT;
  else if (!strcmp(key, "Shiftj")) *v = in->shiftj;
  else if (!strcmp(key, "WRITEFORMAT_ASCII")) *v = in->ASCII;
  else if (!strcmp(key, "Writecomposition")) *v = in->WRITECOMPOSITION;
  else if (!strcmp(key, "ISOTHERMAL")) *v = in->ISOTHERMAL;
  else if (!strcmp(key, "Noise_phasefield")) *v = in->NOISE_PHASEFIELD;
  else if (!strcmp(key, "n_unknown")) *v = in->n_unknown;
  else if (!strcmp(key, "nfill")) *v = in->nfill;
  else return GP_E_ARG;
  return GP_OK;
}

int gp_input_get_double(const gp_input *in, const char *key, double *v) {
  if (!in || !key || !v) return GP_E_ARG;
  if (!strcmp(key, "DELTA_X")) *v = in->deltax;
  else if (!strcmp(key, "DELTA_Y")) *v = in->deltay;
  else if (!strcmp(key, "DELTA_Z")) *v = in->deltaz;
  else if (!strcmp(key, "DELTA_t")) *v = in->deltat;
  else if (!strcmp(key, "epsilon")) *v = in->epsilon;
  else if (!strcmp(key, "tau")) *v = in->tau;
  else if (!strcmp(key, "T")) *v = in->T;
  else if (!strcmp(key, "Equilibrium_temperature")) *v = in->Teq;
  else if (!strcmp(key, "Filling_temperature")) *v = in->Tfill;
  else return GP_E_ARG;
  return GP_OK;
}

int gp_input_name(const gp_input *in, int which, int index, char *buf, size_t len) {
  if (!in || !buf || len == 0) return GP_E_ARG;
  if (which == 0) {
    if (index < 0 || index >= in->NUMPHASES || index >= PMAX) return GP_E_ARG;
    snprintf(buf, len, "%s", in->Phases[index]);
  } else {
    if (index < 0 || index >= in->NUMCOMPONENTS || index >= KMAX) return GP_E_ARG;
    snprintf(buf, len, "%s", in->Components[index]);
  }
  return GP_OK;
}

/* ------------------------------------------------------------------------- */
/* model constants                                                           */
/* ------------------------------------------------------------------------- */

/* function_F_01_function_B / _C at temperature T (functionF_01.h:62-104),
 * with DELTA_C / DELTA_T of the current init_propertymatrices call. */
static double fB(const gp_input *in, double DT[PMAX][PMAX], double DC[PMAX][KMAX], double T, int i, int a) {
  int N = in->NUMPHASES, K1 = in->NUMCOMPONENTS - 1, k;
  double cl[KMAX], cs[KMAX], sum_c = 0.0, B_ai = 0.0;
  if (a != N - 1) {
    for (k = 0; k < K1; k++) {
      cl[k] = in->ceq[a][N - 1][k] - (DC[a][k]) * (in->Teq - T) / (DT[a][N - 1]);
      cs[k] = in->ceq[a][a][k] - (DC[a][k]) * (in->Teq - T) / (DT[a][a]);
      if (k != i) sum_c += in->A[N - 1][k][i] * cl[k] - in->A[a][k][i] * cs[k];
    }
    B_ai = (2.0 * (in->A[N - 1][i][i] * cl[i] - in->A[a][i][i] * cs[i]) + sum_c);
  }
  return B_ai;
}

static double fC(const gp_input *in, double DT[PMAX][PMAX], double DC[PMAX][KMAX], double T, int a) {
  int N = in->NUMPHASES, K1 = in->NUMCOMPONENTS - 1, i, j, k;
  double cl[KMAX], cs[KMAX], sum_c = 0.0;
  if (a != N - 1) {
    for (k = 0; k < K1; k++) {
      cl[k] = in->ceq[a][N - 1][k] - (DC[a][k]) * (in->Teq - T) / (DT[a][N - 1]);
      cs[k] = in->ceq[a][a][k] - (DC[a][k]) * (in->Teq - T) / (DT[a][a]);
    }
    for (i = 0; i < K1; i++)
      for (j = 0; j < K1; j++)
        if (i <= j) sum_c += (in->A[a][i][j] * cs[i] * cs[j] - in->A[N - 1][i][j] * cl[i] * cl[j]);
  }
  return sum_c;
}

int gp_model_from_input(const gp_input *in, gp_model *m) {
  int N, K1, a, b, c, i, j, k;
  if (!in || !m) return GP_E_ARG;
  N = in->NUMPHASES;
  K1 = in->NUMCOMPONENTS - 1;
  memset(m, 0, sizeof *m);
  if (in->DIMENSION != 2) { gp_set_error("DIMENSION=%d: only the 2D solver is on this path", in->DIMENSION); return GP_E_UNSUPPORTED; }
  if (N < 2 || N > GP_MAX_PHASES) { gp_set_error("NUMPHASES=%d outside 2..%d", N, GP_MAX_PHASES); return GP_E_UNSUPPORTED; }
  if (K1 < 1 || K1 > GP_MAX_K1) { gp_set_error("NUMCOMPONENTS=%d outside 2..%d", K1 + 1, GP_MAX_K1 + 1); return GP_E_UNSUPPORTED; }
  if (in->MESH_X < 4 || in->MESH_Y < 4) { gp_set_error("MESH_X, MESH_Y must be >= 4"); return GP_E_UNSUPPORTED; }
  if (!in->ISOTHERMAL && in->SHIFT) {
    gp_set_error("ISOTHERMAL=0 with Shift=1 (a moving frame under the frozen gradient) is not on this path");
    return GP_E_UNSUPPORTED;
  }
  if (in->FUNCTION_F != 1) { gp_set_error("Function_F=%d: only the quadratic free energy (1) is on this path", in->FUNCTION_F); return GP_E_UNSUPPORTED; }
  if (in->NOISE_PHASEFIELD) { gp_set_error("Noise_phasefield uses rand(); not on this path"); return GP_E_UNSUPPORTED; }
  if (!in->have_gamma || !in->have_tau) { gp_set_error("GAMMA and Tau are required"); return GP_E_PARSE; }
  if (N >= 3 && !in->have_gabc) { gp_set_error("Gamma_abc is required for NUMPHASES >= 3"); return GP_E_PARSE; }
  /* initialize_functions_solverloop.h:16-41 */
  if (in->FUNCTION_W == 1) m->obstacle = 1;
  else if (in->FUNCTION_W == 2) m->obstacle = 0;
  else { gp_set_error("Function_W=%d unsupported", in->FUNCTION_W); return GP_E_UNSUPPORTED; }
  if (in->FUNCTION_ANISOTROPY == 0) m->anisotropy = 0;
  else if (in->FUNCTION_ANISOTROPY == 1) {
    m->anisotropy = 1;
    if (in->FOLD != 4) { gp_set_error("Anisotropy_type=%d: only 4-fold cubic is implemented by the reference", in->FOLD); return GP_E_UNSUPPORTED; }
    if (!in->have_dab) { gp_set_error("dab is required with Function_anisotropy=1"); return GP_E_PARSE; }
    for (a = 0; a < N; a++)
      for (b = 0; b < N; b++)
        if (a != b && !in->have_rot[a][b]) {
          gp_set_error("Rotation_matrix missing for phases %d,%d (the reference would read uninitialised memory)", a, b);
          return GP_E_PARSE;
        }
  } else { gp_set_error("Function_anisotropy=%d unsupported", in->FUNCTION_ANISOTROPY); return GP_E_UNSUPPORTED; }
  if (in->BINARY) m->mu_solver = GP_MU_BINARY;
  else if (in->TERNARY) {
    m->mu_solver = GP_MU_TERNARY;
    if (K1 != 2) { gp_set_error("TERNARY=1 needs NUMCOMPONENTS=3"); return GP_E_UNSUPPORTED; }
  } else if (in->DILUTE) m->mu_solver = GP_MU_DILUTE;
  else m->mu_solver = GP_MU_LU;
  /* boundary_serial.h copies when the current type is 1 or 3, from the proxy
   * rows that BOUNDARY_VALUE assigned for the type seen at that line */
  for (i = 0; i < 4; i++) {
    int f;
    for (f = 0; f < 2; f++) {
      int tcur = in->bc_type[i][f], tprx = in->bc_proxy_type[i][f];
      if (tcur != 1 && tcur != 3) {
        gp_set_error("boundary %d (%s): type %d; only Neumann (1) and periodic (3) are applied by the reference",
                     i, f ? "mu" : "phi", tcur);
        return GP_E_UNSUPPORTED;
      }
      if (tprx != 1 && tprx != 3) {
        gp_set_error("boundary %d (%s): no BOUNDARY_VALUE line after its BOUNDARY line (the reference would copy "
                     "from unassigned proxy rows)", i, f ? "mu" : "phi");
        return GP_E_PARSE;
      }
      if (f == 0) m->bc_phi[i] = tprx; else m->bc_mu[i] = tprx;
    }
  }

  m->N = N; m->K1 = K1;
  m->mesh_x = in->MESH_X; m->mesh_y = in->MESH_Y;
  m->dx = in->deltax; m->dy = in->deltay; m->dt = in->deltat;
  m->epsilon = in->epsilon; m->tau = in->tau;
  m->T = in->T; m->Teq = in->Teq;
  for (a = 0; a < N; a++)
    for (b = 0; b < N; b++) {
      m->Gamma[a][b] = in->Gamma[a][b];
      m->tau_ab[a][b] = in->tau_ab[a][b];
      m->dab[a][b] = in->have_dab ? in->dab[a][b] : 0.0;
      for (i = 0; i < 2; i++)
        for (j = 0; j < 2; j++) {
          m->R[a][b][i][j] = (a != b && m->anisotropy) ? in->Rot[a][b][i][j] : 0.0;
          m->Rinv[a][b][i][j] = (a != b && m->anisotropy) ? in->RotInv[a][b][i][j] : 0.0;
        }
      for (c = 0; c < N; c++) m->Gamma_abc[a][b][c] = in->Gamma_abc[a][b][c];
    }
  /* init_propertymatrices(T), functionF_01.h:169-230 */
  {
    double muc[KMAX * KMAX], cmu[KMAX * KMAX];
    double DT[PMAX][PMAX], DC[PMAX][KMAX], dcbdT[PMAX][PMAX][KMAX], dBbdT[PMAX][KMAX], Beq[PMAX][KMAX];
    memset(DT, 0, sizeof DT); memset(DC, 0, sizeof DC); memset(dcbdT, 0, sizeof dcbdT);
    memset(dBbdT, 0, sizeof dBbdT); memset(Beq, 0, sizeof Beq);
    for (a = 0; a < N; a++) {
      for (i = 0; i < K1; i++)
        for (j = 0; j < K1; j++) muc[i * K1 + j] = (i == j) ? 2.0 * in->A[a][i][j] : in->A[a][i][j];
      host_matinv(muc, cmu, K1);
      for (i = 0; i < K1; i++)
        for (j = 0; j < K1; j++) m->cmu[a][i][j] = cmu[i * K1 + j];
    }
    for (a = 0; a < N - 1; a++) {
      DT[a][N - 1] = 0.0;
      DT[a][a] = 0.0;
      for (k = 0; k < K1; k++) {
        DT[a][a] += in->slopes[a][a][k] * (in->ceq[a][N - 1][k] - in->ceq[a][a][k]);
        DT[a][N - 1] += in->slopes[a][N - 1][k] * (in->ceq[a][N - 1][k] - in->ceq[a][a][k]);
        DC[a][k] = in->ceq[a][N - 1][k] - in->ceq[a][a][k];
      }
      for (k = 0; k < K1; k++) {
        dcbdT[a][a][k] = DC[a][k] / DT[a][a];
        dcbdT[a][N - 1][k] = DC[a][k] / DT[a][N - 1];
      }
      for (k = 0; k < K1; k++) {
        dBbdT[a][k] = 2.0 * (in->A[N - 1][k][k] * dcbdT[a][N - 1][k] - in->A[a][k][k] * dcbdT[a][a][k]);
        for (i = 0; i < K1; i++)
          if (k != i) dBbdT[a][k] += (in->A[N - 1][k][i] * dcbdT[a][N - 1][i] - in->A[a][k][i] * dcbdT[a][a][i]);
      }
    }
    for (k = 0; k < K1; k++) dBbdT[N - 1][k] = 0.0;
    for (a = 0; a < N; a++)
      for (i = 0; i < K1; i++) Beq[a][i] = fB(in, DT, DC, in->Teq, i, a);
    for (a = 0; a < N; a++) {
      for (i = 0; i < K1; i++) m->B[a][i] = fB(in, DT, DC, in->T, i, a);
      m->C[a] = fC(in, DT, DC, in->T, a);
    }
    for (a = 0; a < N; a++)
      for (i = 0; i < K1; i++) {
        m->Beff[a][i] = (Beq[a][i] + dBbdT[a][i] * (in->T - in->Teq));
        m->Bfill[a][i] = (Beq[a][i] + dBbdT[a][i] * (in->Teq - in->Teq));
        m->Beq[a][i] = Beq[a][i];
        m->dBbdT[a][i] = dBbdT[a][i];
        m->ceq_s[a][i] = in->ceq[a][a][i];
        m->ceq_l[a][i] = in->ceq[a][N - 1][i];
        m->dC[a][i] = DC[a][i];
      }
    for (a = 0; a < N; a++) {
      m->dT_s[a] = DT[a][a];
      m->dT_l[a] = DT[a][N - 1];
    }
    if (!in->ISOTHERMAL) {
      /* the T copy of boundary_serial.h (field 2): from the proxy rows when the current type is 1 or 3 */
      for (i = 0; i < 4; i++) {
        const int tcur = in->bc_type[i][2], tprx = in->bc_proxy_type[i][2];
        m->bc_T[i] = (tcur == 1 || tcur == 3) ? ((tprx == 1 || tprx == 3) ? tprx : -1) : 0;
        if (m->bc_T[i] < 0) {
          gp_set_error("boundary %d (T): no BOUNDARY_VALUE line after its BOUNDARY line", i);
          return GP_E_PARSE;
        }
      }
      if (m->bc_T[2] != m->bc_T[3]) {
        gp_set_error("both y sides must share the temperature's boundary type");
        return GP_E_UNSUPPORTED;
      }
      m->nonisothermal = 1;
      m->tg_base = in->tempgrady[0];
      m->tg_deltaT = in->tempgrady[1];
      m->tg_distance = in->tempgrady[2];
      m->tg_offset = in->tempgrady[3];
      m->tg_velocity = in->tempgrady[4];
    }
    /* apply_shiftY's liquid rows, functions/shift.h:24-37 with function_F_01_Mu */
    for (k = 0; k < K1; k++) {
      const int L = N - 1;
      double v = 2.0 * in->A[L][k][k] * in->cfill[L][L][k] + (Beq[L][k] + dBbdT[L][k] * (in->Tfill - in->Teq));
      for (j = 0; j < K1; j++)
        if (k != j) v += in->A[L][k][j] * in->cfill[L][L][j];
      m->mu_shift[k] = v;
    }
  }
  for (a = 0; a < N; a++)
    for (i = 0; i < K1; i++)
      for (j = 0; j < K1; j++) {
        m->A[a][i][j] = in->A[a][i][j];
        m->Diff[a][i][j] = in->Diffusivity[a][i][j];
      }
  m->inv_eps = 1.0 / in->epsilon;
  m->w_obstacle = 16.0 / (M_PI * M_PI);
  m->jat_obst = -0.25 * M_PI * in->epsilon;
  m->jat_well = -1.0 * in->epsilon;
  m->s_well = 0.5 / sqrt(2.0);
  return GP_OK;
}

/* ------------------------------------------------------------------------- */
/* filling                                                                   */
/* ------------------------------------------------------------------------- */

/* One fill of phase b and the liquid re-balance that follows it
 * (fill_domain.h:151-205 -> filling.h:6-52, 117-219).  Works on the ghosted
 * grid coordinates of the reference (x, y in [0, rows)), skipping ghosts. */
static int fill_one(const gp_input *in, const fill_op *op, long b, double *phi, long mx, long my) {
  int N = in->NUMPHASES;
  long x, y, a;
  long rx = mx + 6, ry = my + 6;
  long np = mx * my;
  for (x = 0; x < rx; x++)
    for (y = 0; y < ry; y++) {
      if (x < 3 || y < 3 || x >= rx - 3 || y >= ry - 3) continue; /* ghosts are refilled by the BC copy */
      long id = (x - 3) * my + (y - 3);
      if (b < N - 1) {
        int inside = 0;
        if (op->kind == FILL_CUBE) {
          long xs = op->v[0] + 3, ys = op->v[1] + 3, zs = op->v[2], xe = op->v[3] + 3, ye = op->v[4] + 3, ze = op->v[5];
          inside = (x >= xs) && (x <= xe) && (y >= ys) && (y <= ye) && (0 >= zs) && (0 <= ze);
        } else if (op->kind == FILL_CYLINDER) {
          long xc = op->v[0] + 3, yc = op->v[1] + 3, zs = op->v[2], ze = op->v[3];
          inside = (((x - xc) * (x - xc) + (y - yc) * (y - yc) <= op->r * op->r) && (0 >= zs) && (0 <= ze));
        } else if (op->kind == FILL_SPHERE) {
          long xc = op->v[0] + 3, yc = op->v[1] + 3, zc = op->v[2];
          inside = ((x - xc) * (x - xc) + (y - yc) * (y - yc) + (0 - zc) * (0 - zc) <= op->r * op->r);
        }
        if (inside) {
          phi[b * np + id] = 1.00000;
          for (a = 0; a < N; a++)
            if (a != b) phi[a * np + id] = 0.00000;
        } else if (phi[b * np + id] != 1.0000) {
          phi[b * np + id] = 0.00000;
        }
      } else {
        double sum = 0.0;
        for (a = 0; a < N - 1; a++) sum += phi[a * np + id];
        if (sum > 1.0) {
          phi[b * np + id] = 1.0;
          for (a = 0; a < N - 1; a++)
            if (a != b) phi[a * np + id] = 0.00000;
        } else {
          phi[b * np + id] = 1.0 - sum;
        }
      }
    }
  return GP_OK;
}

int gp_fill(const gp_input *in, const gp_model *m, double *phi, double *mu) {
  int N, K1, f, k, b;
  long mx, my, np, id;
  if (!in || !m || !phi || !mu) return GP_E_ARG;
  N = m->N; K1 = m->K1; mx = m->mesh_x; my = m->mesh_y; np = mx * my;
  memset(phi, 0, sizeof(double) * N * np);
  for (f = 0; f < in->nfill; f++) {
    const fill_op *op = &in->fill[f];
    if (op->kind == FILL_ELLIPSE) {
      gp_set_error("FILLELLIPSE: the reference fills it with an uninitialised rotation angle and a mismatched cell index (filling.h:54-116); not supported");
      return GP_E_UNSUPPORTED;
    }
    fill_one(in, op, op->phase, phi, mx, my);
    fill_one(in, op, N - 1, phi, mx, my);
  }
  /* fill_composition_cube, filling.h:221-270: Mu at Teq of ceq (solid) or cfill (liquid) */
  for (id = 0; id < np; id++) {
    double cc[KMAX];
    int filled = 0;
    for (b = 0; b < N - 1; b++) {
      if (phi[b * np + id] == 1.0) {
        for (k = 0; k < K1; k++) cc[k] = in->ceq[b][b][k];
        filled = 1;
        break;
      }
    }
    if (!filled) {
      b = N - 1;
      for (k = 0; k < K1; k++) cc[k] = in->cfill[N - 1][N - 1][k];
    }
    for (k = 0; k < K1; k++) {
      /* function_F_01_Mu, functionF_01.h:19-29, at T = Teq */
      int j;
      double s = 2.0 * m->A[b][k][k] * cc[k] + m->Bfill[b][k];
      for (j = 0; j < K1; j++)
        if (k != j) s += m->A[b][k][j] * cc[j];
      mu[k * np + id] = s;
    }
  }
  return GP_OK;
}

/* ------------------------------------------------------------------------- */
/* VTK                                                                       */
/* ------------------------------------------------------------------------- */

static double be64(double v) {
  unsigned char b[8], r[8];
  int i;
  memcpy(b, &v, 8);
  for (i = 0; i < 8; i++) r[i] = b[7 - i];
  memcpy(&v, r, 8);
  return v;
}

/* c_a(mu) h_a(phi) summed over phases: the Composition_ field, file_writer.h:203-235 */
/* The frozen gradient's temperature of ghost-padded row gy after step t (microsim_gp.c:77-82,
 * 108-113; functions/Temperature_gradient.h:19), no moving frame. */
static double temp_after(const gp_model *m, long t, long gy) {
  const double shift_offset = 0.0;
  const double base_pos = t == 0 ? (m->tg_offset / m->dy) - shift_offset
                                 : (m->tg_offset / m->dy) - shift_offset + ((m->tg_velocity / m->dy) * ((double)t * m->dt));
  const double grad = (m->tg_deltaT) * m->dy / (m->tg_distance);
  const double bottom = m->tg_base - base_pos * grad;
  return bottom + (double)gy * grad;
}

/* sum_a c_a(mu, T) h_a(phi) (file_writer.h:115-133); T only for a non-isothermal model */
static double composition(const gp_model *m, const double *ph, const double *mu, int k, double T) {
  int a, b2, c2, l, N = m->N, K1 = m->K1;
  double comp = 0.0;
  for (a = 0; a < N; a++) {
    double cm = 0.0, h, s1 = 0.0;
    for (l = 0; l < K1; l++)
      cm += m->cmu[a][k][l] *
            (mu[l] - (m->nonisothermal ? (m->Beq[a][l] + m->dBbdT[a][l] * (T - m->Teq)) : m->Beff[a][l]));
    h = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a];
    for (b2 = 0; b2 < N; b2++)
      for (c2 = b2 + 1; c2 < N; c2++)
        if (b2 != a && c2 != a) s1 += ph[b2] * ph[c2];
    s1 *= 2.0 * ph[a];
    comp += cm * (h + s1);
  }
  return comp;
}

int gp_write_vtk(const gp_input *in, const gp_model *m, const char *path, const double *phi, const double *mu) {
  return gp_write_vtk_t(in, m, path, phi, mu, 0);
}

int gp_write_vtk_t(const gp_input *in, const gp_model *m, const char *path, const double *phi, const double *mu,
                   int64_t tstep) {
  FILE *fp;
  long mx, my, np, x, y;
  int a, k;
  if (!in || !m || !path || !phi || !mu) return GP_E_ARG;
  mx = m->mesh_x; my = m->mesh_y; np = mx * my;
  fp = fopen(path, in->ASCII ? "w" : "wb");
  if (!fp) { gp_set_error("cannot write %s", path); return GP_E_IO; }
  fprintf(fp, "# vtk DataFile Version 3.0\n");
  fprintf(fp, "Microsim_fields\n");
  fprintf(fp, in->ASCII ? "ASCII\n" : "BINARY\n");
  fprintf(fp, "DATASET STRUCTURED_POINTS\n");
  fprintf(fp, "DIMENSIONS %ld %ld %ld\n", my, mx, (long)1);
  fprintf(fp, "ORIGIN 0 0 0\n");
  fprintf(fp, "SPACING %le %le %le\n", in->deltax, in->deltay, in->deltaz);
  fprintf(fp, "POINT_DATA %ld\n", (long)mx * (long)my);
  for (a = 0; a < m->N; a++) {
    fprintf(fp, "SCALARS %s double 1\n", in->Phases[a]);
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (x = 0; x < mx; x++)
      for (y = 0; y < my; y++) {
        double v = phi[a * np + x * my + y];
        if (in->ASCII) fprintf(fp, "%le\n", v);
        else { v = be64(v); fwrite(&v, sizeof(double), 1, fp); }
      }
    if (in->ASCII) fprintf(fp, "\n");
  }
  for (k = 0; k < m->K1; k++) {
    fprintf(fp, "SCALARS Mu_%s double 1\n", in->Components[k]);
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (x = 0; x < mx; x++)
      for (y = 0; y < my; y++) {
        double v = mu[k * np + x * my + y];
        if (in->ASCII) fprintf(fp, "%le\n", v);
        else { v = be64(v); fwrite(&v, sizeof(double), 1, fp); }
      }
    if (in->ASCII) fprintf(fp, "\n");
  }
  if (in->WRITECOMPOSITION) {
    for (k = 0; k < m->K1; k++) {
      fprintf(fp, "SCALARS Composition_%s double 1\n", in->Components[k]);
      fprintf(fp, "LOOKUP_TABLE default\n");
      for (x = 0; x < mx; x++)
        for (y = 0; y < my; y++) {
          double ph[GP_MAX_PHASES], mm[GP_MAX_K1], v;
          int l;
          for (l = 0; l < m->N; l++) ph[l] = phi[l * np + x * my + y];
          for (l = 0; l < m->K1; l++) mm[l] = mu[l * np + x * my + y];
          v = composition(m, ph, mm, k, m->nonisothermal ? temp_after(m, (long)tstep, y + 3) : m->T);
          if (in->ASCII) fprintf(fp, "%le \n", v);
          else { v = be64(v); fwrite(&v, sizeof(double), 1, fp); }
        }
      if (in->ASCII) fprintf(fp, "\n");
    }
  }
  if (m->nonisothermal) { /* file_writer.h:138-150 / 238-253: the cells' temperature after step tstep */
    fprintf(fp, "SCALARS Temperature double 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (x = 0; x < mx; x++)
      for (y = 0; y < my; y++) {
        double v = temp_after(m, (long)tstep, y + 3);
        if (in->ASCII) fprintf(fp, "%le \n", v);
        else { v = be64(v); fwrite(&v, sizeof(double), 1, fp); }
      }
  }
  if (fclose(fp) != 0) return GP_E_IO;
  return GP_OK;
}

/* skip one header line like fscanf("%*[^\n]\n") (which also eats leading
 * blanks of what follows, a quirk the binary reader inherits) */
static void skip_line(FILE *fp) {
  int ch;
  while ((ch = fgetc(fp)) != EOF && ch != '\n') {}
  while ((ch = fgetc(fp)) != EOF && isspace(ch)) {}
  if (ch != EOF) ungetc(ch, fp);
}

int gp_read_vtk(const gp_input *in, const gp_model *m, const char *path, double *phi, double *mu) {
  FILE *fp;
  long mx, my, np, x, y;
  int a, k, i;
  if (!in || !m || !path || !phi || !mu) return GP_E_ARG;
  mx = m->mesh_x; my = m->mesh_y; np = mx * my;
  fp = fopen(path, in->ASCII ? "r" : "rb");
  if (!fp) { gp_set_error("cannot read %s", path); return GP_E_IO; }
  for (i = 0; i < 8; i++) skip_line(fp);
  for (a = 0; a < m->N + m->K1; a++) {
    double *dst = a < m->N ? phi + (long)a * np : mu + (long)(a - m->N) * np;
    skip_line(fp);
    skip_line(fp);
    for (x = 0; x < mx; x++)
      for (y = 0; y < my; y++) {
        double v;
        if (in->ASCII) {
          /* fscanf("%le \n") of the reference: the number, then all whitespace */
          if (fscanf(fp, "%le ", &v) != 1) { fclose(fp); return GP_E_PARSE; }
        } else {
          if (fread(&v, sizeof(double), 1, fp) != 1) { fclose(fp); return GP_E_IO; }
          v = be64(v);
        }
        dst[x * my + y] = v;
      }
  }
  (void)k;
  fclose(fp);
  return GP_OK;
}
