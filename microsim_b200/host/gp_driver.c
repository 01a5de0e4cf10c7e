/*
 * gp_driver.c -- `microsim_gp_b200 Input.in Filling.in Out [fp64|fp32]`
 *
 * Drop-in for the reference's CLI driver (Grand_potential_Finite_difference_2D_serial/
 * microsim_gp.c:41-151): same arguments, same DATA/<Out>_<t>.vtk files every
 * SAVET steps, same DATA/shift.dat lines and the same progress lines every
 * TRACK_PROGRESS steps, with the time loop running on the GPU through the C ABI.
 * The optional fourth argument (or GP_PRECISION=fp32) selects the FP32 form.
 *
 * Differences, stated: the progress extrema are sampled when they are printed
 * (the reference updates them every step, ghost rings included); with fp32
 * the first step after a moving-frame shift reads ghost rows through the
 * boundary map (fp64 reproduces the reference's shifted ghost rows); a restart
 * (STARTTIME > 0) under a frozen temperature gradient is rejected with a
 * message.
 *
 * `microsim_gp_b200 --batch list.txt` (no counterpart in the reference, which
 * runs one simulation per process) runs many simulations as one FP32 batch: each
 * line of list.txt is `<directory> <Input.in> <Filling.in> <Out>` (input paths
 * relative to the directory), every instance writes its own
 * <directory>/DATA/<Out>_<t>.vtk every SAVET of its own steps up to its own
 * NTIMESTEPS, and prints its progress lines every TRACK_PROGRESS steps after a
 * "[<directory>]" line.  The instances share NUMPHASES and NUMCOMPONENTS; no
 * moving frame, no restart.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "gp_b200.h"

static int fail(const char *what, int rc) {
  fprintf(stderr, "microsim_gp_b200: %s failed (%d): %s\n", what, rc, gp_last_error());
  return 1;
}

/* One simulation of a batch run. */
typedef struct {
  char dir[512], out[256];
  gp_input *in;
  gp_model m;
  int64_t ntimesteps, saveT, track;
  double *phi, *mu;
} job_t;

/* The progress block of one instance (microsim_gp.c:137-147's lines, after a "[<directory>]" line). */
static int batch_progress(gp_batch *b, int i, const job_t *j, int64_t t) {
  gp_stats st;
  int rc = gp_batch_get_stats(b, i, &st);
  if (rc != GP_OK && rc != GP_E_NONFINITE) return fail("gp_batch_get_stats", rc);
  char pname[GP_MAX_PHASES][GP_NAME_LEN], cname[GP_MAX_K1][GP_NAME_LEN];
  int max_length = 0, a, k;
  for (a = 0; a < j->m.N; a++) {
    gp_input_name(j->in, 0, a, pname[a], GP_NAME_LEN);
    if ((int)strlen(pname[a]) > max_length) max_length = (int)strlen(pname[a]);
  }
  for (k = 0; k < j->m.K1; k++) {
    gp_input_name(j->in, 1, k, cname[k], GP_NAME_LEN);
    if ((int)strlen(cname[k]) > max_length) max_length = (int)strlen(cname[k]);
  }
  double dt;
  gp_input_get_double(j->in, "DELTA_t", &dt);
  fprintf(stdout, "[%s]\nTime=%le\n", j->dir, t * dt);
  for (a = 0; a < j->m.N; a++)
    fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, pname[a], st.phi_max[a],
            st.phi_min[a], sqrt(st.rel_change_phi[a]));
  for (k = 0; k < j->m.K1; k++)
    fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, cname[k], st.mu_max[k],
            st.mu_min[k], sqrt(st.rel_change_mu[k]));
  fprintf(stdout, "\n");
  if (rc == GP_E_NONFINITE) {
    fprintf(stderr, "microsim_gp_b200: %s: non-finite values at t=%lld (unstable DELTA_t?)\n", j->dir, (long long)t);
    return 3;
  }
  return 0;
}

static int run_batch(const char *list) {
  FILE *lf = fopen(list, "r");
  if (!lf) {
    fprintf(stderr, "microsim_gp_b200: cannot read %s\n", list);
    return 2;
  }
  job_t *jobs = NULL;
  int n = 0, cap = 0, rc;
  char line[2048], ip[1100], fp[1100];
  while (fgets(line, sizeof line, lf)) {
    char d[512], i1[256], f1[256], o[256];
    if (sscanf(line, "%511s %255s %255s %255s", d, i1, f1, o) != 4 || d[0] == '#') continue;
    if (n == cap) {
      cap = cap ? 2 * cap : 16;
      job_t *nj = (job_t *)realloc(jobs, sizeof(job_t) * cap);
      if (!nj) return fail("host allocation", GP_E_NOMEM);
      jobs = nj;
    }
    job_t *j = &jobs[n];
    memset(j, 0, sizeof *j);
    snprintf(j->dir, sizeof j->dir, "%s", d);
    snprintf(j->out, sizeof j->out, "%s", o);
    snprintf(ip, sizeof ip, "%s/%s", d, i1);
    snprintf(fp, sizeof fp, "%s/%s", d, f1);
    if ((rc = gp_input_read(ip, fp, &j->in)) != GP_OK) return fail("reading inputs", rc);
    if ((rc = gp_model_from_input(j->in, &j->m)) != GP_OK) return fail("model constants", rc);
    int64_t nsmooth = 0, starttime = 0, restart = 0, shift = 0;
    gp_input_get_long(j->in, "NTIMESTEPS", &j->ntimesteps);
    gp_input_get_long(j->in, "SAVET", &j->saveT);
    gp_input_get_long(j->in, "NSMOOTH", &nsmooth);
    gp_input_get_long(j->in, "STARTTIME", &starttime);
    gp_input_get_long(j->in, "RESTART", &restart);
    gp_input_get_long(j->in, "Shift", &shift);
    gp_input_get_long(j->in, "TRACK_PROGRESS", &j->track);
    if (j->saveT <= 0) j->saveT = j->ntimesteps > 0 ? j->ntimesteps : 1;
    if (shift || starttime || restart) {
      fprintf(stderr, "microsim_gp_b200: %s: a moving frame or a restart is not available in a batch\n", ip);
      return 2;
    }
    const size_t np = (size_t)j->m.mesh_x * (size_t)j->m.mesh_y;
    j->phi = (double *)malloc(sizeof(double) * np * j->m.N);
    j->mu = (double *)malloc(sizeof(double) * np * j->m.K1);
    if (!j->phi || !j->mu) return fail("host allocation", GP_E_NOMEM);
    if ((rc = gp_fill(j->in, &j->m, j->phi, j->mu)) != GP_OK) return fail("filling", rc);
    char name[1400];
    snprintf(name, sizeof name, "%s/DATA", d);
    mkdir(name, 0777);
    snprintf(name, sizeof name, "%s/DATA/%s_0.vtk", d, o);
    if ((rc = gp_write_vtk(j->in, &j->m, name, j->phi, j->mu)) != GP_OK) return fail("vtk write", rc);
    if (nsmooth > 1) { /* the smoothing pre-steps in FP64, as for a single fp32 run */
      gp_ctx *pre = NULL;
      if ((rc = gp_create(&j->m, GP_FP64, &pre)) != GP_OK) return fail("gp_create", rc);
      if ((rc = gp_upload(pre, j->phi, j->mu)) != GP_OK) return fail("gp_upload", rc);
      if ((rc = gp_smooth(pre, nsmooth - 1)) != GP_OK) return fail("gp_smooth", rc);
      if ((rc = gp_download(pre, j->phi, j->mu)) != GP_OK) return fail("gp_download", rc);
      gp_destroy(pre);
    }
    n++;
  }
  fclose(lf);
  if (n == 0) {
    fprintf(stderr, "microsim_gp_b200: %s lists no simulation\n", list);
    return 2;
  }
  gp_model *models = (gp_model *)malloc(sizeof(gp_model) * n);
  if (!models) return fail("host allocation", GP_E_NOMEM);
  int64_t tmax = 0;
  for (int i = 0; i < n; i++) {
    models[i] = jobs[i].m;
    if (jobs[i].ntimesteps > tmax) tmax = jobs[i].ntimesteps;
  }
  gp_batch *b = NULL;
  if ((rc = gp_batch_create(models, n, &b)) != GP_OK) return fail("gp_batch_create", rc);
  for (int i = 0; i < n; i++)
    if ((rc = gp_batch_upload(b, i, jobs[i].phi, jobs[i].mu)) != GP_OK) return fail("gp_batch_upload", rc);
  int tx, ty;
  if ((rc = gp_batch_autotune(b, NULL, &tx, &ty)) != GP_OK) return fail("gp_batch_autotune", rc);
  int64_t t = 0;
  while (t < tmax) {
    int64_t next = tmax; /* the next step some instance writes or prints at */
    for (int i = 0; i < n; i++) {
      const int64_t ns = (t / jobs[i].saveT + 1) * jobs[i].saveT;
      if (ns <= jobs[i].ntimesteps && ns < next) next = ns;
      if (jobs[i].track > 0) {
        const int64_t nt = (t / jobs[i].track + 1) * jobs[i].track;
        if (nt <= jobs[i].ntimesteps && nt < next) next = nt;
      }
    }
    if ((rc = gp_batch_step(b, next - t)) != GP_OK) return fail("gp_batch_step", rc);
    t = next;
    for (int i = 0; i < n; i++) {
      if (t <= jobs[i].ntimesteps && jobs[i].track > 0 && t % jobs[i].track == 0) {
        const int prc = batch_progress(b, i, &jobs[i], t);
        if (prc) return prc;
      }
      if (t > jobs[i].ntimesteps || t % jobs[i].saveT != 0) continue;
      char name[1400];
      if ((rc = gp_batch_download(b, i, jobs[i].phi, jobs[i].mu)) != GP_OK) return fail("gp_batch_download", rc);
      snprintf(name, sizeof name, "%s/DATA/%s_%lld.vtk", jobs[i].dir, jobs[i].out, (long long)t);
      if ((rc = gp_write_vtk_t(jobs[i].in, &jobs[i].m, name, jobs[i].phi, jobs[i].mu, t)) != GP_OK)
        return fail("vtk write", rc);
    }
  }
  if ((rc = gp_batch_sync(b)) != GP_OK) return fail("gp_batch_sync", rc);
  gp_batch_destroy(b);
  for (int i = 0; i < n; i++) {
    gp_input_free(jobs[i].in);
    free(jobs[i].phi);
    free(jobs[i].mu);
  }
  free(jobs);
  free(models);
  return 0;
}

int main(int argc, char *argv[]) {
  if (argc == 3 && !strcmp(argv[1], "--batch")) return run_batch(argv[2]);
  gp_input *in = NULL;
  gp_model m;
  gp_ctx *ctx = NULL;
  int64_t ntimesteps, saveT, nsmooth, starttime, restart, track, shift;
  int precision = GP_FP64;
  int rc;
  if (argc < 4) {
    fprintf(stderr, "usage: %s Input.in Filling.in Out [fp64|fp32]\n       %s --batch list.txt\n", argv[0],
            argv[0]);
    return 2;
  }
  if ((argc > 4 && !strcmp(argv[4], "fp32")) || (getenv("GP_PRECISION") && !strcmp(getenv("GP_PRECISION"), "fp32")))
    precision = GP_FP32;
  mkdir("DATA", 0777);
  if ((rc = gp_input_read(argv[1], argv[2], &in)) != GP_OK) return fail("reading inputs", rc);
  if ((rc = gp_model_from_input(in, &m)) != GP_OK) return fail("model constants", rc);
  gp_input_get_long(in, "NTIMESTEPS", &ntimesteps);
  gp_input_get_long(in, "SAVET", &saveT);
  gp_input_get_long(in, "NSMOOTH", &nsmooth);
  gp_input_get_long(in, "STARTTIME", &starttime);
  gp_input_get_long(in, "RESTART", &restart);
  gp_input_get_long(in, "TRACK_PROGRESS", &track);
  gp_input_get_long(in, "Shift", &shift);
  int64_t shiftj = 0, shift_offset = 0, shift_position = 0;
  gp_input_get_long(in, "Shiftj", &shiftj);
  if (saveT <= 0) saveT = ntimesteps > 0 ? ntimesteps : 1;
  const size_t np = (size_t)m.mesh_x * (size_t)m.mesh_y;
  double *phi = (double *)malloc(sizeof(double) * np * m.N);
  double *mu = (double *)malloc(sizeof(double) * np * m.K1);
  if (!phi || !mu) return fail("host allocation", GP_E_NOMEM);
  char name[1200];
  if (starttime == 0 && restart == 0) {
    if ((rc = gp_fill(in, &m, phi, mu)) != GP_OK) return fail("filling", rc);
  } else {
    /* microsim_gp.c:55-66: a restarted moving frame continues from DATA/shift.dat */
    FILE *sf = shift ? fopen("DATA/shift.dat", "r") : NULL;
    if (sf) {
      long tf, pf;
      for (int64_t it = 0; it <= starttime / saveT; it++)
        if (fscanf(sf, "%ld %ld\n", &tf, &pf) == 2) shift_position = pf;
      fclose(sf);
    }
    snprintf(name, sizeof name, "DATA/%s_%lld.vtk", argv[3], (long long)starttime);
    if ((rc = gp_read_vtk(in, &m, name, phi, mu)) != GP_OK) return fail("restart read", rc);
  }
  if (m.nonisothermal && starttime > 0) {
    /* microsim_gp.c:68-74 moves gradient_OFFSET on a restart; not on this path */
    fprintf(stderr, "microsim_gp_b200: a restart (STARTTIME > 0) under a frozen temperature gradient is not supported\n");
    return 2;
  }
  if ((rc = gp_create(&m, precision, &ctx)) != GP_OK) return fail("gp_create", rc);
  if ((rc = gp_upload(ctx, phi, mu)) != GP_OK) return fail("gp_upload", rc);
  if (restart == 0 || starttime == 0) {
    snprintf(name, sizeof name, "DATA/%s_%lld.vtk", argv[3], (long long)0);
    if ((rc = gp_write_vtk(in, &m, name, phi, mu)) != GP_OK) return fail("vtk write", rc);
  }
  /* microsim_gp.c:96-100: NSMOOTH - 1 smoothing pre-steps after the first file,
   * in FP64 on the filled doubles whatever the precision of the time loop */
  if (nsmooth > 1 && precision == GP_FP64) {
    if ((rc = gp_smooth(ctx, nsmooth - 1)) != GP_OK) return fail("gp_smooth", rc);
  } else if (nsmooth > 1) {
    gp_ctx *pre = NULL;
    if ((rc = gp_create(&m, GP_FP64, &pre)) != GP_OK) return fail("gp_create", rc);
    if ((rc = gp_upload(pre, phi, mu)) != GP_OK) return fail("gp_upload", rc);
    if ((rc = gp_smooth(pre, nsmooth - 1)) != GP_OK) return fail("gp_smooth", rc);
    if ((rc = gp_download(pre, phi, mu)) != GP_OK) return fail("gp_download", rc);
    gp_destroy(pre);
    if ((rc = gp_upload(ctx, phi, mu)) != GP_OK) return fail("gp_upload", rc);
  }
  int max_length = 0, a, k;
  char pname[GP_MAX_PHASES][GP_NAME_LEN], cname[GP_MAX_K1][GP_NAME_LEN];
  for (a = 0; a < m.N; a++) {
    gp_input_name(in, 0, a, pname[a], GP_NAME_LEN);
    if ((int)strlen(pname[a]) > max_length) max_length = (int)strlen(pname[a]);
  }
  for (k = 0; k < m.K1; k++) {
    gp_input_name(in, 1, k, cname[k], GP_NAME_LEN);
    if ((int)strlen(cname[k]) > max_length) max_length = (int)strlen(cname[k]);
  }
  int64_t t = 0;
  while (t < ntimesteps) {
    /* advance to the next step that writes or prints (microsim_gp.c:129-148) */
    int64_t next = ntimesteps;
    int64_t ns = (t / saveT + 1) * saveT;
    if (ns < next) next = ns;
    if (track > 0) {
      int64_t nt = (t / track + 1) * track;
      if (nt < next) next = nt;
    }
    if (shift) {
      int64_t nh = (t / 100 + 1) * 100;
      if (nh < next) next = nh;
    }
    if ((rc = gp_step(ctx, next - t)) != GP_OK) return fail("gp_step", rc);
    t = next;
    /* microsim_gp.c:115-125: the moving frame, every 100 steps */
    if (shift && t % 100 == 0) {
      int64_t pos = 0;
      if ((rc = gp_interface_y(ctx, &pos)) != GP_OK) return fail("gp_interface_y", rc);
      if (pos > shiftj) {
        if ((rc = gp_shift_y(ctx, pos - shiftj)) != GP_OK) return fail("gp_shift_y", rc);
        shift_offset += pos - shiftj;
      }
    }
    if (t % saveT == 0) {
      if ((rc = gp_download(ctx, phi, mu)) != GP_OK) return fail("gp_download", rc);
      snprintf(name, sizeof name, "DATA/%s_%lld.vtk", argv[3], (long long)(t + starttime));
      if ((rc = gp_write_vtk_t(in, &m, name, phi, mu, t)) != GP_OK) return fail("vtk write", rc);
      FILE *fp = fopen("DATA/shift.dat", "a");
      if (fp) {
        fprintf(fp, "%ld %ld\n", (long)(t + starttime), (long)(shift_offset + shift_position));
        fclose(fp);
      }
    }
    if (track > 0 && t % track == 0) {
      gp_stats st;
      rc = gp_get_stats(ctx, &st);
      if (rc != GP_OK && rc != GP_E_NONFINITE) return fail("gp_get_stats", rc);
      double dt;
      gp_input_get_double(in, "DELTA_t", &dt);
      fprintf(stdout, "Time=%le\n", t * dt);
      for (a = 0; a < m.N; a++)
        fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, pname[a], st.phi_max[a],
                st.phi_min[a], sqrt(st.rel_change_phi[a]));
      for (k = 0; k < m.K1; k++)
        fprintf(stdout, "%*s, Max = %le, Min = %le, Relative_Change=%le\n", max_length, cname[k], st.mu_max[k],
                st.mu_min[k], sqrt(st.rel_change_mu[k]));
      fprintf(stdout, "\n");
      if (rc == GP_E_NONFINITE) {
        fprintf(stderr, "microsim_gp_b200: non-finite values at t=%lld (unstable DELTA_t?)\n", (long long)t);
        return 3;
      }
    }
  }
  if ((rc = gp_sync(ctx)) != GP_OK) return fail("gp_sync", rc);
  gp_destroy(ctx);
  gp_input_free(in);
  free(phi);
  free(mu);
  return 0;
}
