// Finite-difference check of the hand-written reverses in
// microsim_b200/csrc/gp_adjoint_cell.cuh, compiled for the host by
// tests/test_adjoint_local.py.  Prints one line per check:
//   <name> <max relative error over inputs> <number of inputs>
// Relative error of the vector-Jacobian product against central differences
// (step 1e-6 relative), scaled by the largest term.
#define GP_HD inline
#include <stdio.h>
#include <stdlib.h>
#include <math.h>

#include "gp_adjoint_cell.cuh"

using namespace gpadj;
typedef AM<double> Mdl;

static double urand(double a, double b) { return a + (b - a) * (double)rand() / (double)RAND_MAX; }

static Mdl model(int obstacle, double Ds) {
  Mdl m;
  m.dx = 1.0; m.dy = 1.0; m.dt = 0.05; m.eps = 4.0; m.inv_eps = 0.25;
  m.mob = 1.0 / 1.7776; m.tau_ratio = 1.3;
  m.gam = 1.1; m.dab = 0.03;
  m.wobs = 16.0 / (M_PI * M_PI);
  m.jscale = obstacle ? -0.25 * M_PI * 4.0 : -4.0;
  m.swell = 0.5 / sqrt(2.0);
  const double th[2] = {0.26, -0.4};
  for (int a = 0; a < 2; a++) {
    const double c = cos(th[a]), s = sin(th[a]);
    m.R[a][0][0] = c; m.R[a][0][1] = -s; m.R[a][1][0] = s; m.R[a][1][1] = c;
    m.Ri[a][0][0] = c; m.Ri[a][0][1] = s; m.Ri[a][1][0] = -s; m.Ri[a][1][1] = c;
  }
  m.A[0] = 1.0; m.A[1] = 0.8;
  for (int a = 0; a < 2; a++) m.cmu[a] = 1.0 / (2.0 * m.A[a]);
  m.B[0] = -0.2; m.B[1] = 0.05; m.C[0] = 0.01; m.C[1] = 0.0;
  m.Beff[0] = -0.3; m.Beff[1] = 0.15;
  m.Ds = Ds; m.Dl = 1.2;
  m.obstacle = obstacle;
  m.skip_row = -100;
  return m;
}

static double* par_ptr(Mdl& m, int p) {
  switch (p) {
    case P_MOB: return &m.mob;
    case P_DELTA: return &m.dab;
    case P_GAMMA: return &m.gam;
    default: return &m.Dl;
  }
}

static void report(const char* name, double err, int n) { printf("%s %.3e %d\n", name, err, n); }

// -------------------------------------------------------------- Delta-phi of a cell
static double dphi_dot(const Mdl& m, const double (&P)[3][3][2], double mu, const double (&w)[2]) {
  double dp[2];
  dphi_fwd(m, P, mu, dp);
  return w[0] * dp[0] + w[1] * dp[1];
}

static void check_dphi(int obstacle, int trials) {
  double worst = 0.0;
  int n = 0;
  for (int t = 0; t < trials; t++) {
    Mdl m = model(obstacle, 0.0);
    double P[3][3][2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        const double p0 = urand(0.15, 0.85);
        P[i][j][0] = p0;
        P[i][j][1] = 1.0 - p0 + urand(-0.02, 0.02);
      }
    const double mu = urand(-0.3, 0.3);
    const double w[2] = {urand(-1, 1), urand(-1, 1)};
    double LP[3][3][2] = {}, lmu = 0.0, lpar[NPARAM] = {0, 0, 0, 0};
    dphi_rev(m, P, mu, w, LP, lmu, lpar);
    double scale = 1e-30, e = 0.0;
    double fd[3][3][2], fdmu, fdp[NPARAM];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int a = 0; a < 2; a++) {
          const double h = 1e-6;
          double Pp[3][3][2], Pm[3][3][2];
          for (int x = 0; x < 18; x++) { ((double*)Pp)[x] = ((double*)P)[x]; ((double*)Pm)[x] = ((double*)P)[x]; }
          Pp[i][j][a] += h; Pm[i][j][a] -= h;
          fd[i][j][a] = (dphi_dot(m, Pp, mu, w) - dphi_dot(m, Pm, mu, w)) / (2 * h);
          scale = fmax(scale, fabs(fd[i][j][a]));
        }
    {
      const double h = 1e-6;
      fdmu = (dphi_dot(m, P, mu + h, w) - dphi_dot(m, P, mu - h, w)) / (2 * h);
      scale = fmax(scale, fabs(fdmu));
    }
    for (int p = 0; p < NPARAM; p++) {
      Mdl mp = m, mm = m;
      const double h = 1e-6 * fmax(fabs(*par_ptr(mp, p)), 1e-3);
      *par_ptr(mp, p) += h; *par_ptr(mm, p) -= h;
      fdp[p] = (dphi_dot(mp, P, mu, w) - dphi_dot(mm, P, mu, w)) / (2 * h);
      scale = fmax(scale, fabs(fdp[p]));
    }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int a = 0; a < 2; a++) e = fmax(e, fabs(fd[i][j][a] - LP[i][j][a]));
    e = fmax(e, fabs(fdmu - lmu));
    for (int p = 0; p < NPARAM; p++) e = fmax(e, fabs(fdp[p] - lpar[p]));
    worst = fmax(worst, e / scale);
    n += 18 + 1 + NPARAM;
  }
  report(obstacle ? "dphi_obstacle" : "dphi_well", worst, n);
}

// projection branches: states whose unprojected step leaves [0, 1]
static void check_dphi_projection(int trials) {
  double worst = 0.0;
  int n = 0, hits = 0;
  for (int t = 0; t < trials; t++) {
    Mdl m = model(1, 0.0);
    m.mob *= 40.0;  // large steps push phi + dp out of [0, 1]
    double P[3][3][2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        const double p0 = urand(0.0, 1.0);
        P[i][j][0] = p0;
        P[i][j][1] = 1.0 - p0;
      }
    P[1][1][0] = urand(0.01, 0.08);
    P[1][1][1] = 1.0 - P[1][1][0] + urand(-0.01, 0.01);
    const double mu = urand(-0.3, 0.3);
    const double w[2] = {urand(-1, 1), urand(-1, 1)};
    double dp[2];
    dphi_fwd(m, P, mu, dp);
    if (P[1][1][0] + dp[0] <= 0.0 || P[1][1][1] + dp[1] <= 0.0 || P[1][1][0] + dp[0] >= 1.0) hits++;
    double LP[3][3][2] = {}, lmu = 0.0, lpar[NPARAM] = {0, 0, 0, 0};
    dphi_rev(m, P, mu, w, LP, lmu, lpar);
    double scale = 1e-30, e = 0.0;
    for (int x = 0; x < 18; x++) {
      const double h = 1e-7;
      double Pp[3][3][2], Pm[3][3][2];
      for (int y = 0; y < 18; y++) { ((double*)Pp)[y] = ((double*)P)[y]; ((double*)Pm)[y] = ((double*)P)[y]; }
      ((double*)Pp)[x] += h; ((double*)Pm)[x] -= h;
      const double fd = (dphi_dot(m, Pp, mu, w) - dphi_dot(m, Pm, mu, w)) / (2 * h);
      scale = fmax(scale, fabs(fd));
      e = fmax(e, fabs(fd - ((double*)LP)[x]));
    }
    worst = fmax(worst, e / scale);
    n += 18;
  }
  report("dphi_projection", worst, n);
  printf("projection_cases %d %d\n", hits, trials);
}

// -------------------------------------------------------------- faces
static Face<double> rand_face() {
  Face<double> f;
  for (int a = 0; a < 2; a++) {
    f.pc[a] = urand(0.1, 0.9);
    f.pn[a] = urand(0.1, 0.9);
    f.tc[a] = urand(-0.3, 0.3);
    f.tn[a] = urand(-0.3, 0.3);
  }
  f.muc = urand(-0.3, 0.3); f.mun = urand(-0.3, 0.3);
  f.dpc = urand(-0.05, 0.05); f.dpn = urand(-0.05, 0.05);
  f.h = 1.0;
  f.skip = false;
  return f;
}

static double* face_in(Face<double>& f, int i) {
  double* v[14] = {&f.pc[0], &f.pc[1], &f.pn[0], &f.pn[1], &f.tc[0], &f.tc[1], &f.tn[0], &f.tn[1],
                   &f.muc, &f.mun, &f.dpc, &f.dpn, nullptr, nullptr};
  return v[i];
}
static double face_adj(const FaceAdj<double>& L, int i) {
  const double v[12] = {L.pc[0], L.pc[1], L.pn[0], L.pn[1], L.tc[0], L.tc[1], L.tn[0], L.tn[1],
                        L.muc, L.mun, L.dpc, L.dpn};
  return v[i];
}

static void check_face(int which, int obstacle, int trials) {
  double worst = 0.0;
  int n = 0;
  for (int t = 0; t < trials; t++) {
    Mdl m = model(obstacle, 0.3);
    Face<double> f = rand_face();
    const double w = urand(-1, 1);
    FaceAdj<double> L = {};
    double lpar[NPARAM] = {0, 0, 0, 0};
    if (which == 0) fface_rev(m, f, w, L, lpar);
    else jface_rev(m, f, w, L, lpar);
    double scale = 1e-30, e = 0.0;
    for (int i = 0; i < 12; i++) {
      Face<double> fp = f, fm = f;
      const double h = 1e-6;
      *face_in(fp, i) += h; *face_in(fm, i) -= h;
      const double fd = w * ((which == 0 ? fface(m, fp) : jface(m, fp)) - (which == 0 ? fface(m, fm) : jface(m, fm))) / (2 * h);
      scale = fmax(scale, fabs(fd));
      e = fmax(e, fabs(fd - face_adj(L, i)));
    }
    {
      Mdl mp = m, mm = m;
      const double h = 1e-6;
      mp.Dl += h; mm.Dl -= h;
      const double fd = w * ((which == 0 ? fface(mp, f) : jface(mp, f)) - (which == 0 ? fface(mm, f) : jface(mm, f))) / (2 * h);
      scale = fmax(scale, fabs(fd));
      e = fmax(e, fabs(fd - lpar[P_DLIQ]));
    }
    worst = fmax(worst, e / scale);
    n += 13;
  }
  report(which == 0 ? "face_diffusion" : (obstacle ? "face_antitrapping_obstacle" : "face_antitrapping_well"), worst,
         n);
}

// -------------------------------------------------------------- cell update
static void check_mu(int bulk, int trials) {
  double worst = 0.0;
  int n = 0;
  for (int t = 0; t < trials; t++) {
    Mdl m = model(1, 0.0);
    double ph[2], dp[2], F[4], J[4];
    if (bulk) { ph[0] = 0.0; ph[1] = 1.0; }
    else { ph[0] = urand(0.1, 0.9); ph[1] = 1.0 - ph[0] + urand(-0.01, 0.01); }
    for (int a = 0; a < 2; a++) dp[a] = urand(-0.05, 0.05);
    for (int k = 0; k < 4; k++) { F[k] = urand(-0.2, 0.2); J[k] = urand(-0.2, 0.2); }
    const double mu = urand(-0.3, 0.3), w = urand(-1, 1);
    double lph[2] = {0, 0}, lmu = 0, ldp[2] = {0, 0}, gdf = 0, gdj = 0;
    mu_new_rev(m, ph, mu, dp, F, J, w, lph, lmu, ldp, gdf, gdj);
    double scale = 1e-30, e = 0.0;
    const double h = 1e-6;
    auto fn = [&](const double (&p)[2], double u, const double (&d)[2], const double (&FF)[4], const double (&JJ)[4]) {
      return w * mu_new(m, p, u, d, FF, JJ);
    };
    for (int a = 0; a < 2 && !bulk; a++) {
      double pp[2] = {ph[0], ph[1]}, pm[2] = {ph[0], ph[1]};
      pp[a] += h; pm[a] -= h;
      const double fd = (fn(pp, mu, dp, F, J) - fn(pm, mu, dp, F, J)) / (2 * h);
      scale = fmax(scale, fabs(fd)); e = fmax(e, fabs(fd - lph[a]));
      double dpp[2] = {dp[0], dp[1]}, dpm[2] = {dp[0], dp[1]};
      dpp[a] += h; dpm[a] -= h;
      const double fd2 = (fn(ph, mu, dpp, F, J) - fn(ph, mu, dpm, F, J)) / (2 * h);
      scale = fmax(scale, fabs(fd2)); e = fmax(e, fabs(fd2 - ldp[a]));
    }
    {
      const double fd = (fn(ph, mu + h, dp, F, J) - fn(ph, mu - h, dp, F, J)) / (2 * h);
      scale = fmax(scale, fabs(fd)); e = fmax(e, fabs(fd - lmu));
    }
    for (int k = 0; k < 4; k++) {
      double Fp[4], Fm[4], Jp[4], Jm[4];
      for (int q = 0; q < 4; q++) { Fp[q] = Fm[q] = F[q]; Jp[q] = Jm[q] = J[q]; }
      Fp[k] += h; Fm[k] -= h; Jp[k] += h; Jm[k] -= h;
      const double hk = (k >> 1) ? m.dy : m.dx, sg = (k & 1) ? -1.0 : 1.0;
      const double fdF = (fn(ph, mu, dp, Fp, J) - fn(ph, mu, dp, Fm, J)) / (2 * h);
      const double fdJ = (fn(ph, mu, dp, F, Jp) - fn(ph, mu, dp, F, Jm)) / (2 * h);
      scale = fmax(scale, fmax(fabs(fdF), fabs(fdJ)));
      e = fmax(e, fabs(fdF - gdf * sg / hk));
      e = fmax(e, fabs(fdJ - gdj * sg * m.jscale / hk));
    }
    worst = fmax(worst, e / scale);
    n += bulk ? 9 : 13;
  }
  report(bulk ? "mu_update_bulk" : "mu_update_interface", worst, n);
}

int main() {
  srand(12345);
  check_dphi(1, 200);
  check_dphi(0, 200);
  check_dphi_projection(400);
  check_face(0, 1, 200);
  check_face(1, 1, 200);
  check_face(1, 0, 200);
  check_mu(0, 200);
  check_mu(1, 200);
  return 0;
}
