/*
 * gp_oracle.c -- CPU restatement of the MicroSim grand-potential explicit step.
 *
 * TEST INFRASTRUCTURE ONLY (see gp_oracle.h).  Written from the reference's
 * algorithm, not copied from it: the reference sweeps x-rows through a rolling
 * four-layer gradient buffer; here every gradient record is evaluated from the
 * old phi on demand, which is the same Jacobi update (every read of the
 * reference's two sweeps sees pre-step values).  Operation order inside each
 * expression follows the reference so that doubles agree bit for bit; that is
 * why some sums start at 0.0 and some zero terms are kept.
 *
 * Reference files below are relative to Grand_potential_Finite_difference_2D_serial/.
 */
#include "gp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 8
#define MAXK 4

/* Face/centre gradient record of one cell, the content of one `struct
 * gradlayer` entry for the phase field (functions/global_vars.h:338-346),
 * filled as calculate_gradients_phasefield_2D does
 * (solverloop/calculate_gradients.h:92-131). */
typedef struct {
  double gx[MAXN], gy[MAXN]; /* gradphi[X], gradphi[Y]: forward differences    */
  double sx[MAXN], sy[MAXN]; /* phistagg[X], phistagg[Y]: face averages          */
  double cx[MAXN], cy[MAXN]; /* gradphi_c[X], gradphi_c[Y]: centred gradients    */
} grad_rec;

typedef struct {
  const gpo_params *p;
  long rx, ry;   /* rows_x, rows_y */
  long ncell;
  const double *phi, *mu, *dphi;
} ctx_t;

static inline long IDX(const ctx_t *c, long x, long y) { return y + x * c->ry; }
static inline double PHI(const ctx_t *c, long x, long y, int a) { return c->phi[a * c->ncell + IDX(c, x, y)]; }
static inline double MU(const ctx_t *c, long x, long y, int k) { return c->mu[k * c->ncell + IDX(c, x, y)]; }

/* calculate_gradients.h:100-129.  gradphi_c[X] averages this cell's and the
 * previous x-layer's forward difference; gradphi_c[Y] is the centred difference
 * (valid for 0 < y <= rows_y-2, the only rows used here). */
static void grad_at(const ctx_t *c, long x, long y, grad_rec *g) {
  const gpo_params *p = c->p;
  int a;
  for (a = 0; a < p->N; a++) {
    double pc = PHI(c, x, y, a);
    double pf = PHI(c, x + 1, y, a);
    double pr = PHI(c, x, y + 1, a);
    double pl = PHI(c, x, y - 1, a);
    double pb = PHI(c, x - 1, y, a);
    double gx_back = (pc - pb) / p->dx;
    g->gx[a] = (pf - pc) / p->dx;
    g->sx[a] = 0.5 * (pf + pc);
    g->gy[a] = (pr - pc) / p->dy;
    g->sy[a] = 0.5 * (pr + pc);
    g->cy[a] = (pr - pl) / (2.0 * p->dy);
    g->cx[a] = 0.5 * (g->gx[a] + gx_back);
  }
}

/* functions/functionH.h:24-36 */
static double hphi(const gpo_params *p, const double *phi, int a) {
  double sum1 = 0.0;
  double sum = 3.0 * phi[a] * phi[a] - 2.0 * phi[a] * phi[a] * phi[a];
  int b, d;
  for (b = 0; b < p->N; b++)
    for (d = b + 1; d < p->N; d++)
      if (b != a && d != a) sum1 += phi[b] * phi[d];
  sum1 *= 2.0 * phi[a];
  return sum + sum1;
}

/* dh_b/dphi_a, functions/functionH.h:1-23 (called there as dhphi(phi, b, a)) */
static double dhphi(const gpo_params *p, const double *phi, int b, int a) {
  double sum = 0.0;
  int e, f;
  if (a == b) {
    sum = 6.0 * phi[a] * (1.0 - phi[a]);
    for (e = 0; e < p->N; e++)
      for (f = e + 1; f < p->N; f++)
        if (e != b && f != b) sum += 2.0 * phi[e] * phi[f];
  } else {
    for (e = 0; e < p->N; e++)
      if (e != b && e != a) sum += 2.0 * phi[e];
    sum *= phi[b];
  }
  return sum;
}

/* functions/functionF_01.h:30-37 */
static double c_mu(const gpo_params *p, const double *mu, int a, int i) {
  double sum = 0.0;
  int k, K1 = p->K1;
  for (k = 0; k < K1; k++)
    sum += p->cmu[(a * K1 + i) * K1 + k] * (mu[k] - (p->Beq[a * K1 + k] + p->dBbdT[a * K1 + k] * (p->T - p->Teq)));
  return sum;
}

/* functions/functionF_01.h:19-29 */
static double Mu(const gpo_params *p, const double *cc, int a, int i) {
  int j, K1 = p->K1;
  double sum = 2.0 * p->A[(a * K1 + i) * K1 + i] * cc[i] + (p->Beq[a * K1 + i] + p->dBbdT[a * K1 + i] * (p->T - p->Teq));
  for (j = 0; j < K1; j++)
    if (i != j) sum += p->A[(a * K1 + i) * K1 + j] * cc[j];
  return sum;
}

/* functions/functionF_01.h:5-18 */
static double free_energy(const gpo_params *p, const double *cc, int a) {
  int i, j, K1 = p->K1;
  double sum = 0.0;
  for (i = 0; i < K1; i++) {
    for (j = 0; j < K1; j++)
      if (i <= j) sum += p->A[(a * K1 + i) * K1 + j] * cc[i] * cc[j];
    sum += p->B[a * K1 + i] * cc[i];
  }
  sum += p->C[a];
  return sum;
}

/* d(psi)/d(phi_a) = sum_b psi_b(mu) dh_b/dphi_a, functions/functionF_01.h:41-57 */
static double dpsi(const gpo_params *p, const double *mu, const double *phi, int a) {
  double sum = 0.0, cc[MAXK];
  int b, k;
  for (b = 0; b < p->N; b++) {
    double psi = 0.0;
    for (k = 0; k < p->K1; k++) {
      cc[k] = c_mu(p, mu, b, k);
      psi -= mu[k] * cc[k];
    }
    psi += free_energy(p, cc, b);
    sum += psi * dhphi(p, phi, b, a);
  }
  return sum;
}

/* 2x2 block of a 3x3 matrix times a vector with z = 0 (functions/matrix.h:22-33
 * called with size DIMENSION = 2). */
static void mul2(const double *M, const double *v, double *out) {
  int i;
  for (i = 0; i < 2; i++) {
    double s = 0;
    s = s + M[i * 3 + 0] * v[0];
    s = s + M[i * 3 + 1] * v[1];
    out[i] = s;
  }
}

static const double *Rot(const gpo_params *p, int a, int b) { return p->R + (a * p->N + b) * 9; }
static const double *RotInv(const gpo_params *p, int a, int b) { return p->Rinv + (a * p->N + b) * 9; }

/* functions/anisotropy_01.h:30-48 (4-fold cubic a_c) */
static double aniso_ac(const gpo_params *p, const double *q, int a, int b) {
  double qx2 = q[0] * q[0], qx4 = qx2 * qx2;
  double qy2 = q[1] * q[1], qy4 = qy2 * qy2;
  double qz2 = q[2] * q[2], qz4 = qz2 * qz2;
  double q2 = qx2 + qy2 + qz2;
  if (fabs(q2) > 1.0e-15) return 1.0 - p->dab[a * p->N + b] * (3.0 - 4.0 * (qx4 + qy4 + qz4) / (q2 * q2));
  return 1.0;
}

/* functions/anisotropy_01.h:9-28 (d a_c / d q) */
static void aniso_dadq(const gpo_params *p, const double *q, double *d, int a, int b) {
  double qx3 = q[0] * q[0] * q[0];
  double qy3 = q[1] * q[1] * q[1];
  double qz3 = q[2] * q[2] * q[2];
  double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
  double q22 = q2 * q2;
  double q23 = q2 * q2 * q2;
  double q4 = qx3 * q[0] + qy3 * q[1] + qz3 * q[2];
  double dd = p->dab[a * p->N + b];
  if (fabs(q2) > 1.0e-15) {
    d[0] = 16.0 * dd * (qx3 / q22 - q[0] * q4 / q23);
    d[1] = 16.0 * dd * (qy3 / q22 - q[1] * q4 / q23);
    d[2] = 16.0 * dd * (qz3 / q22 - q[2] * q4 / q23);
  } else {
    d[0] = d[1] = d[2] = 0.0;
  }
}

/* q_ab on an x-face (functions/functionQ.h:4-22), rotated into the pair frame. */
static void q_xface(const gpo_params *p, const grad_rec *g, const grad_rec *gf, int a, int b, double *q) {
  double v[2];
  v[0] = (g->sx[a] * g->gx[b] - g->sx[b] * g->gx[a]);
  v[1] = 0.5 * (g->sx[a] * (g->cy[b] + gf->cy[b]) - g->sx[b] * (g->cy[a] + gf->cy[a]));
  mul2(Rot(p, a, b), v, q);
  q[2] = 0.0;
}

/* q_ab on a y-face (functions/functionQ.h:23-41). */
static void q_yface(const gpo_params *p, const grad_rec *g, const grad_rec *gr, int a, int b, double *q) {
  double v[2];
  v[0] = 0.5 * (g->sy[a] * (g->cx[b] + gr->cx[b]) - g->sy[b] * (g->cx[a] + gr->cx[a]));
  v[1] = (g->sy[a] * g->gy[b] - g->sy[b] * g->gy[a]);
  mul2(Rot(p, a, b), v, q);
  q[2] = 0.0;
}

/* q_ab at the cell centre (functions/functionQ.h:56-68). */
static void q_centre(const gpo_params *p, const double *phi, const grad_rec *g, int a, int b, double *q) {
  double v[2];
  v[0] = (phi[a] * g->cx[b] - phi[b] * g->cx[a]);
  v[1] = (phi[a] * g->cy[b] - phi[b] * g->cy[a]);
  mul2(Rot(p, a, b), v, q);
  q[2] = 0.0;
}

/* dA/dphi_a, isotropic: functions/function_A_00.h:4-19 */
static double dAdphi_iso(const gpo_params *p, const double *phi, const grad_rec *g, int a) {
  double sum = 0.0;
  int b;
  for (b = 0; b < p->N; b++) {
    if (b == a) continue;
    double sp = 0.0;
    sp += (phi[a] * g->cx[b] - phi[b] * g->cx[a]) * g->cx[b];
    sp += (phi[a] * g->cy[b] - phi[b] * g->cy[a]) * g->cy[b];
    sp *= p->Gamma[a * p->N + b];
    sum += sp;
  }
  return 2.0 * sum;
}

/* div(dA/dgrad phi_a), isotropic: functions/function_A_00.h:20-58 */
static double divdA_iso(const gpo_params *p, const grad_rec *g, const grad_rec *gb, const grad_rec *gl, int a) {
  double sum = 0.0;
  int b;
  for (b = 0; b < p->N; b++) {
    if (b == a) continue;
    double dv;
    dv = ((g->sx[a] * g->gx[b] - g->sx[b] * g->gx[a]) * (-g->sx[b]) -
          ((gb->sx[a] * gb->gx[b] - gb->sx[b] * gb->gx[a]) * (-gb->sx[b]))) / p->dx;
    dv += ((g->sy[a] * g->gy[b] - g->sy[b] * g->gy[a]) * (-g->sy[b]) -
           ((gl->sy[a] * gl->gy[b] - gl->sy[b] * gl->gy[a]) * (-gl->sy[b]))) / p->dy;
    dv *= p->Gamma[a * p->N + b];
    sum += dv;
  }
  return 2.0 * sum;
}

/* dA/dphi_a, 4-fold anisotropic: functions/function_A_01.h:4-71 */
static double dAdphi_aniso(const gpo_params *p, const double *phi, const grad_rec *g, int a) {
  double sum1 = 0.0, sum2 = 0.0;
  int b, dir;
  for (b = 0; b < p->N; b++) {
    if (b == a) continue;
    double q[3], dadq[3], dq[2], rdq[2];
    double gam = p->Gamma[a * p->N + b];
    q_centre(p, phi, g, a, b, q);
    aniso_dadq(p, q, dadq, a, b);
    double q2 = (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    double ac1 = aniso_ac(p, q, a, b);
    double ac2 = ac1 * ac1;
    double sp1 = 0.0, sp2 = 0.0;
    dq[0] = g->cx[b];
    dq[1] = g->cy[b];
    mul2(Rot(p, a, b), dq, rdq);
    for (dir = 0; dir < 2; dir++) sp1 += q[dir] * rdq[dir];
    for (dir = 0; dir < 2; dir++) sp2 += (dadq[dir]) * rdq[dir];
    sp1 *= gam * ac2;
    sp2 *= gam * ac1 * q2;
    sum1 += sp1;
    sum2 += sp2;
  }
  return 2.0 * (sum1 + sum2);
}

/* div(dA/dgrad phi_a), 4-fold anisotropic: functions/function_A_01.h:101-219 */
static double divdA_aniso(const gpo_params *p, const grad_rec *g, const grad_rec *gb, const grad_rec *gf,
                          const grad_rec *gl, const grad_rec *gr, int a) {
  double sum1 = 0.0, sum2 = 0.0, div3 = 0.0;
  int b;
  for (b = 0; b < p->N; b++) {
    if (b == a) continue;
    double gam = p->Gamma[a * p->N + b];
    double qf[3], qb[3], qr[3], ql[3];
    double df[3], db[3], dr[3], dl[3];
    double rf[2], rb[2], rr[2], rl[2];
    q_xface(p, g, gf, a, b, qf);
    q_xface(p, gb, g, a, b, qb);
    q_yface(p, g, gr, a, b, qr);
    q_yface(p, gl, g, a, b, ql);
    double acf = aniso_ac(p, qf, a, b), acf2 = acf * acf;
    double acb = aniso_ac(p, qb, a, b), acb2 = acb * acb;
    double acr = aniso_ac(p, qr, a, b), acr2 = acr * acr;
    double acl = aniso_ac(p, ql, a, b), acl2 = acl * acl;
    double d1;
    d1 = ((acf2 * (g->sx[a] * g->gx[b] - g->sx[b] * g->gx[a]) * (-g->sx[b])) -
          (acb2 * (gb->sx[a] * gb->gx[b] - gb->sx[b] * gb->gx[a]) * (-gb->sx[b]))) / p->dx;
    d1 += ((acr2 * (g->sy[a] * g->gy[b] - g->sy[b] * g->gy[a]) * (-g->sy[b])) -
           (acl2 * (gl->sy[a] * gl->gy[b] - gl->sy[b] * gl->gy[a]) * (-gl->sy[b]))) / p->dy;
    d1 *= gam;
    sum1 += d1;

    aniso_dadq(p, qf, df, a, b);
    mul2(RotInv(p, a, b), df, rf);
    double qf2 = qf[0] * qf[0] + qf[1] * qf[1] + qf[2] * qf[2];
    aniso_dadq(p, qb, db, a, b);
    mul2(RotInv(p, a, b), db, rb);
    double qb2 = qb[0] * qb[0] + qb[1] * qb[1] + qb[2] * qb[2];
    aniso_dadq(p, qr, dr, a, b);
    mul2(RotInv(p, a, b), dr, rr);
    double qr2 = qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2];
    aniso_dadq(p, ql, dl, a, b);
    mul2(RotInv(p, a, b), dl, rl);
    double ql2 = ql[0] * ql[0] + ql[1] * ql[1] + ql[2] * ql[2];

    double d2;
    d2 = (acf * qf2 * rf[0] * (-g->sx[b]) - acb * qb2 * rb[0] * (-gb->sx[b])) / p->dx;
    d2 += (acr * qr2 * rr[1] * (-g->sy[b]) - acl * ql2 * rl[1] * (-gl->sy[b])) / p->dy;
    d2 *= gam;
    sum2 += d2;
  }
  return (2.0 * (sum1 + sum2) + div3);
}

/* dw/dphi_a: obstacle functions/functionW_01.h:6-39, well functions/functionW_02.h:4-33 */
static double dwdphi(const gpo_params *p, const double *phi, const double *divphi, int a) {
  int b, d, N = p->N;
  double sum = 0.0;
  if (p->obstacle) {
    for (b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      if ((phi[a] * phi[b]) >= 0.00000) sum += p->Gamma[a * N + b] * (phi[b]);
      else sum += -p->Gamma[a * N + b] * (phi[b]);
    }
    sum *= 16.0 / (M_PI * M_PI);
  } else {
    for (b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += 2.0 * p->Gamma[a * N + b] * (phi[b] * phi[b] * phi[a]);
    }
    sum *= 9.0;
  }
  for (b = 0; b < N; b++) {
    for (d = b + 1; d < N; d++) {
      if (b == a || d == a) continue;
      if (fabs(divphi[b]) > 0.0 && fabs(divphi[d]) > 0.0) {
        double g3 = p->Gamma_abc[(a * N + b) * N + d];
        double pbc = phi[b] * phi[d];
        if (phi[a] * pbc >= 0.00000) sum += g3 * pbc;
        else sum += -g3 * pbc;
      }
    }
  }
  return sum;
}

/* dw/dphi of the smoothing pre-steps: functionW_01.h:41-62 (obstacle) and
 * functionW_02.h:35-59 (well), without the sign factors */
static double dwdphi_smooth(const gpo_params *p, const double *phi, const double *divphi, int a) {
  int b, d, N = p->N;
  double sum = 0.0;
  if (p->obstacle) {
    for (b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += p->Gamma[a * N + b] * phi[b];
    }
    sum *= 16.0 / (M_PI * M_PI);
  } else {
    for (b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += 2.0 * p->Gamma[a * N + b] * (phi[b] * phi[b] * phi[a]);
    }
    sum *= 9.0;
  }
  for (b = 0; b < N; b++)
    for (d = b + 1; d < N; d++) {
      if (b == a || d == a) continue;
      if (fabs(divphi[b]) > 0.0 && fabs(divphi[d]) > 0.0) sum += p->Gamma_abc[(a * N + b) * N + d] * phi[b] * phi[d];
    }
  return sum;
}

/* projection of the smoothing pre-steps, solverloop/simplex_projection.h:50-91:
 * phases in index order; a phase above 1 takes the rest and ends the loop */
static void project_simplex_unweighted(const gpo_params *p, const double *phi, const double *divphi, double *dp) {
  int a, b, N = p->N;
  long count = 0;
  for (a = 0; a < N; a++)
    if ((fabs(divphi[a]) > 0.0) && (phi[a] + dp[a]) > 0.0 && (phi[a] + dp[a]) < 1.0) count++;
  for (a = 0; a < N; a++) {
    if (!(fabs(divphi[a]) > 0.0)) continue;
    if ((phi[a] + dp[a]) > 1.0) {
      dp[a] = (1.0 - phi[a]);
      for (b = 0; b < N; b++)
        if ((fabs(divphi[b]) > 0.0) && b != a) dp[b] = -phi[b];
      break;
    }
    if ((phi[a] + dp[a]) < 0.0) {
      double D = fabs(dp[a] + phi[a]);
      dp[a] += D;
      for (b = 0; b < N; b++)
        if (((fabs(divphi[b]) > 0.0) && b != a) && (phi[b] + dp[b]) > 0.0 && (phi[b] + dp[b]) < 1.0)
          dp[b] -= D / (count);
    }
  }
}

/* functions/functionTau.h:1-16 */
static double tau_phi(const gpo_params *p, const double *phi) {
  double sum = 0.0, sum1 = 0.0;
  int a, b;
  for (a = 0; a < p->N; a++)
    for (b = a + 1; b < p->N; b++) {
      sum += p->tau_ab[a * p->N + b] * phi[a] * phi[b];
      sum1 += phi[a] * phi[b];
    }
  if (sum1) return sum / sum1;
  return p->tau;
}

/* Weighted projection back onto the Gibbs simplex, solverloop/simplex_projection.h:1-49.
 * phi: the cell's phases, dp: its Delta-phi (modified in place). */
static void project_simplex(const gpo_params *p, const double *phi, const double *divphi, double *dp) {
  int a, b, N = p->N;
  double Deltaphi = 0.0, sum_phib = 0.0;
  long count = 0;
  for (a = 0; a < N; a++) {
    if ((fabs(divphi[a]) > 0.0) && (phi[a] + dp[a]) > 0.0 && (phi[a] + dp[a]) < 1.0) {
      count++;
      sum_phib += phi[a];
    }
  }
  for (a = 0; a < N; a++) {
    if ((phi[a] + dp[a]) < 0.0) {
      double over = fabs(dp[a] + phi[a]);
      dp[a] += over;
      Deltaphi += over;
    }
  }
  if (Deltaphi > 0.0) {
    for (b = 0; b < N; b++) {
      if ((fabs(divphi[b]) > 0.0) && ((phi[b] + dp[b]) > 0.0) && ((phi[b] + dp[b]) < 1.0)) {
        if (fabs(sum_phib) > 0.0) dp[b] -= Deltaphi * (phi[b]) / (sum_phib);
        else dp[b] -= Deltaphi / (count);
      }
    }
  }
  for (a = 0; a < N; a++) {
    if (fabs(divphi[a]) > 0.0 && (phi[a] + dp[a]) > 1.0) {
      dp[a] = (1.0 - phi[a]);
      for (b = 0; b < N; b++)
        if ((fabs(divphi[b]) > 0.0) && b != a) dp[b] = -phi[b];
      break;
    }
  }
}

/* Delta-phi of one cell: solverloop/calculate_divergence_phasefield.h:4-62;
 * smooth: the pre-step form of :63-158 (isotropic gradient energy
 * (function_A_01.h:73-99, 220-260 equal function_A_00's), no dpsi, the
 * unsigned potential when anisotropic, unweighted projection) */
static void delta_phi_cell(const ctx_t *c, long x, long y, double *dp, int smooth) {
  const gpo_params *p = c->p;
  int a, N = p->N;
  grad_rec g, gb, gf, gl, gr;
  double phi[MAXN], mu[MAXK], divphi[MAXN], lambda[MAXN];
  double sum_lambda = 0.0;
  long active = 0;
  grad_at(c, x, y, &g);
  grad_at(c, x - 1, y, &gb);
  grad_at(c, x + 1, y, &gf);
  grad_at(c, x, y - 1, &gl);
  grad_at(c, x, y + 1, &gr);
  for (a = 0; a < N; a++) phi[a] = PHI(c, x, y, a);
  for (a = 0; a < p->K1; a++) mu[a] = MU(c, x, y, a);
  for (a = 0; a < N; a++) {
    divphi[a] = (g.gx[a] - gb.gx[a]) / p->dx;
    divphi[a] += (g.gy[a] - gl.gy[a]) / p->dy;
  }
  for (a = 0; a < N; a++) {
    if (fabs(divphi[a]) > 0.0) {
      double dA, divA;
      if (p->anisotropy && !smooth) {
        dA = dAdphi_aniso(p, phi, &g, a);
        divA = divdA_aniso(p, &g, &gb, &gf, &gl, &gr, a);
      } else {
        dA = dAdphi_iso(p, phi, &g, a);
        divA = divdA_iso(p, &g, &gb, &gl, a);
      }
      if (smooth) /* the unsigned potential only with anisotropy (calculate_divergence_phasefield.h:89-97) */
        lambda[a] = p->epsilon * (-dA + divA) -
                    (1.0 / p->epsilon) * (p->anisotropy ? dwdphi_smooth(p, phi, divphi, a) : dwdphi(p, phi, divphi, a));
      else
        lambda[a] = p->epsilon * (-dA + divA) - (1.0 / p->epsilon) * dwdphi(p, phi, divphi, a) - dpsi(p, mu, phi, a);
      sum_lambda += lambda[a];
      active++;
    }
  }
  if (active) sum_lambda /= active;
  for (a = 0; a < N; a++) {
    if (fabs(divphi[a]) > 0.0) dp[a] = p->dt * (lambda[a] - sum_lambda) / (tau_phi(p, phi) * p->epsilon);
    else dp[a] = 0.0;
  }
  if (smooth) project_simplex_unweighted(p, phi, divphi, dp);
  else project_simplex(p, phi, divphi, dp);
}

static void cell_vec(const ctx_t *c, const double *base, int n, long x, long y, double *out) {
  int a;
  for (a = 0; a < n; a++) out[a] = base[a * c->ncell + IDX(c, x, y)];
}

/* s(phi) = phi (1 - h) / sqrt(phi (1 - phi)) of the obstacle antitrapping
 * term, calculate_fluxes_concentration.h:43-59 */
static double s_obstacle(const gpo_params *p, const double *phi, int a) {
  if (phi[a] * (1.0 - phi[a]) > 0.0) return phi[a] * (1.0 - hphi(p, phi, a)) / (sqrt(phi[a] * (1.0 - phi[a])));
  return 0.0;
}

/* Antitrapping currents on the +x face (jx) and +y face (jy) of cell (x, y):
 * solverloop/calculate_fluxes_concentration.h:4-145.  jy is zero on the row
 * gidy == MESH_Y-2, as in the reference (:65). */
static void jat_cell(const ctx_t *c, long x, long y, double *jx, double *jy) {
  const gpo_params *p = c->p;
  int a, k, N = p->N, K1 = p->K1, L = p->N - 1;
  grad_rec g, gr, gf;
  double phc[MAXN], phr[MAXN], phf[MAXN], muc[MAXK], mur[MAXK], muf[MAXK];
  double dpc[MAXN], dpr[MAXN], dpf[MAXN];
  grad_at(c, x, y, &g);
  grad_at(c, x, y + 1, &gr);
  grad_at(c, x + 1, y, &gf);
  cell_vec(c, c->phi, N, x, y, phc);
  cell_vec(c, c->phi, N, x, y + 1, phr);
  cell_vec(c, c->phi, N, x + 1, y, phf);
  cell_vec(c, c->mu, K1, x, y, muc);
  cell_vec(c, c->mu, K1, x, y + 1, mur);
  cell_vec(c, c->mu, K1, x + 1, y, muf);
  cell_vec(c, c->dphi, N, x, y, dpc);
  cell_vec(c, c->dphi, N, x, y + 1, dpr);
  cell_vec(c, c->dphi, N, x + 1, y, dpf);

  double gradphix_l = 0.5 * (g.cx[L] + gr.cx[L]);
  double normgradphiy_l = sqrt(gradphix_l * gradphix_l + g.gy[L] * g.gy[L]);
  double gradphiy_l = 0.5 * (g.cy[L] + gf.cy[L]);
  double normgradphix_l = sqrt(gradphiy_l * gradphiy_l + g.gx[L] * g.gx[L]);
  for (k = 0; k < K1; k++) { jx[k] = 0.0; jy[k] = 0.0; }
  for (a = 0; a < N - 1; a++) {
    double s_r = 0.0, s_c = 0.0, s_f = 0.0;
    double gradphix = 0.5 * (g.cx[a] + gr.cx[a]);
    double normgradphi = sqrt(gradphix * gradphix + g.gy[a] * g.gy[a]);
    if (p->obstacle) {
      s_r = s_obstacle(p, phr, a);
      s_c = s_obstacle(p, phc, a);
      s_f = s_obstacle(p, phf, a);
    }
    for (k = 0; k < K1; k++) {
      if (normgradphi != 0.0 && (y != 0 && y != (p->mesh_y - 2))) {
        double cl_r = c_mu(p, mur, L, k), cl_c = c_mu(p, muc, L, k);
        double cs_r = c_mu(p, mur, a, k), cs_c = c_mu(p, muc, a, k);
        double sp = g.gy[a] * g.gy[L];
        sp += gradphix * gradphix_l;
        if (normgradphiy_l > 0.0) sp /= (normgradphiy_l * normgradphi);
        double f = (1.0 - p->Diff[(a * K1 + k) * K1 + k] / p->Diff[(L * K1 + k) * K1 + k]);
        if (p->obstacle)
          jy[k] += f * fabs(sp) * 0.5 * (s_r * (cl_r - cs_r) * dpr[a] + s_c * (cl_c - cs_c) * dpc[a]) * g.gy[a] / normgradphi;
        else
          jy[k] += f * fabs(sp) * (0.5 / sqrt(2.0)) * ((cl_r - cs_r) * dpr[a] + (cl_c - cs_c) * dpc[a]) * g.gy[a] / normgradphi;
      }
    }
    double gradphiy = 0.5 * (g.cy[a] + gf.cy[a]);
    normgradphi = sqrt(gradphiy * gradphiy + g.gx[a] * g.gx[a]);
    for (k = 0; k < K1; k++) {
      if (normgradphi != 0.0) {
        double cl_f = c_mu(p, muf, L, k), cl_c = c_mu(p, muc, L, k);
        double cs_f = c_mu(p, muf, a, k), cs_c = c_mu(p, muc, a, k);
        double sp = g.gx[a] * g.gx[L];
        sp += gradphiy * gradphiy_l;
        if (normgradphix_l > 0.0) sp /= (normgradphix_l * normgradphi);
        double f = (1.0 - p->Diff[(a * K1 + k) * K1 + k] / p->Diff[(L * K1 + k) * K1 + k]);
        if (p->obstacle)
          jx[k] += f * fabs(sp) * 0.5 * (s_f * (cl_f - cs_f) * dpf[a] + s_c * (cl_c - cs_c) * dpc[a]) * (g.gx[a]) / normgradphi;
        else
          jx[k] += f * fabs(sp) * (0.5 / sqrt(2.0)) * ((cl_f - cs_f) * dpf[a] + (cl_c - cs_c) * dpc[a]) * (g.gx[a]) / normgradphi;
      }
    }
  }
}

/* Mobility D_ij of one cell, functions/functionD.h:1-16 (phi-weighted). */
static double Dcell(const gpo_params *p, const double *phi, int i, int j) {
  double sum = 0.0;
  int b, k, K1 = p->K1;
  for (b = 0; b < p->N; b++)
    for (k = 0; k < K1; k++) sum += p->Diff[(b * K1 + i) * K1 + k] * p->cmu[(b * K1 + k) * K1 + j] * phi[b];
  return sum;
}

/* Port of the reference's LU inverse (functions/matrix.h:50-218), including
 * its pivot that keeps the signed, not absolute, largest entry. */
static void lu_inverse(double m[MAXK][MAXK], double inv[MAXK][MAXK], int n) {
  double fac[MAXK][MAXK], inv1[MAXK][MAXK];
  int tag[MAXK], i, j, k;
  for (k = 0; k < n; k++) tag[k] = k;
  for (i = 0; i < n; i++) for (j = 0; j < n; j++) fac[i][j] = 0.0;
  for (k = 0; k < n; k++) {
    double big = fabs(m[k][k]);
    int t1 = k, ts;
    for (i = k + 1; i < n; i++)
      if (fabs(m[i][k]) > big) { t1 = i; big = m[i][k]; }
    ts = tag[k]; tag[k] = tag[t1]; tag[t1] = ts;
    for (i = 0; i < n; i++) { double s = m[k][i]; m[k][i] = m[t1][i]; m[t1][i] = s; }
    for (i = 0; i < k; i++) { double s = fac[k][i]; fac[k][i] = fac[t1][i]; fac[t1][i] = s; }
    for (i = k + 1; i < n; i++) {
      double f = -m[i][k] / m[k][k];
      fac[i][k] = -f;
      for (j = k; j <= n - 1; j++) m[i][j] = f * m[k][j] + m[i][j];
    }
  }
  for (i = 0; i < n; i++) for (j = 0; j < n; j++) {
    if (i == j) fac[i][j] = 1;
    if (j > i) fac[i][j] = 0;
  }
  for (i = 0; i < n; i++) {
    double v1[MAXK], v[MAXK];
    /* forward substitution on column i of the identity */
    v1[0] = (i == 0) ? 1.0 : 0.0;
    for (k = 1; k < n; k++) {
      double s = 0;
      for (j = 0; j < k; j++) s = s - fac[k][j] * v1[j];
      v1[k] = ((k == i) ? 1.0 : 0.0) + s;
    }
    /* back substitution */
    v[n - 1] = v1[n - 1] * pow(m[n - 1][n - 1], -1);
    for (k = n - 2; k >= 0; k--) {
      double s = 0;
      for (j = k + 1; j < n; j++) s = s - m[k][j] * v[j];
      v[k] = (v1[k] + s) * pow(m[k][k], -1);
    }
    for (j = 0; j < n; j++) inv1[j][i] = v[j];
  }
  for (j = 0; j < n; j++) for (k = 0; k < n; k++) inv[k][tag[j]] = inv1[k][j];
}

/* Cell index maps of the ghost copies (functions/utility_functions.h:471-653). */
static long ghost_src(int type, int side_hi, long g, long rows) {
  /* g: 0,1,2 = distance index j of boundary->points[j]; returns proxy[j]. */
  if (type == 1) return side_hi ? rows - 5 - g : 4 + g;
  return side_hi ? 4 + g : rows - 5 - g; /* periodic */
}

void gpo_apply_bc(const gpo_params *p, double *phi, double *mu) {
  long rx = p->mesh_x + 6, ry = p->mesh_y + 6, n = rx * ry;
  int side, j, a;
  long x, y;
  /* x faces first: boundary[0] (x = 2,1,0) then boundary[1] (x = rows_x-3..-1),
   * whole y-columns (copyYZ, boundary_serial.h:63-119) */
  for (side = 0; side < 2; side++) {
    for (j = 0; j < 3; j++) {
      long to = side ? rx - 3 + j : 2 - j;
      int tp = p->bc_phi[side], tm = p->bc_mu[side];
      if (tp == 1 || tp == 3) {
        long from = ghost_src(tp, side, j, rx);
        for (y = 0; y < ry; y++)
          for (a = 0; a < p->N; a++) phi[a * n + y + to * ry] = phi[a * n + y + from * ry];
      }
      if (tm == 1 || tm == 3) {
        long from = ghost_src(tm, side, j, rx);
        for (y = 0; y < ry; y++)
          for (a = 0; a < p->K1; a++) mu[a * n + y + to * ry] = mu[a * n + y + from * ry];
      }
    }
  }
  /* then y faces over every x: boundary[2] (y = rows_y-3..-1), boundary[3] (y = 2,1,0)
   * (copyXZ, boundary_serial.h:8-62) */
  for (side = 2; side < 4; side++) {
    int hi = (side == 2);
    for (j = 0; j < 3; j++) {
      long to = hi ? ry - 3 + j : 2 - j;
      int tp = p->bc_phi[side], tm = p->bc_mu[side];
      if (tp == 1 || tp == 3) {
        long from = ghost_src(tp, hi, j, ry);
        for (x = 0; x < rx; x++)
          for (a = 0; a < p->N; a++) phi[a * n + to + x * ry] = phi[a * n + from + x * ry];
      }
      if (tm == 1 || tm == 3) {
        long from = ghost_src(tm, hi, j, ry);
        for (x = 0; x < rx; x++)
          for (a = 0; a < p->K1; a++) mu[a * n + to + x * ry] = mu[a * n + from + x * ry];
      }
    }
  }
}

/* One explicit step: the phase-field half step (solverloop.h:21-34) fills
 * Delta-phi on the ring [2, rows-3]^2, the concentration half step
 * (solverloop.h:35-71 -> calculate_divergence_concentration.h:4-153) updates
 * mu and phi on the interior, then the ghosts are refilled (microsim_gp.c:103-106). */
/* One time step (solverloop.h:21-71), or with smooth one pre-step
 * (solverloop.h:72-90: calculate_divergence_concentration.h:154-253, no
 * antitrapping current and no dh/dt source, the LU inverse for every mu solve). */
static int one_step(const gpo_params *p, double *phi, double *mu, double *dphi, double *phi_new, double *mu_new,
                    double *jxa, double *jya, gpo_stats *st, int smooth) {
  long rx = p->mesh_x + 6, ry = p->mesh_y + 6, n = rx * ry;
  int N = p->N, K1 = p->K1, a, k, l;
  long x, y;
  ctx_t c;
  c.p = p; c.rx = rx; c.ry = ry; c.ncell = n; c.phi = phi; c.mu = mu; c.dphi = dphi;

  for (x = 2; x <= rx - 3; x++)
    for (y = 2; y <= ry - 3; y++) {
      double dp[MAXN];
      delta_phi_cell(&c, x, y, dp, smooth);
      for (a = 0; a < N; a++) dphi[a * n + y + x * ry] = dp[a];
    }
  /* microsim_gp.c:103-106: the boundary copy between the two half steps (a no-op
   * unless the ghost rows were left stale, as a moving-frame shift leaves them;
   * the smoothing pre-step is one sweep, solverloop.h:72-90) */
  if (!smooth) gpo_apply_bc(p, phi, mu);
  /* antitrapping currents on faces touching the interior */
  for (x = 2; x <= rx - 4 && !smooth; x++)
    for (y = 2; y <= ry - 4; y++) {
      double jx[MAXK], jy[MAXK];
      jat_cell(&c, x, y, jx, jy);
      for (k = 0; k < K1; k++) {
        jxa[k * n + y + x * ry] = jx[k];
        jya[k * n + y + x * ry] = jy[k];
      }
    }
  memcpy(phi_new, phi, sizeof(double) * N * n);
  memcpy(mu_new, mu, sizeof(double) * K1 * n);
  if (st && !smooth) {
    for (a = 0; a < N; a++) st->rel_change_phi[a] = 0.0;
    for (k = 0; k < K1; k++) st->rel_change_mu[k] = 0.0;
  }
  for (x = 3; x <= rx - 4; x++)
    for (y = 3; y <= ry - 4; y++) {
      long id = y + x * ry;
      double ph[MAXN], dp[MAXN], m[MAXK];
      double sum[MAXK], divflux[MAXK], divjat[MAXK], dcdmu[MAXK][MAXK], inv[MAXK][MAXK], deltac[MAXK], deltamu[MAXK];
      cell_vec(&c, phi, N, x, y, ph);
      cell_vec(&c, dphi, N, x, y, dp);
      cell_vec(&c, mu, K1, x, y, m);
      double phf[MAXN], phb[MAXN], phr[MAXN], phl[MAXN];
      cell_vec(&c, phi, N, x + 1, y, phf);
      cell_vec(&c, phi, N, x - 1, y, phb);
      cell_vec(&c, phi, N, x, y + 1, phr);
      cell_vec(&c, phi, N, x, y - 1, phl);
      for (k = 0; k < K1; k++) {
        sum[k] = 0.0;
        for (l = 0; l < K1; l++) dcdmu[k][l] = 0.0;
      }
      for (a = 0; a < N; a++) {
        double sdh = 0.0;
        int b;
        for (b = 0; b < N; b++) sdh += dhphi(p, ph, a, b) * dp[b];
        for (k = 0; k < K1; k++) sum[k] += c_mu(p, m, a, k) * sdh;
      }
      for (k = 0; k < K1; k++) {
        divflux[k] = 0.0;
        for (l = 0; l < K1; l++) {
          /* face mobilities and mu gradients, calculate_gradients.h:132-185 */
          double Dx = (Dcell(p, phf, k, l) + Dcell(p, ph, k, l)) * 0.5;
          double Dxb = (Dcell(p, ph, k, l) + Dcell(p, phb, k, l)) * 0.5;
          double Dy = (Dcell(p, phr, k, l) + Dcell(p, ph, k, l)) * 0.5;
          double Dyl = (Dcell(p, ph, k, l) + Dcell(p, phl, k, l)) * 0.5;
          double gmx = (MU(&c, x + 1, y, l) - MU(&c, x, y, l)) / p->dx;
          double gmxb = (MU(&c, x, y, l) - MU(&c, x - 1, y, l)) / p->dx;
          double gmy = (MU(&c, x, y + 1, l) - MU(&c, x, y, l)) / p->dy;
          double gmyl = (MU(&c, x, y, l) - MU(&c, x, y - 1, l)) / p->dy;
          divflux[k] += (Dx * gmx - Dxb * gmxb) / p->dx;
          divflux[k] += (Dy * gmy - Dyl * gmyl) / p->dy;
        }
        double jx = smooth ? 0.0 : jxa[k * n + id], jxb = smooth ? 0.0 : jxa[k * n + id - ry];
        double jy = smooth ? 0.0 : jya[k * n + id], jyl = smooth ? 0.0 : jya[k * n + id - 1];
        if (smooth) {
          divjat[k] = 0.0;
        } else if (p->obstacle) {
          divjat[k] = (jx - jxb) * (-0.25 * M_PI * p->epsilon) / p->dx;
          divjat[k] += (jy - jyl) * (-0.25 * M_PI * p->epsilon) / p->dy;
        } else {
          divjat[k] = (jx - jxb) * (-1.0 * p->epsilon) / p->dx;
          divjat[k] += (jy - jyl) * (-1.0 * p->epsilon) / p->dy;
        }
      }
      int bulk = -1;
      for (a = 0; a < N; a++)
        if (ph[a] == 1.0) { bulk = a; break; }
      double mnew[MAXK];
      if (bulk >= 0 && smooth) {
        double cnew[MAXK];
        for (k = 0; k < K1; k++) cnew[k] = c_mu(p, m, bulk, k) + p->dt * (divflux[k]);
        for (k = 0; k < K1; k++) mnew[k] = Mu(p, cnew, bulk, k);
      } else if (smooth) {
        /* deltac = dt divflux; dcdmu^-1 by matinvnew (LU); mu += inv deltac */
        for (k = 0; k < K1; k++) {
          deltac[k] = p->dt * (divflux[k]);
          for (l = 0; l < K1; l++)
            for (a = 0; a < N; a++) dcdmu[k][l] += p->cmu[(a * K1 + k) * K1 + l] * hphi(p, ph, a);
        }
        lu_inverse(dcdmu, inv, K1);
        for (k = 0; k < K1; k++) {
          double s = 0;
          for (l = 0; l < K1; l++) s = s + inv[k][l] * deltac[l];
          deltamu[k] = s;
        }
        for (k = 0; k < K1; k++) mnew[k] = deltamu[k] + m[k];
      } else if (bulk >= 0) {
        double cnew[MAXK];
        for (k = 0; k < K1; k++) cnew[k] = c_mu(p, m, bulk, k) + p->dt * (divflux[k]) - divjat[k];
        for (k = 0; k < K1; k++) {
          double v = Mu(p, cnew, bulk, k);
          deltamu[k] = v - m[k];
          mnew[k] = v;
        }
      } else {
        for (k = 0; k < K1; k++) {
          deltac[k] = p->dt * (divflux[k]) - divjat[k] - sum[k];
          for (l = 0; l < K1; l++)
            for (a = 0; a < N; a++) dcdmu[k][l] += p->cmu[(a * K1 + k) * K1 + l] * hphi(p, ph, a);
        }
        for (k = 0; k < K1; k++) mnew[k] = m[k];
        if (p->binary) {
          double iv = 1.0 / dcdmu[0][0];
          deltamu[0] = deltac[0] * iv;
          mnew[0] = m[0] + deltamu[0];
          for (k = 1; k < K1; k++) deltamu[k] = 0.0;
        } else if (p->ternary) {
          double DET = dcdmu[0][0] * dcdmu[1][1] - dcdmu[0][1] * dcdmu[1][0];
          inv[0][0] = dcdmu[1][1] / DET;
          inv[1][1] = dcdmu[0][0] / DET;
          inv[0][1] = -dcdmu[0][1] / DET;
          inv[1][0] = -dcdmu[1][0] / DET;
          for (k = 0; k < K1; k++) {
            deltamu[k] = 0.0;
            for (l = 0; l < K1; l++) deltamu[k] += inv[k][l] * deltac[l];
          }
          for (k = 0; k < K1; k++) mnew[k] = deltamu[k] + m[k];
        } else if (p->dilute) {
          for (k = 0; k < K1; k++) {
            double iv = 1.0 / dcdmu[k][k];
            deltamu[k] = deltac[k] * iv;
            mnew[k] = m[k] + deltamu[k];
          }
        } else {
          lu_inverse(dcdmu, inv, K1);
          for (k = 0; k < K1; k++) {
            double s = 0;
            for (l = 0; l < K1; l++) s = s + inv[k][l] * deltac[l];
            deltamu[k] = s;
          }
          for (k = 0; k < K1; k++) mnew[k] = deltamu[k] + m[k];
        }
      }
      for (k = 0; k < K1; k++) mu_new[k * n + id] = mnew[k];
      for (a = 0; a < N; a++) {
        double v = ph[a] + dp[a];
        phi_new[a * n + id] = v;
        if (st && !smooth) {
          if (v > st->phi_max[a]) st->phi_max[a] = v;
          if (v < st->phi_min[a]) st->phi_min[a] = v;
          st->rel_change_phi[a] += dp[a] * dp[a];
        }
      }
      if (st && !smooth) {
        for (k = 0; k < K1; k++) {
          if (mnew[k] > st->mu_max[k]) st->mu_max[k] = mnew[k];
          if (mnew[k] < st->mu_min[k]) st->mu_min[k] = mnew[k];
          st->rel_change_mu[k] += deltamu[k] * deltamu[k];
        }
      }
    }
  memcpy(phi, phi_new, sizeof(double) * N * n);
  memcpy(mu, mu_new, sizeof(double) * K1 * n);
  gpo_apply_bc(p, phi, mu);
  return 0;
}

int gpo_step(const gpo_params *p, double *phi, double *mu, long nsteps, double *dphi_first, gpo_stats *st) {
  long rx, ry, n, t;
  int a, k;
  if (p->N < 2 || p->N > MAXN || p->K1 < 1 || p->K1 > MAXK) return -1;
  if (p->mesh_x < 4 || p->mesh_y < 4) return -1;
  for (a = 0; a < 4; a++) {
    if (p->bc_phi[a] != 1 && p->bc_phi[a] != 3) return -1;
    if (p->bc_mu[a] != 1 && p->bc_mu[a] != 3) return -1;
  }
  if (p->ternary && p->K1 != 2) return -1;
  rx = p->mesh_x + 6; ry = p->mesh_y + 6; n = rx * ry;
  double *dphi = (double *)calloc((size_t)(p->N * n), sizeof(double));
  double *pn = (double *)malloc(sizeof(double) * p->N * n);
  double *mn = (double *)malloc(sizeof(double) * p->K1 * n);
  double *jx = (double *)calloc((size_t)(p->K1 * n), sizeof(double));
  double *jy = (double *)calloc((size_t)(p->K1 * n), sizeof(double));
  if (st) {
    /* serialinfo_xy.h:59-66: running extrema start at 1/0 (phi) and 1/1 (mu) */
    for (a = 0; a < p->N; a++) { st->phi_max[a] = 1.0; st->phi_min[a] = 0.0; st->rel_change_phi[a] = 0.0; }
    for (k = 0; k < p->K1; k++) { st->mu_max[k] = 1.0; st->mu_min[k] = 1.0; st->rel_change_mu[k] = 0.0; }
  }
  for (t = 0; t < nsteps; t++) {
    one_step(p, phi, mu, dphi, pn, mn, jx, jy, st, 0);
    if (t == 0 && dphi_first) memcpy(dphi_first, dphi, sizeof(double) * p->N * n);
  }
  free(dphi); free(pn); free(mn); free(jx); free(jy);
  return 0;
}

/* NSMOOTH - 1 pre-steps (microsim_gp.c:97-100), each followed by the boundary copy */
int gpo_smooth(const gpo_params *p, double *phi, double *mu, long nsteps) {
  long rx, ry, n, t;
  int a;
  if (p->N < 2 || p->N > MAXN || p->K1 < 1 || p->K1 > MAXK) return -1;
  if (p->mesh_x < 4 || p->mesh_y < 4) return -1;
  for (a = 0; a < 4; a++) {
    if (p->bc_phi[a] != 1 && p->bc_phi[a] != 3) return -1;
    if (p->bc_mu[a] != 1 && p->bc_mu[a] != 3) return -1;
  }
  rx = p->mesh_x + 6; ry = p->mesh_y + 6; n = rx * ry;
  double *dphi = (double *)calloc((size_t)(p->N * n), sizeof(double));
  double *pn = (double *)malloc(sizeof(double) * p->N * n);
  double *mn = (double *)malloc(sizeof(double) * p->K1 * n);
  for (t = 0; t < nsteps; t++) one_step(p, phi, mu, dphi, pn, mn, NULL, NULL, NULL, 1);
  free(dphi); free(pn); free(mn);
  return 0;
}
