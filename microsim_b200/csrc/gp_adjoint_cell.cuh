// gp_adjoint_cell.cuh -- the explicit step of a binary alloy (2 phases, one
// independent chemical potential) as cell- and face-level functions, each with
// its hand-written reverse (vector-Jacobian product).
//
// Forward: the same model as the plain step (gp_f64.cu, reference
// Grand_potential_Finite_difference_2D_serial/solverloop/*), specialised to
// N = 2, K-1 = 1, isothermal, anisotropic gradient energy (function_A_01 with
// anisotropy_01; an isotropic model is the special case delta = 0 with the
// identity rotation), obstacle or well potential, antitrapping current:
//   * Delta-phi of a cell from its 3x3 phi stencil and its mu
//     (calculate_divergence_phasefield.h:4-62, simplex_projection.h:1-49);
//   * face diffusion flux F and antitrapping current J between two cells
//     (calculate_gradients.h:132-185, calculate_fluxes_concentration.h:4-145);
//   * the cell's mu update from its four faces
//     (calculate_divergence_concentration.h:4-153), phi += Delta-phi.
// For two phases dh_b/dphi_a = delta_ab 6 phi_a (1 - phi_a) and
// h_a = phi_a^2 (3 - 2 phi_a) (functionH.h with N = 2).
//
// Reverse: every function *_rev takes the adjoint of the forward outputs and
// accumulates (+=) the adjoints of its inputs and of the four calibration
// parameters: mobility M = 1/tau (tau and tau_ab scaled together),
// anisotropy strength delta, interface energy gamma, liquid diffusivity D_l.
// Branches (active phases, projection cases, bulk cells, |q|^2 guard) are
// taken as in the forward: the reverse is the derivative of the branch taken.
//
// Everything is __host__ __device__ so the local reverses can be checked
// against finite differences on the CPU.
#pragma once

#include <math.h>

#ifndef GP_HD
#define GP_HD __host__ __device__ __forceinline__
#endif

namespace gpadj {

enum { P_MOB = 0, P_DELTA = 1, P_GAMMA = 2, P_DLIQ = 3, NPARAM = 4 };

// Model constants of one instance, in the working precision T.
template <typename T>
struct AM {
  T dx, dy, dt, eps, inv_eps;
  T mob;             // 1 / tau_ab[0][1]
  T tau_ratio;       // tau / tau_ab[0][1] (the fallback tau of cells with phi_0 phi_1 = 0)
  T gam, dab;        // Gamma[0][1], dab[0][1]
  T wobs;            // 16 / pi^2
  T jscale, swell;   // -pi eps / 4 (obstacle) or -eps (well); 1 / (2 sqrt 2)
  T R[2][2][2];      // R[a] = Rotation_matrix of pair (a, 1-a)
  T Ri[2][2][2];     // its inverse
  T cmu[2], A[2], B[2], C[2], Beff[2];
  T Ds, Dl;          // Diff of the solid (phase 0) and the liquid (phase 1)
  int obstacle;
  int skip_row;      // interior row whose upper y-face carries no antitrapping current
};

// ------------------------------------------------------------------ small pieces

template <typename T>
GP_HD T hfun(T p) { return p * p * ((T)3 - (T)2 * p); }  // h_a for two phases
template <typename T>
GP_HD T dhfun(T p) { return (T)6 * p * ((T)1 - p); }     // dh_a / dphi_a
template <typename T>
GP_HD T d2hfun(T p) { return (T)6 - (T)12 * p; }

template <typename T>
GP_HD T cmu_of(const AM<T>& m, int a, T mu) { return m.cmu[a] * (mu - m.Beff[a]); }  // c_a(mu)

// psi_a(mu) = f_a(c) - mu c, c = c_a(mu); and d psi_a / d mu
template <typename T>
GP_HD T psi_of(const AM<T>& m, int a, T mu) {
  const T c = cmu_of(m, a, mu);
  return m.A[a] * c * c + m.B[a] * c + m.C[a] - mu * c;
}
template <typename T>
GP_HD T dpsi_dmu(const AM<T>& m, int a, T mu) {
  const T c = cmu_of(m, a, mu);
  return ((T)2 * m.A[a] * c + m.B[a] - mu) * m.cmu[a] - c;
}

// 2x2 matrix times vector
template <typename T>
GP_HD void mv(const T (&M)[2][2], T v0, T v1, T& o0, T& o1) {
  o0 = M[0][0] * v0 + M[0][1] * v1;
  o1 = M[1][0] * v0 + M[1][1] * v1;
}
// reverse of mv: adjoints of v from adjoints of o
template <typename T>
GP_HD void mv_rev(const T (&M)[2][2], T l0, T l1, T& lv0, T& lv1) {
  lv0 += M[0][0] * l0 + M[1][0] * l1;
  lv1 += M[0][1] * l0 + M[1][1] * l1;
}

// Cubic anisotropy (anisotropy_01.h): a_c(q) = 1 - delta (3 - 4 s4),
// s4 = (q0^4 + q1^4) / |q|^4, and d = d a_c / d q = 16 delta u(q),
// u_i = q_i^3/|q|^4 - q_i (q0^4 + q1^4)/|q|^6; a_c = 1, d = 0 when |q|^2 <= 1e-15.
template <typename T>
struct Aniso {
  T ac, d0, d1;       // a_c and its gradient
  T g;                // d a_c / d delta = -(3 - 4 s4)
  T u0, u1;           // d / 16 delta
  T J[2][2];          // d u_i / d q_j
  bool on;
};

template <typename T>
GP_HD Aniso<T> aniso(T dab, T q0, T q1) {
  Aniso<T> r;
  const T q2 = q0 * q0 + q1 * q1;
  r.on = fabs(q2) > (T)1.0e-15;
  if (!r.on) {
    r.ac = (T)1;
    r.d0 = r.d1 = r.g = r.u0 = r.u1 = (T)0;
    r.J[0][0] = r.J[0][1] = r.J[1][0] = r.J[1][1] = (T)0;
    return r;
  }
  // in the components of the unit vector n = q/|q| (no high powers of 1/|q|,
  // which overflow single precision near the guard):
  //   s4 = n0^4 + n1^4,  u_i = (n_i^3 - n_i s4) / |q|,
  //   du_i/dq_i = (3 n_i^2 - 8 n_i^4 - s4 + 6 n_i^2 s4) / |q|^2,
  //   du_i/dq_j = (-4 n_i^3 n_j - 4 n_i n_j^3 + 6 n_i n_j s4) / |q|^2
  const T rq = (T)1 / sqrt(q2), i2 = rq * rq;
  const T n0 = q0 * rq, n1 = q1 * rq, a0 = n0 * n0, a1 = n1 * n1;
  const T s4 = a0 * a0 + a1 * a1;
  r.g = -((T)3 - (T)4 * s4);
  r.ac = (T)1 + dab * r.g;
  r.u0 = (a0 * n0 - n0 * s4) * rq;
  r.u1 = (a1 * n1 - n1 * s4) * rq;
  r.d0 = (T)16 * dab * r.u0;
  r.d1 = (T)16 * dab * r.u1;
  r.J[0][0] = ((T)3 * a0 - (T)8 * a0 * a0 - s4 + (T)6 * a0 * s4) * i2;
  r.J[1][1] = ((T)3 * a1 - (T)8 * a1 * a1 - s4 + (T)6 * a1 * s4) * i2;
  r.J[0][1] = n0 * n1 * (-(T)4 * a0 - (T)4 * a1 + (T)6 * s4) * i2;
  r.J[1][0] = r.J[0][1];
  return r;
}

// Gradient record pieces of a Delta-phi cell (calculate_gradients.h:92-131),
// per phase, from P[i][j][a] = phi_a at (x+i-1, y+j-1).
template <typename T>
struct Grad {
  T gx[2], sx[2], gy[2], sy[2], cy[2], bgx[2], cx[2], bsx[2], bcy[2], fcy[2], lgy[2], lsy[2], lcx[2], rcx[2];
};

template <typename T>
GP_HD void grad_fwd(const AM<T>& m, const T (&P)[3][3][2], Grad<T>& G) {
  const T ty = (T)2 * m.dy;
  for (int a = 0; a < 2; a++) {
    G.gx[a] = (P[2][1][a] - P[1][1][a]) / m.dx;
    G.sx[a] = (T)0.5 * (P[2][1][a] + P[1][1][a]);
    G.gy[a] = (P[1][2][a] - P[1][1][a]) / m.dy;
    G.sy[a] = (T)0.5 * (P[1][2][a] + P[1][1][a]);
    G.cy[a] = (P[1][2][a] - P[1][0][a]) / ty;
    G.bgx[a] = (P[1][1][a] - P[0][1][a]) / m.dx;
    G.cx[a] = (T)0.5 * (G.gx[a] + G.bgx[a]);
    G.bsx[a] = (T)0.5 * (P[1][1][a] + P[0][1][a]);
    G.bcy[a] = (P[0][2][a] - P[0][0][a]) / ty;
    G.fcy[a] = (P[2][2][a] - P[2][0][a]) / ty;
    G.lgy[a] = (P[1][1][a] - P[1][0][a]) / m.dy;
    G.lsy[a] = (T)0.5 * (P[1][1][a] + P[1][0][a]);
    G.lcx[a] = (T)0.5 * ((P[2][0][a] - P[1][0][a]) / m.dx + (P[1][0][a] - P[0][0][a]) / m.dx);
    G.rcx[a] = (T)0.5 * ((P[2][2][a] - P[1][2][a]) / m.dx + (P[1][2][a] - P[0][2][a]) / m.dx);
  }
}

// reverse of grad_fwd: LG holds the adjoints of the record, accumulated into LP
template <typename T>
GP_HD void grad_rev(const AM<T>& m, const Grad<T>& LG, T (&LP)[3][3][2]) {
  const T ty = (T)2 * m.dy;
  for (int a = 0; a < 2; a++) {
    const T lgx = LG.gx[a] + (T)0.5 * LG.cx[a], lbgx = LG.bgx[a] + (T)0.5 * LG.cx[a];
    LP[2][1][a] += lgx / m.dx + (T)0.5 * LG.sx[a];
    LP[1][1][a] += -lgx / m.dx + (T)0.5 * LG.sx[a];
    LP[1][2][a] += LG.gy[a] / m.dy + (T)0.5 * LG.sy[a];
    LP[1][1][a] += -LG.gy[a] / m.dy + (T)0.5 * LG.sy[a];
    LP[1][2][a] += LG.cy[a] / ty;
    LP[1][0][a] -= LG.cy[a] / ty;
    LP[1][1][a] += lbgx / m.dx + (T)0.5 * LG.bsx[a];
    LP[0][1][a] += -lbgx / m.dx + (T)0.5 * LG.bsx[a];
    LP[0][2][a] += LG.bcy[a] / ty;
    LP[0][0][a] -= LG.bcy[a] / ty;
    LP[2][2][a] += LG.fcy[a] / ty;
    LP[2][0][a] -= LG.fcy[a] / ty;
    LP[1][1][a] += LG.lgy[a] / m.dy + (T)0.5 * LG.lsy[a];
    LP[1][0][a] += -LG.lgy[a] / m.dy + (T)0.5 * LG.lsy[a];
    const T hl = (T)0.5 * LG.lcx[a] / m.dx, hr = (T)0.5 * LG.rcx[a] / m.dx;
    LP[2][0][a] += hl;
    LP[0][0][a] -= hl;
    LP[2][2][a] += hr;
    LP[0][2][a] -= hr;
  }
}

// ------------------------------------------------------------------ gradient energy

// One face term of div(dA/dgrad phi_a) (function_A_01.h:101-219):
//   V = (-S) [a_c(q)^2 Qn + a_c(q) |q|^2 (Rinv d(q))_n],  q = R (Qx, Qy),
// n = 0 for an x-face (Qn = Qx), 1 for a y-face.
template <typename T>
GP_HD T face_term(const T (&R)[2][2], const T (&Ri)[2][2], T dab, T Qx, T Qy, T S, int n) {
  T q0, q1, r0, r1;
  mv(R, Qx, Qy, q0, q1);
  const Aniso<T> A = aniso(dab, q0, q1);
  mv(Ri, A.d0, A.d1, r0, r1);
  const T q2 = q0 * q0 + q1 * q1;
  const T Qn = n ? Qy : Qx, rn = n ? r1 : r0;
  return -S * (A.ac * A.ac * Qn + A.ac * q2 * rn);
}

template <typename T>
GP_HD void face_term_rev(const T (&R)[2][2], const T (&Ri)[2][2], T dab, T Qx, T Qy, T S, int n, T lam, T& lQx,
                         T& lQy, T& lS, T& ldab) {
  T q0, q1, r0, r1;
  mv(R, Qx, Qy, q0, q1);
  const Aniso<T> A = aniso(dab, q0, q1);
  mv(Ri, A.d0, A.d1, r0, r1);
  const T q2 = q0 * q0 + q1 * q1;
  const T Qn = n ? Qy : Qx, rn = n ? r1 : r0;
  const T W = A.ac * A.ac * Qn + A.ac * q2 * rn;
  lS += -W * lam;
  const T lW = -S * lam;
  const T lac = lW * ((T)2 * A.ac * Qn + q2 * rn);
  const T lQn = lW * A.ac * A.ac;
  const T lq2 = lW * A.ac * rn;
  const T lrn = lW * A.ac * q2;
  const T le0 = Ri[n][0] * lrn, le1 = Ri[n][1] * lrn;  // e = d(q)
  const T c = (T)16 * dab;
  T lq0 = c * (le0 * A.J[0][0] + le1 * A.J[1][0]) + lac * A.d0 + (T)2 * q0 * lq2;
  T lq1 = c * (le0 * A.J[0][1] + le1 * A.J[1][1]) + lac * A.d1 + (T)2 * q1 * lq2;
  ldab += (T)16 * (le0 * A.u0 + le1 * A.u1) + lac * A.g;
  mv_rev(R, lq0, lq1, lQx, lQy);
  if (n) lQy += lQn;
  else lQx += lQn;
}

// The four face operands of div(dA/dgrad phi_a), b = 1 - a:
// k = 0 front (+x), 1 back (-x), 2 right (+y), 3 left (-y)
template <typename T>
GP_HD void face_ops(const Grad<T>& G, int a, int k, T& Qx, T& Qy, T& S) {
  const int b = 1 - a;
  if (k == 0) {
    Qx = G.sx[a] * G.gx[b] - G.sx[b] * G.gx[a];
    Qy = (T)0.5 * (G.sx[a] * (G.cy[b] + G.fcy[b]) - G.sx[b] * (G.cy[a] + G.fcy[a]));
    S = G.sx[b];
  } else if (k == 1) {
    Qx = G.bsx[a] * G.bgx[b] - G.bsx[b] * G.bgx[a];
    Qy = (T)0.5 * (G.bsx[a] * (G.bcy[b] + G.cy[b]) - G.bsx[b] * (G.bcy[a] + G.cy[a]));
    S = G.bsx[b];
  } else if (k == 2) {
    Qx = (T)0.5 * (G.sy[a] * (G.cx[b] + G.rcx[b]) - G.sy[b] * (G.cx[a] + G.rcx[a]));
    Qy = G.sy[a] * G.gy[b] - G.sy[b] * G.gy[a];
    S = G.sy[b];
  } else {
    Qx = (T)0.5 * (G.lsy[a] * (G.lcx[b] + G.cx[b]) - G.lsy[b] * (G.lcx[a] + G.cx[a]));
    Qy = G.lsy[a] * G.lgy[b] - G.lsy[b] * G.lgy[a];
    S = G.lsy[b];
  }
}

template <typename T>
GP_HD void face_ops_rev(const Grad<T>& G, int a, int k, T lQx, T lQy, T lS, Grad<T>& L) {
  const int b = 1 - a;
  if (k == 0) {
    L.sx[a] += lQx * G.gx[b] + (T)0.5 * lQy * (G.cy[b] + G.fcy[b]);
    L.gx[b] += lQx * G.sx[a];
    L.sx[b] += -lQx * G.gx[a] - (T)0.5 * lQy * (G.cy[a] + G.fcy[a]) + lS;
    L.gx[a] += -lQx * G.sx[b];
    L.cy[b] += (T)0.5 * lQy * G.sx[a];
    L.fcy[b] += (T)0.5 * lQy * G.sx[a];
    L.cy[a] += -(T)0.5 * lQy * G.sx[b];
    L.fcy[a] += -(T)0.5 * lQy * G.sx[b];
  } else if (k == 1) {
    L.bsx[a] += lQx * G.bgx[b] + (T)0.5 * lQy * (G.bcy[b] + G.cy[b]);
    L.bgx[b] += lQx * G.bsx[a];
    L.bsx[b] += -lQx * G.bgx[a] - (T)0.5 * lQy * (G.bcy[a] + G.cy[a]) + lS;
    L.bgx[a] += -lQx * G.bsx[b];
    L.bcy[b] += (T)0.5 * lQy * G.bsx[a];
    L.cy[b] += (T)0.5 * lQy * G.bsx[a];
    L.bcy[a] += -(T)0.5 * lQy * G.bsx[b];
    L.cy[a] += -(T)0.5 * lQy * G.bsx[b];
  } else if (k == 2) {
    L.sy[a] += (T)0.5 * lQx * (G.cx[b] + G.rcx[b]) + lQy * G.gy[b];
    L.sy[b] += -(T)0.5 * lQx * (G.cx[a] + G.rcx[a]) - lQy * G.gy[a] + lS;
    L.cx[b] += (T)0.5 * lQx * G.sy[a];
    L.rcx[b] += (T)0.5 * lQx * G.sy[a];
    L.cx[a] += -(T)0.5 * lQx * G.sy[b];
    L.rcx[a] += -(T)0.5 * lQx * G.sy[b];
    L.gy[b] += lQy * G.sy[a];
    L.gy[a] += -lQy * G.sy[b];
  } else {
    L.lsy[a] += (T)0.5 * lQx * (G.lcx[b] + G.cx[b]) + lQy * G.lgy[b];
    L.lsy[b] += -(T)0.5 * lQx * (G.lcx[a] + G.cx[a]) - lQy * G.lgy[a] + lS;
    L.lcx[b] += (T)0.5 * lQx * G.lsy[a];
    L.cx[b] += (T)0.5 * lQx * G.lsy[a];
    L.lcx[a] += -(T)0.5 * lQx * G.lsy[b];
    L.cx[a] += -(T)0.5 * lQx * G.lsy[b];
    L.lgy[b] += lQy * G.lsy[a];
    L.lgy[a] += -lQy * G.lsy[b];
  }
}

// t_a = -dA/dphi_a + div dA/dgrad phi_a for the pair (a, 1-a)
// (function_A_01.h:4-71, 101-219)
template <typename T>
GP_HD T tterm(const AM<T>& m, const Grad<T>& G, const T (&ph)[2], int a) {
  const int b = 1 - a;
  const T v0 = ph[a] * G.cx[b] - ph[b] * G.cx[a], v1 = ph[a] * G.cy[b] - ph[b] * G.cy[a];
  T q0, q1, r0, r1;
  mv(m.R[a], v0, v1, q0, q1);
  mv(m.R[a], G.cx[b], G.cy[b], r0, r1);
  const Aniso<T> A = aniso(m.dab, q0, q1);
  const T q2 = q0 * q0 + q1 * q1;
  const T qr = q0 * r0 + q1 * r1, dr = A.d0 * r0 + A.d1 * r1;
  const T dA = (T)2 * m.gam * (A.ac * A.ac * qr + A.ac * q2 * dr);
  T sum = (T)0;
  for (int k = 0; k < 4; k++) {
    T Qx, Qy, S;
    face_ops(G, a, k, Qx, Qy, S);
    const T V = face_term(m.R[a], m.Ri[a], m.dab, Qx, Qy, S, k >> 1);
    const T h = (k >> 1) ? m.dy : m.dx;
    sum += (k & 1) ? -V / h : V / h;
  }
  return -dA + (T)2 * m.gam * sum;
}

template <typename T>
GP_HD void tterm_rev(const AM<T>& m, const Grad<T>& G, const T (&ph)[2], int a, T lam, Grad<T>& LG, T (&lph)[2],
                     T& ldab, T& lgam) {
  const int b = 1 - a;
  // divA = 2 gam sum_k sign_k V_k / h_k
  T sum = (T)0;
  for (int k = 0; k < 4; k++) {
    T Qx, Qy, S;
    face_ops(G, a, k, Qx, Qy, S);
    const T h = (k >> 1) ? m.dy : m.dx;
    const T sg = (k & 1) ? (T)-1 : (T)1;
    sum += sg * face_term(m.R[a], m.Ri[a], m.dab, Qx, Qy, S, k >> 1) / h;
    T lQx = 0, lQy = 0, lS = 0;
    face_term_rev(m.R[a], m.Ri[a], m.dab, Qx, Qy, S, k >> 1, (T)2 * m.gam * sg / h * lam, lQx, lQy, lS, ldab);
    face_ops_rev(G, a, k, lQx, lQy, lS, LG);
  }
  lgam += (T)2 * sum * lam;
  // -dA
  const T v0 = ph[a] * G.cx[b] - ph[b] * G.cx[a], v1 = ph[a] * G.cy[b] - ph[b] * G.cy[a];
  T q0, q1, r0, r1;
  mv(m.R[a], v0, v1, q0, q1);
  mv(m.R[a], G.cx[b], G.cy[b], r0, r1);
  const Aniso<T> A = aniso(m.dab, q0, q1);
  const T q2 = q0 * q0 + q1 * q1;
  const T qr = q0 * r0 + q1 * r1, dr = A.d0 * r0 + A.d1 * r1;
  const T ldA = -lam;
  lgam += (T)2 * (A.ac * A.ac * qr + A.ac * q2 * dr) * ldA;
  const T L = (T)2 * m.gam * ldA;
  const T lac = L * ((T)2 * A.ac * qr + q2 * dr);
  const T lqr = L * A.ac * A.ac, lq2 = L * A.ac * dr, ldr = L * A.ac * q2;
  const T ld0 = ldr * r0, ld1 = ldr * r1;
  const T lr0 = lqr * q0 + ldr * A.d0, lr1 = lqr * q1 + ldr * A.d1;
  const T c = (T)16 * m.dab;
  const T lq0 = lqr * r0 + c * (ld0 * A.J[0][0] + ld1 * A.J[1][0]) + lac * A.d0 + (T)2 * q0 * lq2;
  const T lq1 = lqr * r1 + c * (ld0 * A.J[0][1] + ld1 * A.J[1][1]) + lac * A.d1 + (T)2 * q1 * lq2;
  ldab += (T)16 * (ld0 * A.u0 + ld1 * A.u1) + lac * A.g;
  T lcxb = 0, lcyb = 0, lv0 = 0, lv1 = 0;
  mv_rev(m.R[a], lr0, lr1, lcxb, lcyb);
  mv_rev(m.R[a], lq0, lq1, lv0, lv1);
  lph[a] += lv0 * G.cx[b] + lv1 * G.cy[b];
  lph[b] += -lv0 * G.cx[a] - lv1 * G.cy[a];
  LG.cx[b] += lcxb + lv0 * ph[a];
  LG.cy[b] += lcyb + lv1 * ph[a];
  LG.cx[a] += -lv0 * ph[b];
  LG.cy[a] += -lv1 * ph[b];
}

// ------------------------------------------------------------------ Delta-phi of a cell

// Branches of the simplex projection (simplex_projection.h:1-49), two phases.
struct Proj {
  bool inr[2];   // step 1: active and 0 < phi + dp < 1
  bool neg[2];   // step 2: phi + dp < 0, clamped
  bool inr2[2];  // step 3: receives a share of the clamped amount
  bool redist, use_sum;
  int cnt, hit;
};

template <typename T>
GP_HD void proj_fwd(const T (&ph)[2], const bool (&act)[2], T (&dp)[2], Proj& r, T& Dsum, T& sphi) {
  r.cnt = 0;
  sphi = (T)0;
  for (int a = 0; a < 2; a++) {
    const T v = ph[a] + dp[a];
    r.inr[a] = act[a] && v > (T)0 && v < (T)1;
    if (r.inr[a]) {
      r.cnt++;
      sphi += ph[a];
    }
  }
  Dsum = (T)0;
  for (int a = 0; a < 2; a++) {
    r.neg[a] = (ph[a] + dp[a]) < (T)0;
    if (r.neg[a]) {
      const T over = fabs(dp[a] + ph[a]);
      dp[a] += over;
      Dsum += over;
    }
  }
  r.redist = Dsum > (T)0;
  r.use_sum = fabs(sphi) > (T)0;
  for (int b = 0; b < 2; b++) {
    const T v = ph[b] + dp[b];
    r.inr2[b] = r.redist && act[b] && v > (T)0 && v < (T)1;
    if (r.inr2[b]) dp[b] -= r.use_sum ? Dsum * ph[b] / sphi : Dsum / (T)r.cnt;
  }
  r.hit = -1;
  for (int a = 0; a < 2; a++)
    if (r.hit < 0 && act[a] && ph[a] + dp[a] > (T)1) r.hit = a;
  if (r.hit >= 0)
    for (int a = 0; a < 2; a++) {
      if (a == r.hit) dp[a] = (T)1 - ph[a];
      else if (act[a]) dp[a] = -ph[a];
    }
}

// reverse: ld holds the adjoints of the projected dp on entry and of the
// unprojected dp on return
template <typename T>
GP_HD void proj_rev(const T (&ph)[2], const bool (&act)[2], const Proj& r, T Dsum, T sphi, T (&ld)[2], T (&lph)[2]) {
  if (r.hit >= 0)
    for (int a = 0; a < 2; a++)
      if (a == r.hit || act[a]) {
        lph[a] -= ld[a];
        ld[a] = (T)0;
      }
  T lD = (T)0, ls = (T)0;
  for (int b = 0; b < 2; b++)
    if (r.inr2[b]) {
      if (r.use_sum) {
        lD -= ld[b] * ph[b] / sphi;
        lph[b] -= ld[b] * Dsum / sphi;
        ls += ld[b] * Dsum * ph[b] / (sphi * sphi);
      } else {
        lD -= ld[b] / (T)r.cnt;
      }
    }
  for (int a = 0; a < 2; a++)
    if (r.inr[a]) lph[a] += ls;
  for (int a = 0; a < 2; a++)
    if (r.neg[a]) {  // dp -> -phi, Dsum += -(phi + dp)
      lph[a] -= ld[a] + lD;
      ld[a] = -lD;
    }
}

// Effective mobility 1/tau(phi) (functionTau.h:1-16 for two phases:
// tau_ab when phi_0 phi_1 != 0, else tau)
template <typename T>
GP_HD T mob_eff(const AM<T>& m, const T (&ph)[2]) {
  const T st1 = ph[0] * ph[1];
  return (st1 != (T)0 || st1 != st1) ? m.mob : m.mob / m.tau_ratio;
}

// obstacle / well derivative w_a (functionW_01.h:6-39, functionW_02.h:4-33)
template <typename T>
GP_HD T wfun(const AM<T>& m, const T (&ph)[2], const bool (&act)[2], int a) {
  const int b = 1 - a;
  if (!act[b]) return (T)0;
  if (m.obstacle) return m.wobs * ((ph[a] * ph[b] >= (T)0) ? m.gam : -m.gam) * ph[b];
  return (T)18 * m.gam * ph[b] * ph[b] * ph[a];
}

// Delta-phi of a cell from its 3x3 phi stencil and its mu
// (calculate_divergence_phasefield.h:4-62)
template <typename T>
GP_HD void dphi_fwd(const AM<T>& m, const T (&P)[3][3][2], T mu, T (&dp)[2]) {
  Grad<T> G;
  grad_fwd(m, P, G);
  const T ph[2] = {P[1][1][0], P[1][1][1]};
  bool act[2];
  T lam[2], sum = (T)0;
  int cnt = 0;
  for (int a = 0; a < 2; a++) {
    const T dv = (G.gx[a] - G.bgx[a]) / m.dx + (G.gy[a] - G.lgy[a]) / m.dy;
    act[a] = fabs(dv) > (T)0;
  }
  for (int a = 0; a < 2; a++) {
    lam[a] = (T)0;
    if (act[a]) {
      lam[a] = m.eps * tterm(m, G, ph, a) - m.inv_eps * wfun(m, ph, act, a) - psi_of(m, a, mu) * dhfun(ph[a]);
      sum += lam[a];
      cnt++;
    }
  }
  if (cnt) sum /= (T)cnt;
  const T k = m.dt * mob_eff(m, ph) / m.eps;
  for (int a = 0; a < 2; a++) dp[a] = act[a] ? k * (lam[a] - sum) : (T)0;
  Proj r;
  T Dsum, sphi;
  proj_fwd(ph, act, dp, r, Dsum, sphi);
}

// reverse of dphi_fwd: ldp = adjoint of dp; accumulates LP, lmu, lpar
template <typename T>
GP_HD void dphi_rev(const AM<T>& m, const T (&P)[3][3][2], T mu, const T (&ldp)[2], T (&LP)[3][3][2], T& lmu,
                    T (&lpar)[NPARAM]) {
  Grad<T> G;
  grad_fwd(m, P, G);
  const T ph[2] = {P[1][1][0], P[1][1][1]};
  bool act[2];
  T lam[2], sum = (T)0;
  int cnt = 0;
  for (int a = 0; a < 2; a++) {
    const T dv = (G.gx[a] - G.bgx[a]) / m.dx + (G.gy[a] - G.lgy[a]) / m.dy;
    act[a] = fabs(dv) > (T)0;
  }
  for (int a = 0; a < 2; a++) {
    lam[a] = (T)0;
    if (act[a]) {
      lam[a] = m.eps * tterm(m, G, ph, a) - m.inv_eps * wfun(m, ph, act, a) - psi_of(m, a, mu) * dhfun(ph[a]);
      sum += lam[a];
      cnt++;
    }
  }
  if (!cnt) return;  // Delta-phi is 0 whatever the inputs
  sum /= (T)cnt;
  const T me = mob_eff(m, ph);
  const T k = m.dt * me / m.eps;
  T dp[2];
  for (int a = 0; a < 2; a++) dp[a] = act[a] ? k * (lam[a] - sum) : (T)0;
  Proj r;
  T Dsum, sphi;
  proj_fwd(ph, act, dp, r, Dsum, sphi);
  T ld[2] = {ldp[0], ldp[1]}, lph[2] = {(T)0, (T)0};
  proj_rev(ph, act, r, Dsum, sphi, ld, lph);
  // dp_a = k (lam_a - mean) on active phases
  T llam[2] = {(T)0, (T)0}, lmean = (T)0;
  for (int a = 0; a < 2; a++)
    if (act[a]) {
      llam[a] += k * ld[a];
      lmean -= k * ld[a];
      lpar[P_MOB] += ld[a] * (lam[a] - sum) * k / m.mob;  // d me / d mob = me / mob
    }
  Grad<T> LG = {};
  for (int a = 0; a < 2; a++)
    if (act[a]) {
      const T la = llam[a] + lmean / (T)cnt;
      // lam_a = eps t_a - w_a / eps - psi_a(mu) h'(phi_a)
      tterm_rev(m, G, ph, a, m.eps * la, LG, lph, lpar[P_DELTA], lpar[P_GAMMA]);
      const T lw = -m.inv_eps * la;
      const int b = 1 - a;
      if (act[b]) {
        if (m.obstacle) {
          const T sg = (ph[a] * ph[b] >= (T)0) ? (T)1 : (T)-1;
          lph[b] += m.wobs * sg * m.gam * lw;
          lpar[P_GAMMA] += m.wobs * sg * ph[b] * lw;
        } else {
          lph[b] += (T)36 * m.gam * ph[b] * ph[a] * lw;
          lph[a] += (T)18 * m.gam * ph[b] * ph[b] * lw;
          lpar[P_GAMMA] += (T)18 * ph[b] * ph[b] * ph[a] * lw;
        }
      }
      lmu -= dpsi_dmu(m, a, mu) * dhfun(ph[a]) * la;
      lph[a] -= psi_of(m, a, mu) * d2hfun(ph[a]) * la;
    }
  LP[1][1][0] += lph[0];
  LP[1][1][1] += lph[1];
  grad_rev(m, LG, LP);
}

// ------------------------------------------------------------------ faces of the mu update

// Operands of the face between a lower cell c and its upper neighbour n along
// x (n = (x+1, y)) or y (n = (x, y+1)).  t: the centred gradient of phi along
// the face of each cell (cy for an x-face, cx for a y-face); dp: Delta-phi of
// phase 0 (the solid) of each cell.
template <typename T>
struct Face {
  T pc[2], pn[2], tc[2], tn[2], muc, mun, dpc, dpn, h;
  bool skip;  // the face carries no antitrapping current
};
template <typename T>
struct FaceAdj {
  T pc[2], pn[2], tc[2], tn[2], muc, mun, dpc, dpn;
};

// diffusion flux D_face (mu_n - mu_c) / h, D_face = (D(phi_n) + D(phi_c)) / 2,
// D(phi) = sum_b Diff_b cmu_b phi_b (functionD.h:1-16, calculate_gradients.h:132-185)
template <typename T>
GP_HD T fface(const AM<T>& m, const Face<T>& f) {
  const T Dc = m.Ds * m.cmu[0] * f.pc[0] + m.Dl * m.cmu[1] * f.pc[1];
  const T Dn = m.Ds * m.cmu[0] * f.pn[0] + m.Dl * m.cmu[1] * f.pn[1];
  return (Dn + Dc) * (T)0.5 * ((f.mun - f.muc) / f.h);
}

template <typename T>
GP_HD void fface_rev(const AM<T>& m, const Face<T>& f, T lF, FaceAdj<T>& L, T (&lpar)[NPARAM]) {
  const T Dc = m.Ds * m.cmu[0] * f.pc[0] + m.Dl * m.cmu[1] * f.pc[1];
  const T Dn = m.Ds * m.cmu[0] * f.pn[0] + m.Dl * m.cmu[1] * f.pn[1];
  const T g = (f.mun - f.muc) / f.h;
  const T lD = (T)0.5 * g * lF;  // adjoint of Dc and of Dn
  const T lg = (Dn + Dc) * (T)0.5 * lF;
  L.mun += lg / f.h;
  L.muc -= lg / f.h;
  L.pc[0] += lD * m.Ds * m.cmu[0];
  L.pn[0] += lD * m.Ds * m.cmu[0];
  L.pc[1] += lD * m.Dl * m.cmu[1];
  L.pn[1] += lD * m.Dl * m.cmu[1];
  lpar[P_DLIQ] += lD * m.cmu[1] * (f.pc[1] + f.pn[1]);
}

// s(phi) of the obstacle antitrapping term (calculate_fluxes_concentration.h:43-59)
template <typename T>
GP_HD T sfun(T p) {
  const T g = p * ((T)1 - p);
  return g > (T)0 ? p * ((T)1 - hfun(p)) / sqrt(g) : (T)0;
}
template <typename T>
GP_HD T dsfun(T p) {
  const T g = p * ((T)1 - p);
  if (!(g > (T)0)) return (T)0;
  const T sg = sqrt(g), num = p * ((T)1 - hfun(p));
  const T dnum = ((T)1 - hfun(p)) - p * dhfun(p);
  return (dnum * sg - num * ((T)1 - (T)2 * p) / ((T)2 * sg)) / g;
}

// antitrapping current through the face, solid phase 0 against the liquid
// (calculate_fluxes_concentration.h:25-141 with N = 2, one component)
template <typename T>
GP_HD T jface(const AM<T>& m, const Face<T>& f) {
  if (f.skip) return (T)0;
  const T gn0 = (f.pn[0] - f.pc[0]) / f.h, gn1 = (f.pn[1] - f.pc[1]) / f.h;
  const T ta = (T)0.5 * (f.tc[0] + f.tn[0]), tl = (T)0.5 * (f.tc[1] + f.tn[1]);
  const T norm_l = sqrt(tl * tl + gn1 * gn1), normg = sqrt(ta * ta + gn0 * gn0);
  if (normg == (T)0) return (T)0;
  const T dcn = m.cmu[1] * (f.mun - m.Beff[1]) - m.cmu[0] * (f.mun - m.Beff[0]);
  const T dcc = m.cmu[1] * (f.muc - m.Beff[1]) - m.cmu[0] * (f.muc - m.Beff[0]);
  T sp = gn0 * gn1 + ta * tl;
  if (norm_l > (T)0) sp = sp / norm_l / normg;
  const T fa = (T)1 - m.Ds / m.Dl;
  const T K = m.obstacle ? (T)0.5 * (sfun(f.pn[0]) * dcn * f.dpn + sfun(f.pc[0]) * dcc * f.dpc)
                         : m.swell * (dcn * f.dpn + dcc * f.dpc);
  return fa * fabs(sp) * K * gn0 / normg;
}

template <typename T>
GP_HD void jface_rev(const AM<T>& m, const Face<T>& f, T lJ, FaceAdj<T>& L, T (&lpar)[NPARAM]) {
  if (f.skip) return;
  const T gn0 = (f.pn[0] - f.pc[0]) / f.h, gn1 = (f.pn[1] - f.pc[1]) / f.h;
  const T ta = (T)0.5 * (f.tc[0] + f.tn[0]), tl = (T)0.5 * (f.tc[1] + f.tn[1]);
  const T norm_l = sqrt(tl * tl + gn1 * gn1), normg = sqrt(ta * ta + gn0 * gn0);
  if (normg == (T)0) return;
  const T dcn = m.cmu[1] * (f.mun - m.Beff[1]) - m.cmu[0] * (f.mun - m.Beff[0]);
  const T dcc = m.cmu[1] * (f.muc - m.Beff[1]) - m.cmu[0] * (f.muc - m.Beff[0]);
  const T sp0 = gn0 * gn1 + ta * tl;
  const bool nl = norm_l > (T)0;
  const T sp = nl ? sp0 / norm_l / normg : sp0;
  const T fa = (T)1 - m.Ds / m.Dl;
  const T sn = m.obstacle ? sfun(f.pn[0]) : (T)0, sc = m.obstacle ? sfun(f.pc[0]) : (T)0;
  const T K = m.obstacle ? (T)0.5 * (sn * dcn * f.dpn + sc * dcc * f.dpc) : m.swell * (dcn * f.dpn + dcc * f.dpc);
  const T Gq = gn0 / normg, A = fabs(sp);
  // J = fa A K Gq
  lpar[P_DLIQ] += lJ * A * K * Gq * (m.Ds / (m.Dl * m.Dl));
  const T lsp = lJ * fa * K * Gq * (sp > (T)0 ? (T)1 : (sp < (T)0 ? (T)-1 : (T)0));
  const T lK = lJ * fa * A * Gq;
  const T lG = lJ * fa * A * K;
  // K
  T ldcn, ldcc;
  if (m.obstacle) {
    L.dpn += lK * (T)0.5 * sn * dcn;
    L.dpc += lK * (T)0.5 * sc * dcc;
    ldcn = lK * (T)0.5 * sn * f.dpn;
    ldcc = lK * (T)0.5 * sc * f.dpc;
    L.pn[0] += lK * (T)0.5 * dsfun(f.pn[0]) * dcn * f.dpn;
    L.pc[0] += lK * (T)0.5 * dsfun(f.pc[0]) * dcc * f.dpc;
  } else {
    L.dpn += lK * m.swell * dcn;
    L.dpc += lK * m.swell * dcc;
    ldcn = lK * m.swell * f.dpn;
    ldcc = lK * m.swell * f.dpc;
  }
  L.mun += ldcn * (m.cmu[1] - m.cmu[0]);
  L.muc += ldcc * (m.cmu[1] - m.cmu[0]);
  // Gq = gn0 / normg
  T lgn0 = lG / normg, lgn1 = (T)0, lta = (T)0, ltl = (T)0;
  T lnormg = -lG * (Gq / normg), lnorm_l = (T)0;
  // sp = sp0 / norm_l / normg
  T lsp0 = lsp;
  if (nl) {
    lsp0 = lsp / norm_l / normg;
    lnorm_l -= lsp * (sp / norm_l);
    lnormg -= lsp * (sp / normg);
  }
  lgn0 += lsp0 * gn1;
  lgn1 += lsp0 * gn0;
  lta += lsp0 * tl;
  ltl += lsp0 * ta;
  if (nl) {
    ltl += lnorm_l * tl / norm_l;
    lgn1 += lnorm_l * gn1 / norm_l;
  }
  lta += lnormg * ta / normg;
  lgn0 += lnormg * gn0 / normg;
  L.tc[0] += (T)0.5 * lta;
  L.tn[0] += (T)0.5 * lta;
  L.tc[1] += (T)0.5 * ltl;
  L.tn[1] += (T)0.5 * ltl;
  L.pn[0] += lgn0 / f.h;
  L.pc[0] -= lgn0 / f.h;
  L.pn[1] += lgn1 / f.h;
  L.pc[1] -= lgn1 / f.h;
}

// ------------------------------------------------------------------ mu and phi update of a cell

// F[k], J[k]: fluxes of the faces x+, x-, y+, y- (calculate_divergence_concentration.h:4-153)
template <typename T>
GP_HD T mu_new(const AM<T>& m, const T (&ph)[2], T mu, const T (&dp)[2], const T (&F)[4], const T (&J)[4]) {
  const T divflux = (F[0] - F[1]) / m.dx + (F[2] - F[3]) / m.dy;
  const T divjat = (J[0] - J[1]) * m.jscale / m.dx + (J[2] - J[3]) * m.jscale / m.dy;
  const int bulk = ph[0] == (T)1 ? 0 : (ph[1] == (T)1 ? 1 : -1);
  if (bulk >= 0) {
    const T c = cmu_of(m, bulk, mu) + m.dt * divflux - divjat;
    return (T)2 * m.A[bulk] * c + m.Beff[bulk];
  }
  T sum = (T)0, dcdmu = (T)0;
  for (int a = 0; a < 2; a++) {
    sum += cmu_of(m, a, mu) * dhfun(ph[a]) * dp[a];
    dcdmu += m.cmu[a] * hfun(ph[a]);
  }
  return mu + (m.dt * divflux - divjat - sum) / dcdmu;
}

// reverse of mu_new for the adjoint lmn of the new mu: accumulates lph, lmu,
// ldp; returns the adjoints of divflux and divjat in gdf, gdj
template <typename T>
GP_HD void mu_new_rev(const AM<T>& m, const T (&ph)[2], T mu, const T (&dp)[2], const T (&F)[4], const T (&J)[4],
                      T lmn, T (&lph)[2], T& lmu, T (&ldp)[2], T& gdf, T& gdj) {
  const int bulk = ph[0] == (T)1 ? 0 : (ph[1] == (T)1 ? 1 : -1);
  if (bulk >= 0) {
    const T lc = (T)2 * m.A[bulk] * lmn;
    lmu += lc * m.cmu[bulk];
    gdf = lc * m.dt;
    gdj = -lc;
    return;
  }
  const T divflux = (F[0] - F[1]) / m.dx + (F[2] - F[3]) / m.dy;
  const T divjat = (J[0] - J[1]) * m.jscale / m.dx + (J[2] - J[3]) * m.jscale / m.dy;
  T sum = (T)0, dcdmu = (T)0;
  for (int a = 0; a < 2; a++) {
    sum += cmu_of(m, a, mu) * dhfun(ph[a]) * dp[a];
    dcdmu += m.cmu[a] * hfun(ph[a]);
  }
  const T dc = m.dt * divflux - divjat - sum;
  const T ldc = lmn / dcdmu, lq = -lmn * dc / (dcdmu * dcdmu);
  lmu += lmn;
  gdf = ldc * m.dt;
  gdj = -ldc;
  const T ls = -ldc;
  for (int a = 0; a < 2; a++) {
    lph[a] += lq * m.cmu[a] * dhfun(ph[a]);
    lmu += ls * m.cmu[a] * dhfun(ph[a]) * dp[a];
    lph[a] += ls * cmu_of(m, a, mu) * d2hfun(ph[a]) * dp[a];
    ldp[a] += ls * cmu_of(m, a, mu) * dhfun(ph[a]);
  }
}

}  // namespace gpadj
