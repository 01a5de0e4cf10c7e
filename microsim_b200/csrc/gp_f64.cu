// gp_f64.cu -- the plain form of the step: FP64, bit-faithful to the reference.
//
// Compiled with -fmad=false (and IEEE division / square root): every a*b+c
// stays a rounded multiply followed by a rounded add, as on x86-64 without
// FMA, and every expression keeps the reference's operation order, so the
// doubles produced here equal the reference solver's.
//
// Two kernels per step, the reference's two half steps
// (microsim_gp.c:103-106), both pure functions of the pre-step state (the
// reference's sweeps are Jacobi: every stencil read sees old values):
//   k_dphi   -- Delta-phi on the interior plus one ghost ring
//               (solverloop/calculate_divergence_phasefield.h:4-62), written to
//               a scratch ring array (the reference keeps it in the grid cells);
//   k_update -- antitrapping currents, mu update and phi += Delta-phi on the
//               interior (calculate_fluxes_concentration.h:4-145,
//               calculate_divergence_concentration.h:4-153), into the other
//               buffer of a double-buffered state.
// Ghost cells are read through gp_map (boundary copies as index maps).
//
// Reference paths are relative to Grand_potential_Finite_difference_2D_serial/.

#include "gp_common.cuh"

namespace {

struct Geo {
  int mx, my;      // interior cells
  int pitch;       // elements per x-row of a state plane
  int64_t plane;   // elements per state plane
  int rpitch;      // elements per x-row of the Delta-phi ring array
  int64_t rplane;  // elements per ring plane
  gp_bc bc;
  // ghost rows y = -3..-1, my..my+2 held explicitly ([N + K1 planes][mx][6]), or
  // nullptr: ghost reads through the boundary map.  Set for the phase-field half
  // step right after a moving-frame shift, which reads the shifted ghost rows
  // before the boundary copy refreshes them (microsim_gp.c:103-125).
  const double* gov;
  // non-isothermal frozen gradient: T of ghost-padded row gy = t_bottom + gy * t_grad, for the
  // step being computed; t_linear: the phase-field half step reads the ghost rows' own linear T
  // (every step after the first: the reference resets T after the step's last boundary copy),
  // else their boundary copy
  int noniso, t_linear;
  int bc_t;  // boundary copy of T along y: 1 Neumann, 3 periodic, 0 none
  double t_bottom, t_grad;
};


// T of interior/ghost row y (interior coordinates) in the phase-field half step (linear ghosts, or
// their boundary copy in the first step) or the concentration half step (boundary copy).
__device__ __forceinline__ Th th_row(const gp_model& m, const Geo& g, int y, bool linear) {
  Th t;
  t.on = g.noniso;
  if (!g.noniso) {
    t.T = m.T;
    return t;
  }
  const int yy = (linear || !g.bc_t || (y >= 0 && y < g.my)) ? y : gp_map(y, g.my, g.bc_t);
  t.T = g.t_bottom + (double)(yy + 3) * g.t_grad;
  return t;
}

__device__ __forceinline__ const double* ghost_row(const Geo& g, int x, int y, int xtype, int q) {
  const int slot = y < 0 ? y + 3 : y - g.my + 3;
  return g.gov + ((int64_t)q * g.mx + gp_map(x, g.mx, xtype)) * 6 + slot;
}

template <int N>
__device__ __forceinline__ void load_phi(const double* __restrict__ phi, const Geo& g, int x, int y, double* out) {
  if (g.gov && (y < 0 || y >= g.my)) {
#pragma unroll
    for (int a = 0; a < N; a++) out[a] = *ghost_row(g, x, y, g.bc.phi_x, a);
    return;
  }
  const int ix = gp_map(x, g.mx, g.bc.phi_x), iy = gp_map(y, g.my, g.bc.phi_y);
  const double* p = phi + (int64_t)ix * g.pitch + iy;
#pragma unroll
  for (int a = 0; a < N; a++) out[a] = __ldg(p + a * g.plane);
}

template <int K1>
__device__ __forceinline__ void load_mu(const double* __restrict__ mu, const Geo& g, int x, int y, double* out,
                                        int nphase = 0) {
  if (g.gov && (y < 0 || y >= g.my)) {
#pragma unroll
    for (int k = 0; k < K1; k++) out[k] = *ghost_row(g, x, y, g.bc.mu_x, nphase + k);
    return;
  }
  const int ix = gp_map(x, g.mx, g.bc.mu_x), iy = gp_map(y, g.my, g.bc.mu_y);
  const double* p = mu + (int64_t)ix * g.pitch + iy;
#pragma unroll
  for (int k = 0; k < K1; k++) out[k] = __ldg(p + k * g.plane);
}

// The 3x3 phi block around (x, y).  A cell whose block lies inside the grid reads it with plain
// offsets; the others map each neighbour through the boundary copy (the same values).
template <int N>
__device__ __forceinline__ void load_block(const double* __restrict__ phi, const Geo& g, int x, int y,
                                           double (&P)[3][3][N]) {
  if (x >= 1 && x <= g.mx - 2 && y >= 1 && y <= g.my - 2) {
    const double* p = phi + (int64_t)(x - 1) * g.pitch + (y - 1);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++)
#pragma unroll
        for (int a = 0; a < N; a++) P[i][j][a] = __ldg(p + i * g.pitch + j + a * g.plane);
    return;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) load_phi<N>(phi, g, x + i - 1, y + j - 1, P[i][j]);
}

// ---------------------------------------------------------------- model terms

// h_a(phi), functions/functionH.h:24-36
template <int N>
__device__ __forceinline__ double hphi(const double* phi, int a) {
  double sum1 = 0.0;
  double sum = 3.0 * phi[a] * phi[a] - 2.0 * phi[a] * phi[a] * phi[a];
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = b + 1; c < N; c++)
      if (b != a && c != a) sum1 += phi[b] * phi[c];
  sum1 *= 2.0 * phi[a];
  return sum + sum1;
}

// dh_b/dphi_a, functions/functionH.h:1-23
template <int N>
__device__ __forceinline__ double dhphi(const double* phi, int b, int a) {
  double sum = 0.0;
  if (a == b) {
    sum = 6.0 * phi[a] * (1.0 - phi[a]);
#pragma unroll
    for (int e = 0; e < N; e++)
#pragma unroll
      for (int f = e + 1; f < N; f++)
        if (e != b && f != b) sum += 2.0 * phi[e] * phi[f];
  } else {
#pragma unroll
    for (int e = 0; e < N; e++)
      if (e != b && e != a) sum += 2.0 * phi[e];
    sum *= phi[b];
  }
  return sum;
}

// c_a,i(mu, T), functions/functionF_01.h:30-37
template <int K1>
__device__ __forceinline__ double c_mu(const gp_model& m, Th t, const double* mu, int a, int i) {
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < K1; k++) sum += m.cmu[a][i][k] * (mu[k] - beff(m, t, a, k));
  return sum;
}

// functions/functionF_01.h:19-29
template <int K1>
__device__ __forceinline__ double Mu(const gp_model& m, Th t, const double* c, int a, int i) {
  double sum = 2.0 * m.A[a][i][i] * c[i] + beff(m, t, a, i);
#pragma unroll
  for (int j = 0; j < K1; j++)
    if (i != j) sum += m.A[a][i][j] * c[j];
  return sum;
}

// functions/functionF_01.h:5-18, with B and C at the cell's T (init_propertymatrices(T))
template <int N, int K1>
__device__ __forceinline__ double free_energy(const gp_model& m, Th t, const double* c, int a) {
  double sum = 0.0;
#pragma unroll
  for (int i = 0; i < K1; i++) {
#pragma unroll
    for (int j = i; j < K1; j++) sum += m.A[a][i][j] * c[i] * c[j];
    sum += B_Tn<N, K1>(m, t, i, a) * c[i];
  }
  sum += C_Tn<N, K1>(m, t, a);
  return sum;
}

// d psi / d phi_a, functions/functionF_01.h:41-57
// x / d with IEEE rounding.  When d is an exact power of two the quotient equals
// the product with the exact reciprocal (one rounding of the same real number),
// so that case multiplies: the bits are those of the division, without the
// division routine (dx = dy = 1 and 2 dy = 2 in most inputs).
__device__ __forceinline__ double gp_ddiv(double x, double d) {
  const long long bits = __double_as_longlong(d);
  const long long ex = (bits >> 52) & 0x7FF;
  if ((bits & 0x000FFFFFFFFFFFFFLL) == 0 && ex > 1 && ex < 2046 && bits > 0)
    return x * __longlong_as_double((2046LL << 52) - bits);
  return x / d;
}

template <int N, int K1>
__device__ __forceinline__ double dpsi(const gp_model& m, Th t, const double* mu, const double* phi, int a) {
  double sum = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++) {
    double c[K1];
    double psi = 0.0;
#pragma unroll
    for (int k = 0; k < K1; k++) {
      c[k] = c_mu<K1>(m, t, mu, b, k);
      psi -= mu[k] * c[k];
    }
    psi += free_energy<N, K1>(m, t, c, b);
    sum += psi * dhphi<N>(phi, b, a);
  }
  return sum;
}

// 2x2 block times vector, functions/matrix.h:22-33 with size 2
__device__ __forceinline__ void mul2(const double M[2][2], double v0, double v1, double& o0, double& o1) {
  double s = 0.0;
  s = s + M[0][0] * v0;
  s = s + M[0][1] * v1;
  o0 = s;
  s = 0.0;
  s = s + M[1][0] * v0;
  s = s + M[1][1] * v1;
  o1 = s;
}

// functions/anisotropy_01.h:30-48 (z component is 0 in 2D: dropping its +0.0
// terms is exact because the sums are non-negative)
__device__ __forceinline__ double aniso_ac(double dab, double q0, double q1) {
  const double qx2 = q0 * q0, qx4 = qx2 * qx2;
  const double qy2 = q1 * q1, qy4 = qy2 * qy2;
  const double q2 = qx2 + qy2;
  if (fabs(q2) > 1.0e-15) return 1.0 - dab * (3.0 - 4.0 * (qx4 + qy4) / (q2 * q2));
  return 1.0;
}

// functions/anisotropy_01.h:9-28
__device__ __forceinline__ void aniso_dadq(double dab, double q0, double q1, double& d0, double& d1) {
  const double qx3 = q0 * q0 * q0;
  const double qy3 = q1 * q1 * q1;
  const double q2 = q0 * q0 + q1 * q1;
  const double q22 = q2 * q2;
  const double q23 = q2 * q2 * q2;
  const double q4 = qx3 * q0 + qy3 * q1;
  if (fabs(q2) > 1.0e-15) {
    d0 = 16.0 * dab * (qx3 / q22 - q0 * q4 / q23);
    d1 = 16.0 * dab * (qy3 / q22 - q1 * q4 / q23);
  } else {
    d0 = 0.0;
    d1 = 0.0;
  }
}

// Gradient record fields around one Delta-phi cell (calculate_gradients.h:92-131):
// the centre's full record and the parts of the four neighbours' records that
// the phase-field terms read.
template <int N>
struct Grads {
  double gx[N], gy[N], sx[N], sy[N], cx[N], cy[N];  // centre (x, y)
  double b_gx[N], b_sx[N], b_cy[N];                   // back   (x-1, y)
  double f_cy[N];                                     // front  (x+1, y)
  double l_gy[N], l_sy[N], l_cx[N];                   // left   (x, y-1)
  double r_cx[N];                                     // right  (x, y+1)
};

// P[i][j][a] = phi_a at (x+i-1, y+j-1)
template <int N>
__device__ __forceinline__ void make_grads(const gp_model& m, const double (&P)[3][3][N], double two_dy, Grads<N>& G) {
#pragma unroll
  for (int a = 0; a < N; a++) {
    G.gx[a] = gp_ddiv((P[2][1][a] - P[1][1][a]), m.dx);
    G.sx[a] = 0.5 * (P[2][1][a] + P[1][1][a]);
    G.gy[a] = gp_ddiv((P[1][2][a] - P[1][1][a]), m.dy);
    G.sy[a] = 0.5 * (P[1][2][a] + P[1][1][a]);
    G.cy[a] = gp_ddiv((P[1][2][a] - P[1][0][a]), two_dy);
    G.b_gx[a] = gp_ddiv((P[1][1][a] - P[0][1][a]), m.dx);
    G.cx[a] = 0.5 * (G.gx[a] + G.b_gx[a]);
    G.b_sx[a] = 0.5 * (P[1][1][a] + P[0][1][a]);
    G.b_cy[a] = gp_ddiv((P[0][2][a] - P[0][0][a]), two_dy);
    G.f_cy[a] = gp_ddiv((P[2][2][a] - P[2][0][a]), two_dy);
    G.l_gy[a] = gp_ddiv((P[1][1][a] - P[1][0][a]), m.dy);
    G.l_sy[a] = 0.5 * (P[1][1][a] + P[1][0][a]);
    G.l_cx[a] = 0.5 * (gp_ddiv((P[2][0][a] - P[1][0][a]), m.dx) + gp_ddiv((P[1][0][a] - P[0][0][a]), m.dx));
    G.r_cx[a] = 0.5 * (gp_ddiv((P[2][2][a] - P[1][2][a]), m.dx) + gp_ddiv((P[1][2][a] - P[0][2][a]), m.dx));
  }
}

// dA/dphi_a and div(dA/dgrad phi_a)
//   isotropic:   functions/function_A_00.h:4-58
//   anisotropic: functions/function_A_01.h:4-71, 101-219 with functionQ.h:4-72
template <int N>
__device__ __forceinline__ double grad_energy_term(const gp_model& m, const double* phi, const Grads<N>& G, int a,
                                                   bool iso = false) {
  if (!m.anisotropy || iso) {
    double sum = 0.0;
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a) continue;
      double sp = 0.0;
      sp += (phi[a] * G.cx[b] - phi[b] * G.cx[a]) * G.cx[b];
      sp += (phi[a] * G.cy[b] - phi[b] * G.cy[a]) * G.cy[b];
      sp *= m.Gamma[a][b];
      sum += sp;
    }
    const double dA = 2.0 * sum;
    sum = 0.0;
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a) continue;
      double dv;
      dv = gp_ddiv(((G.sx[a] * G.gx[b] - G.sx[b] * G.gx[a]) * (-G.sx[b]) -
            ((G.b_sx[a] * G.b_gx[b] - G.b_sx[b] * G.b_gx[a]) * (-G.b_sx[b]))), m.dx);
      dv += gp_ddiv(((G.sy[a] * G.gy[b] - G.sy[b] * G.gy[a]) * (-G.sy[b]) -
             ((G.l_sy[a] * G.l_gy[b] - G.l_sy[b] * G.l_gy[a]) * (-G.l_sy[b]))), m.dy);
      dv *= m.Gamma[a][b];
      sum += dv;
    }
    const double divA = 2.0 * sum;
    return -dA + divA;
  }
  // anisotropic
  double s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++) {
    if (b == a) continue;
    const double gam = m.Gamma[a][b], dab = m.dab[a][b];
    double q0, q1, d0, d1, r0, r1;
    mul2(m.R[a][b], (phi[a] * G.cx[b] - phi[b] * G.cx[a]), (phi[a] * G.cy[b] - phi[b] * G.cy[a]), q0, q1);
    aniso_dadq(dab, q0, q1, d0, d1);
    const double q2 = (q0 * q0 + q1 * q1);
    const double ac1 = aniso_ac(dab, q0, q1);
    const double ac2 = ac1 * ac1;
    mul2(m.R[a][b], G.cx[b], G.cy[b], r0, r1);
    double sp1 = 0.0, sp2 = 0.0;
    sp1 += q0 * r0;
    sp1 += q1 * r1;
    sp2 += (d0)*r0;
    sp2 += (d1)*r1;
    sp1 *= gam * ac2;
    sp2 *= gam * ac1 * q2;
    s1 += sp1;
    s2 += sp2;
  }
  const double dA = 2.0 * (s1 + s2);
  s1 = 0.0;
  s2 = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++) {
    if (b == a) continue;
    const double gam = m.Gamma[a][b], dab = m.dab[a][b];
    double qf0, qf1, qb0, qb1, qr0, qr1, ql0, ql1;
    mul2(m.R[a][b], (G.sx[a] * G.gx[b] - G.sx[b] * G.gx[a]),
         0.5 * (G.sx[a] * (G.cy[b] + G.f_cy[b]) - G.sx[b] * (G.cy[a] + G.f_cy[a])), qf0, qf1);
    mul2(m.R[a][b], (G.b_sx[a] * G.b_gx[b] - G.b_sx[b] * G.b_gx[a]),
         0.5 * (G.b_sx[a] * (G.b_cy[b] + G.cy[b]) - G.b_sx[b] * (G.b_cy[a] + G.cy[a])), qb0, qb1);
    mul2(m.R[a][b], 0.5 * (G.sy[a] * (G.cx[b] + G.r_cx[b]) - G.sy[b] * (G.cx[a] + G.r_cx[a])),
         (G.sy[a] * G.gy[b] - G.sy[b] * G.gy[a]), qr0, qr1);
    mul2(m.R[a][b], 0.5 * (G.l_sy[a] * (G.l_cx[b] + G.cx[b]) - G.l_sy[b] * (G.l_cx[a] + G.cx[a])),
         (G.l_sy[a] * G.l_gy[b] - G.l_sy[b] * G.l_gy[a]), ql0, ql1);
    const double acf = aniso_ac(dab, qf0, qf1), acf2 = acf * acf;
    const double acb = aniso_ac(dab, qb0, qb1), acb2 = acb * acb;
    const double acr = aniso_ac(dab, qr0, qr1), acr2 = acr * acr;
    const double acl = aniso_ac(dab, ql0, ql1), acl2 = acl * acl;
    double d1;
    d1 = gp_ddiv(((acf2 * (G.sx[a] * G.gx[b] - G.sx[b] * G.gx[a]) * (-G.sx[b])) -
          (acb2 * (G.b_sx[a] * G.b_gx[b] - G.b_sx[b] * G.b_gx[a]) * (-G.b_sx[b]))), m.dx);
    d1 += gp_ddiv(((acr2 * (G.sy[a] * G.gy[b] - G.sy[b] * G.gy[a]) * (-G.sy[b])) -
           (acl2 * (G.l_sy[a] * G.l_gy[b] - G.l_sy[b] * G.l_gy[a]) * (-G.l_sy[b]))), m.dy);
    d1 *= gam;
    s1 += d1;
    double e0, e1, rf0, rf1, rb0, rb1, rr0, rr1, rl0, rl1;
    aniso_dadq(dab, qf0, qf1, e0, e1);
    mul2(m.Rinv[a][b], e0, e1, rf0, rf1);
    const double qf2 = qf0 * qf0 + qf1 * qf1;
    aniso_dadq(dab, qb0, qb1, e0, e1);
    mul2(m.Rinv[a][b], e0, e1, rb0, rb1);
    const double qb2 = qb0 * qb0 + qb1 * qb1;
    aniso_dadq(dab, qr0, qr1, e0, e1);
    mul2(m.Rinv[a][b], e0, e1, rr0, rr1);
    const double qr2 = qr0 * qr0 + qr1 * qr1;
    aniso_dadq(dab, ql0, ql1, e0, e1);
    mul2(m.Rinv[a][b], e0, e1, rl0, rl1);
    const double ql2 = ql0 * ql0 + ql1 * ql1;
    (void)rf1; (void)rb1; (void)rr0; (void)rl0;
    double d2;
    d2 = gp_ddiv((acf * qf2 * rf0 * (-G.sx[b]) - acb * qb2 * rb0 * (-G.b_sx[b])), m.dx);
    d2 += gp_ddiv((acr * qr2 * rr1 * (-G.sy[b]) - acl * ql2 * rl1 * (-G.l_sy[b])), m.dy);
    d2 *= gam;
    s2 += d2;
  }
  const double divA = (2.0 * (s1 + s2) + 0.0);
  return -dA + divA;
}

// dw/dphi_a: obstacle functions/functionW_01.h:6-39, well functionW_02.h:4-33
template <int N>
__device__ __forceinline__ double dwdphi(const gp_model& m, const double* phi, const double* divphi, int a) {
  double sum = 0.0;
  if (m.obstacle) {
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      if ((phi[a] * phi[b]) >= 0.00000) sum += m.Gamma[a][b] * (phi[b]);
      else sum += -m.Gamma[a][b] * (phi[b]);
    }
    sum *= m.w_obstacle;
  } else {
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += 2.0 * m.Gamma[a][b] * (phi[b] * phi[b] * phi[a]);
    }
    sum *= 9.0;
  }
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = b + 1; c < N; c++) {
      if (b == a || c == a) continue;
      if (fabs(divphi[b]) > 0.0 && fabs(divphi[c]) > 0.0) {
        const double pbc = phi[b] * phi[c];
        if (phi[a] * pbc >= 0.00000) sum += m.Gamma_abc[a][b][c] * pbc;
        else sum += -m.Gamma_abc[a][b][c] * pbc;
      }
    }
  return sum;
}

// dw/dphi of the smoothing pre-steps with anisotropy: functionW_01.h:41-62,
// functionW_02.h:35-59 (no sign factors)
template <int N>
__device__ __forceinline__ double dwdphi_smooth(const gp_model& m, const double* phi, const double* divphi, int a) {
  double sum = 0.0;
  if (m.obstacle) {
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += m.Gamma[a][b] * phi[b];
    }
    sum *= m.w_obstacle;
  } else {
#pragma unroll
    for (int b = 0; b < N; b++) {
      if (b == a || !(fabs(divphi[b]) > 0.0)) continue;
      sum += 2.0 * m.Gamma[a][b] * (phi[b] * phi[b] * phi[a]);
    }
    sum *= 9.0;
  }
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = b + 1; c < N; c++) {
      if (b == a || c == a) continue;
      if (fabs(divphi[b]) > 0.0 && fabs(divphi[c]) > 0.0) sum += m.Gamma_abc[a][b][c] * phi[b] * phi[c];
    }
  return sum;
}

// functions/functionTau.h:1-16
template <int N>
__device__ __forceinline__ double tau_phi(const gp_model& m, const double* phi) {
  double sum = 0.0, sum1 = 0.0;
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int b = a + 1; b < N; b++) {
      sum += m.tau_ab[a][b] * phi[a] * phi[b];
      sum1 += phi[a] * phi[b];
    }
  if (sum1 != 0.0 || sum1 != sum1) return sum / sum1;
  return m.tau;
}

// solverloop/simplex_projection.h:1-49
template <int N>
__device__ __forceinline__ void project_simplex(const double* phi, const double* divphi, double* dp) {
  double Deltaphi = 0.0, sum_phib = 0.0;
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if ((fabs(divphi[a]) > 0.0) && (phi[a] + dp[a]) > 0.0 && (phi[a] + dp[a]) < 1.0) {
      count++;
      sum_phib += phi[a];
    }
#pragma unroll
  for (int a = 0; a < N; a++)
    if ((phi[a] + dp[a]) < 0.0) {
      const double over = fabs(dp[a] + phi[a]);
      dp[a] += over;
      Deltaphi += over;
    }
  if (Deltaphi > 0.0) {
#pragma unroll
    for (int b = 0; b < N; b++)
      if ((fabs(divphi[b]) > 0.0) && ((phi[b] + dp[b]) > 0.0) && ((phi[b] + dp[b]) < 1.0)) {
        if (fabs(sum_phib) > 0.0) dp[b] -= Deltaphi * (phi[b]) / (sum_phib);
        else dp[b] -= gp_ddiv(Deltaphi, (double)(count));
      }
  }
  int hit = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (hit < 0 && fabs(divphi[a]) > 0.0 && (phi[a] + dp[a]) > 1.0) hit = a;
  if (hit >= 0) {
#pragma unroll
    for (int a = 0; a < N; a++)
      if (a == hit) dp[a] = (1.0 - phi[a]);
#pragma unroll
    for (int b = 0; b < N; b++)
      if ((fabs(divphi[b]) > 0.0) && b != hit) dp[b] = -phi[b];
  }
}

// projection of the smoothing pre-steps, solverloop/simplex_projection.h:50-91
template <int N>
__device__ __forceinline__ void project_simplex_unweighted(const double* phi, const double* divphi, double* dp) {
  long count = 0;
#pragma unroll
  for (int a = 0; a < N; a++)
    if ((fabs(divphi[a]) > 0.0) && (phi[a] + dp[a]) > 0.0 && (phi[a] + dp[a]) < 1.0) count++;
  for (int a = 0; a < N; a++) {
    if (!(fabs(divphi[a]) > 0.0)) continue;
    if ((phi[a] + dp[a]) > 1.0) {
      dp[a] = (1.0 - phi[a]);
#pragma unroll
      for (int b = 0; b < N; b++)
        if ((fabs(divphi[b]) > 0.0) && b != a) dp[b] = -phi[b];
      break;
    }
    if ((phi[a] + dp[a]) < 0.0) {
      const double D = fabs(dp[a] + phi[a]);
      dp[a] += D;
#pragma unroll
      for (int b = 0; b < N; b++)
        if (((fabs(divphi[b]) > 0.0) && b != a) && (phi[b] + dp[b]) > 0.0 && (phi[b] + dp[b]) < 1.0)
          dp[b] -= gp_ddiv(D, (double)(count));
    }
  }
}

// True when the 3x3 phi block around a cell holds one value per phase and that value lies in
// [0, 1] (so no NaN, infinity or negative value).  Every phi gradient of such a cell is then
// +0 or -0: no phase is active (|divphi| = 0), the projection changes nothing, Delta-phi is
// +0, and no face next to the cell carries an antitrapping current (each face's |grad phi| is
// 0).  The kernels skip that arithmetic for such cells and store what it would give.
template <int N>
__device__ __forceinline__ bool flat_block(const double (&P)[3][3][N]) {
  bool flat = true;
#pragma unroll
  for (int a = 0; a < N; a++) {
    const double c = P[1][1][a];
    flat = flat && c >= 0.0 && c <= 1.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) flat = flat && P[i][j][a] == c;
  }
  return flat;
}

// ---------------------------------------------------------------- kernels

// Blocks of 256 per SM the kernels are compiled for: three for binary alloys (80 registers; the
// compiler spills some of the interface cells' state, and the occupancy gained pays for it on many
// small grids stepped at once, with no loss on one large grid), two for the other two-phase
// kernels, one beyond (two of those spill heavily).
#define GP_F64_BLOCKS(N, K1) ((N) == 2 && (K1) == 1 ? 3 : ((N) == 2 ? 2 : 1))

// Delta-phi on [-1, mx] x [-1, my] (interior plus the first ghost ring).
// SMOOTH: the smoothing pre-step (calculate_divergence_phasefield.h:63-158):
// isotropic gradient energy, no dpsi, the unsigned potential when anisotropic,
// unweighted projection.
template <int N, int K1, bool SMOOTH>
__global__ void __launch_bounds__(256, GP_F64_BLOCKS(N, K1)) k_dphi(const __grid_constant__ gp_model m, Geo g,
                                              const double* __restrict__ phi, const double* __restrict__ mu,
                                              double* __restrict__ dphi) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int x = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (x > g.mx || y > g.my) return;
  double P[3][3][N];
  load_block<N>(phi, g, x, y, P);
  double* out = dphi + (int64_t)(x + 1) * g.rpitch + (y + 1);
  if (flat_block<N>(P)) {  // no active phase: Delta-phi is +0
#pragma unroll
    for (int a = 0; a < N; a++) out[a * g.rplane] = 0.0;
    return;
  }
  double muc[K1];
  load_mu<K1>(mu, g, x, y, muc, N);
  const double two_dy = 2.0 * m.dy;
  Grads<N> G;
  make_grads<N>(m, P, two_dy, G);
  const double* ph = P[1][1];
  double divphi[N], lambda[N], dp[N];
#pragma unroll
  for (int a = 0; a < N; a++) {
    divphi[a] = gp_ddiv((G.gx[a] - G.b_gx[a]), m.dx);
    divphi[a] += gp_ddiv((G.gy[a] - G.l_gy[a]), m.dy);
  }
  double sum_lambda = 0.0;
  long active = 0;
#pragma unroll
  for (int a = 0; a < N; a++) {
    lambda[a] = 0.0;
    if (fabs(divphi[a]) > 0.0) {
      const double t = grad_energy_term<N>(m, ph, G, a, SMOOTH);
      if (SMOOTH)
        lambda[a] = m.epsilon * (t) - m.inv_eps * (m.anisotropy ? dwdphi_smooth<N>(m, ph, divphi, a)
                                                                : dwdphi<N>(m, ph, divphi, a));
      else
        lambda[a] = m.epsilon * (t) - m.inv_eps * dwdphi<N>(m, ph, divphi, a) -
                    dpsi<N, K1>(m, th_row(m, g, y, g.t_linear), muc, ph, a);
      sum_lambda += lambda[a];
      active++;
    }
  }
  if (active) sum_lambda = gp_ddiv(sum_lambda, (double)active);
  const double tphi = tau_phi<N>(m, ph);
#pragma unroll
  for (int a = 0; a < N; a++) {
    if (fabs(divphi[a]) > 0.0) dp[a] = m.dt * (lambda[a] - sum_lambda) / (tphi * m.epsilon);
    else dp[a] = 0.0;
  }
  if (SMOOTH) project_simplex_unweighted<N>(ph, divphi, dp);
  else project_simplex<N>(ph, divphi, dp);
#pragma unroll
  for (int a = 0; a < N; a++) out[a * g.rplane] = dp[a];
}

// s(phi) of the obstacle antitrapping term, calculate_fluxes_concentration.h:43-59
template <int N>
__device__ __forceinline__ double s_obstacle(const double* phi, int a) {
  if (phi[a] * (1.0 - phi[a]) > 0.0) return phi[a] * (1.0 - hphi<N>(phi, a)) / (sqrt(phi[a] * (1.0 - phi[a])));
  return 0.0;
}

// Antitrapping current through the face between cell c and its neighbour n
// (n = front for an x-face, right for a y-face), one component set:
// calculate_fluxes_concentration.h:25-141.  gn: forward difference across the
// face per phase; t_c, t_n: the tangential centred gradient of c and n.
template <int N, int K1>
__device__ __forceinline__ void jat_face(const gp_model& m, const double* gn, const double* t_c, const double* t_n,
                                         const double* ph_c, const double* ph_n, const double* mu_c,
                                         const double* mu_n, const double* dp_c, const double* dp_n, bool skip,
                                         double* j, Th th_c, Th th_n) {
  constexpr int L = N - 1;
  const double tl = 0.5 * (t_c[L] + t_n[L]);
  const double norm_l = sqrt(tl * tl + gn[L] * gn[L]);
#pragma unroll
  for (int k = 0; k < K1; k++) j[k] = 0.0;
#pragma unroll
  for (int a = 0; a < N - 1; a++) {
    const double ta = 0.5 * (t_c[a] + t_n[a]);
    const double normg = sqrt(ta * ta + gn[a] * gn[a]);
    double s_n = 0.0, s_c = 0.0;
    if (m.obstacle) {
      s_n = s_obstacle<N>(ph_n, a);
      s_c = s_obstacle<N>(ph_c, a);
    }
#pragma unroll
    for (int k = 0; k < K1; k++) {
      if (normg != 0.0 && !skip) {
        const double cl_n = c_mu<K1>(m, th_n, mu_n, L, k), cl_c = c_mu<K1>(m, th_c, mu_c, L, k);
        const double cs_n = c_mu<K1>(m, th_n, mu_n, a, k), cs_c = c_mu<K1>(m, th_c, mu_c, a, k);
        double sp = gn[a] * gn[L];
        sp += ta * tl;
        if (norm_l > 0.0) sp /= (norm_l * normg);
        const double f = (1.0 - m.Diff[a][k][k] / m.Diff[L][k][k]);
        if (m.obstacle)
          j[k] += f * fabs(sp) * 0.5 * (s_n * (cl_n - cs_n) * dp_n[a] + s_c * (cl_c - cs_c) * dp_c[a]) * gn[a] / normg;
        else
          j[k] += f * fabs(sp) * m.s_well * ((cl_n - cs_n) * dp_n[a] + (cl_c - cs_c) * dp_c[a]) * gn[a] / normg;
      }
    }
  }
}

// phi-weighted mobility of one cell, functions/functionD.h:1-16
template <int N, int K1>
__device__ __forceinline__ double Dcell(const gp_model& m, const double* phi, int i, int j) {
  double sum = 0.0;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int k = 0; k < K1; k++) sum += m.Diff[b][i][k] * m.cmu[b][k][j] * phi[b];
  return sum;
}

// LU inverse of the reference (functions/matrix.h:50-114) for the general mu solve.
template <int K>
__device__ __forceinline__ void lu_inverse(double (&mm)[K][K], double (&inv)[K][K]) {
  double fac[K][K], inv1[K][K];
  int tag[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    tag[k] = k;
#pragma unroll
    for (int j = 0; j < K; j++) fac[k][j] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < K; k++) {
    double big = fabs(mm[k][k]);
    int t1 = k;
#pragma unroll
    for (int i = k + 1; i < K; i++)
      if (fabs(mm[i][k]) > big) { t1 = i; big = mm[i][k]; }
    // swap tag[k] <-> tag[t1], rows k <-> t1 of mm, and fac[.][0..k-1]
#pragma unroll
    for (int i = k + 1; i < K; i++) {
      if (i == t1) {
        int ts = tag[k]; tag[k] = tag[i]; tag[i] = ts;
#pragma unroll
        for (int c = 0; c < K; c++) { double s = mm[k][c]; mm[k][c] = mm[i][c]; mm[i][c] = s; }
#pragma unroll
        for (int c = 0; c < k; c++) { double s = fac[k][c]; fac[k][c] = fac[i][c]; fac[i][c] = s; }
      }
    }
#pragma unroll
    for (int i = k + 1; i < K; i++) {
      const double f = -mm[i][k] / mm[k][k];
      fac[i][k] = -f;
#pragma unroll
      for (int j = k; j <= K - 1; j++) mm[i][j] = f * mm[k][j] + mm[i][j];
    }
  }
#pragma unroll
  for (int i = 0; i < K; i++)
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (i == j) fac[i][j] = 1;
      if (j > i) fac[i][j] = 0;
    }
#pragma unroll
  for (int i = 0; i < K; i++) {
    double v1[K], v[K];
    v1[0] = (i == 0) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 1; k < K; k++) {
      double s = 0;
#pragma unroll
      for (int j = 0; j < k; j++) s = s - fac[k][j] * v1[j];
      v1[k] = ((k == i) ? 1.0 : 0.0) + s;
    }
    // pow(x, -1) of the reference equals the correctly rounded 1/x
    v[K - 1] = v1[K - 1] * (1.0 / mm[K - 1][K - 1]);
#pragma unroll
    for (int k = K - 2; k >= 0; k--) {
      double s = 0;
#pragma unroll
      for (int j = k + 1; j < K; j++) s = s - mm[k][j] * v[j];
      v[k] = (v1[k] + s) * (1.0 / mm[k][k]);
    }
#pragma unroll
    for (int j = 0; j < K; j++) inv1[j][i] = v[j];
  }
#pragma unroll
  for (int j = 0; j < K; j++)
#pragma unroll
    for (int t = 0; t < K; t++)
      if (tag[j] == t) {
#pragma unroll
        for (int k = 0; k < K; k++) inv[k][t] = inv1[k][j];
      }
}

// mu and phi update of the interior.  SMOOTH: the smoothing pre-step
// (calculate_divergence_concentration.h:154-253): no antitrapping current, no
// dh/dt source, the LU inverse (matinvnew) for every mu solve.
template <int N, int K1, bool SMOOTH>
__global__ void __launch_bounds__(256, GP_F64_BLOCKS(N, K1)) k_update(const __grid_constant__ gp_model m, Geo g,
                                                const double* __restrict__ phi, const double* __restrict__ mu,
                                                const double* __restrict__ dphi, double* __restrict__ phi_out,
                                                double* __restrict__ mu_out) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  const int x = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.mx || y >= g.my) return;
  double P[3][3][N];
  load_block<N>(phi, g, x, y, P);
  double Mc[K1], Mb[K1], Mf[K1], Ml[K1], Mr[K1];
  if (x >= 1 && x <= g.mx - 2 && y >= 1 && y <= g.my - 2) {  // the four neighbours inside the grid
    const double* q = mu + (int64_t)x * g.pitch + y;
#pragma unroll
    for (int k = 0; k < K1; k++) {
      Mc[k] = __ldg(q + k * g.plane);
      Mb[k] = __ldg(q + k * g.plane - g.pitch);
      Mf[k] = __ldg(q + k * g.plane + g.pitch);
      Ml[k] = __ldg(q + k * g.plane - 1);
      Mr[k] = __ldg(q + k * g.plane + 1);
    }
  } else {
    load_mu<K1>(mu, g, x, y, Mc);
    load_mu<K1>(mu, g, x - 1, y, Mb);
    load_mu<K1>(mu, g, x + 1, y, Mf);
    load_mu<K1>(mu, g, x, y - 1, Ml);
    load_mu<K1>(mu, g, x, y + 1, Mr);
  }
  double Dc[N], Db[N], Df[N], Dl[N], Dr[N];
  {
    const double* r = dphi + (int64_t)(x + 1) * g.rpitch + (y + 1);
#pragma unroll
    for (int a = 0; a < N; a++) {
      Dc[a] = __ldg(r + a * g.rplane);
      Db[a] = __ldg(r + a * g.rplane - g.rpitch);
      Df[a] = __ldg(r + a * g.rplane + g.rpitch);
      Dl[a] = __ldg(r + a * g.rplane - 1);
      Dr[a] = __ldg(r + a * g.rplane + 1);
    }
  }
  // j_at on the four faces; the y-face at ghosted row MESH_Y-2 carries none
  // (calculate_fluxes_concentration.h:65), i.e. interior row my-5.  A flat phi block
  // carries none on any face (flat_block).
  double jx_c[K1], jx_b[K1], jy_c[K1], jy_l[K1];
#pragma unroll
  for (int k = 0; k < K1; k++) jx_c[k] = jx_b[k] = jy_c[k] = jy_l[k] = 0.0;
  // the cells' temperatures in the concentration half step (ghosts: their boundary copy)
  const Th thc = th_row(m, g, y, false), thl = th_row(m, g, y - 1, false), thr = th_row(m, g, y + 1, false);
  if (!SMOOTH && !flat_block<N>(P)) {
    const double two_dy = 2.0 * m.dy;
    // gradient pieces the four faces need (calculate_gradients.h:92-131)
    double gx_c[N], gx_b[N], gy_c[N], gy_l[N];
    double cy_c[N], cy_b[N], cy_f[N], cx_c[N], cx_l[N], cx_r[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      gx_c[a] = gp_ddiv((P[2][1][a] - P[1][1][a]), m.dx);
      gx_b[a] = gp_ddiv((P[1][1][a] - P[0][1][a]), m.dx);
      gy_c[a] = gp_ddiv((P[1][2][a] - P[1][1][a]), m.dy);
      gy_l[a] = gp_ddiv((P[1][1][a] - P[1][0][a]), m.dy);
      cy_c[a] = gp_ddiv((P[1][2][a] - P[1][0][a]), two_dy);
      cy_b[a] = gp_ddiv((P[0][2][a] - P[0][0][a]), two_dy);
      cy_f[a] = gp_ddiv((P[2][2][a] - P[2][0][a]), two_dy);
      cx_c[a] = 0.5 * (gx_c[a] + gx_b[a]);
      cx_l[a] = 0.5 * (gp_ddiv((P[2][0][a] - P[1][0][a]), m.dx) + gp_ddiv((P[1][0][a] - P[0][0][a]), m.dx));
      cx_r[a] = 0.5 * (gp_ddiv((P[2][2][a] - P[1][2][a]), m.dx) + gp_ddiv((P[1][2][a] - P[0][2][a]), m.dx));
    }
    jat_face<N, K1>(m, gx_c, cy_c, cy_f, P[1][1], P[2][1], Mc, Mf, Dc, Df, false, jx_c, thc, thc);
    jat_face<N, K1>(m, gx_b, cy_b, cy_c, P[0][1], P[1][1], Mb, Mc, Db, Dc, false, jx_b, thc, thc);
    jat_face<N, K1>(m, gy_c, cx_c, cx_r, P[1][1], P[1][2], Mc, Mr, Dc, Dr, (y + 3 == g.my - 2), jy_c, thc, thr);
    jat_face<N, K1>(m, gy_l, cx_l, cx_c, P[1][0], P[1][1], Ml, Mc, Dl, Dc, (y + 2 == g.my - 2) || (y + 2 == 0),
                    jy_l, thl, thc);
  }

  const double* ph = P[1][1];
  double sum[K1], divflux[K1], divjat[K1], deltac[K1], dcdmu[K1][K1];
#pragma unroll
  for (int k = 0; k < K1; k++) {
    sum[k] = 0.0;
#pragma unroll
    for (int l = 0; l < K1; l++) dcdmu[k][l] = 0.0;
  }
#pragma unroll
  for (int a = 0; a < N; a++) {
    double sdh = 0.0;
#pragma unroll
    for (int b = 0; b < N; b++) sdh += dhphi<N>(ph, a, b) * Dc[b];
#pragma unroll
    for (int k = 0; k < K1; k++) sum[k] += c_mu<K1>(m, thc, Mc, a, k) * sdh;
  }
  const double jscale = m.obstacle ? m.jat_obst : m.jat_well;
#pragma unroll
  for (int k = 0; k < K1; k++) {
    divflux[k] = 0.0;
#pragma unroll
    for (int l = 0; l < K1; l++) {
      const double Dcc = Dcell<N, K1>(m, ph, k, l);
      const double Dx = (Dcell<N, K1>(m, P[2][1], k, l) + Dcc) * 0.5;
      const double Dxb = (Dcc + Dcell<N, K1>(m, P[0][1], k, l)) * 0.5;
      const double Dy = (Dcell<N, K1>(m, P[1][2], k, l) + Dcc) * 0.5;
      const double Dyl = (Dcc + Dcell<N, K1>(m, P[1][0], k, l)) * 0.5;
      const double gmx = gp_ddiv((Mf[l] - Mc[l]), m.dx);
      const double gmxb = gp_ddiv((Mc[l] - Mb[l]), m.dx);
      const double gmy = gp_ddiv((Mr[l] - Mc[l]), m.dy);
      const double gmyl = gp_ddiv((Mc[l] - Ml[l]), m.dy);
      divflux[k] += gp_ddiv((Dx * gmx - Dxb * gmxb), m.dx);
      divflux[k] += gp_ddiv((Dy * gmy - Dyl * gmyl), m.dy);
    }
    if (!SMOOTH) {
      divjat[k] = gp_ddiv((jx_c[k] - jx_b[k]) * (jscale), m.dx);
      divjat[k] += gp_ddiv((jy_c[k] - jy_l[k]) * (jscale), m.dy);
    }
  }
  int bulk = -1;
#pragma unroll
  for (int a = 0; a < N; a++)
    if (bulk < 0 && ph[a] == 1.0) bulk = a;
  double mnew[K1];
  if (bulk >= 0) {
    double cnew[K1];
#pragma unroll
    for (int k = 0; k < K1; k++) {
      double co = 0.0;
#pragma unroll
      for (int a = 0; a < N; a++)
        if (a == bulk) co = c_mu<K1>(m, thc, Mc, a, k);
      cnew[k] = SMOOTH ? co + m.dt * (divflux[k]) : co + m.dt * (divflux[k]) - divjat[k];
    }
#pragma unroll
    for (int k = 0; k < K1; k++) {
      double v = 0.0;
#pragma unroll
      for (int a = 0; a < N; a++)
        if (a == bulk) v = Mu<K1>(m, thc, cnew, a, k);
      mnew[k] = v;
    }
  } else if (SMOOTH) {
#pragma unroll
    for (int k = 0; k < K1; k++) {
      deltac[k] = m.dt * (divflux[k]);
#pragma unroll
      for (int l = 0; l < K1; l++)
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += m.cmu[a][k][l] * hphi<N>(ph, a);
    }
    double inv[K1][K1];
    lu_inverse<K1>(dcdmu, inv);
#pragma unroll
    for (int k = 0; k < K1; k++) {
      double s = 0;
#pragma unroll
      for (int l = 0; l < K1; l++) s = s + inv[k][l] * deltac[l];
      mnew[k] = s + Mc[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < K1; k++) {
      deltac[k] = m.dt * (divflux[k]) - divjat[k] - sum[k];
#pragma unroll
      for (int l = 0; l < K1; l++)
#pragma unroll
        for (int a = 0; a < N; a++) dcdmu[k][l] += m.cmu[a][k][l] * hphi<N>(ph, a);
    }
#pragma unroll
    for (int k = 0; k < K1; k++) mnew[k] = Mc[k];
    if (m.mu_solver == GP_MU_BINARY) {
      const double iv = 1.0 / dcdmu[0][0];
      mnew[0] = Mc[0] + deltac[0] * iv;
    } else if (m.mu_solver == GP_MU_TERNARY && K1 == 2) {
      const double DET = dcdmu[0][0] * dcdmu[K1 - 1][K1 - 1] - dcdmu[0][K1 - 1] * dcdmu[K1 - 1][0];
      double inv[2][2];
      inv[0][0] = dcdmu[K1 - 1][K1 - 1] / DET;
      inv[1][1] = dcdmu[0][0] / DET;
      inv[0][1] = -dcdmu[0][K1 - 1] / DET;
      inv[1][0] = -dcdmu[K1 - 1][0] / DET;
#pragma unroll
      for (int k = 0; k < K1; k++) {
        double dm = 0.0;
#pragma unroll
        for (int l = 0; l < K1; l++) dm += inv[k & 1][l & 1] * deltac[l];
        mnew[k] = dm + Mc[k];
      }
    } else if (m.mu_solver == GP_MU_DILUTE) {
#pragma unroll
      for (int k = 0; k < K1; k++) {
        const double iv = 1.0 / dcdmu[k][k];
        mnew[k] = Mc[k] + deltac[k] * iv;
      }
    } else {
      double inv[K1][K1];
      lu_inverse<K1>(dcdmu, inv);
#pragma unroll
      for (int k = 0; k < K1; k++) {
        double s = 0;
#pragma unroll
        for (int l = 0; l < K1; l++) s = s + inv[k][l] * deltac[l];
        mnew[k] = s + Mc[k];
      }
    }
  }
  const int64_t o = (int64_t)x * g.pitch + y;
#pragma unroll
  for (int k = 0; k < K1; k++) mu_out[o + k * g.plane] = mnew[k];
#pragma unroll
  for (int a = 0; a < N; a++) phi_out[o + a * g.plane] = ph[a] + Dc[a];
}

template <int N, int K1, bool SMOOTH>
cudaError_t launch_step(const gp_model& m, const Geo& g, const double* phi, const double* mu, double* dphi,
                        double* phi_out, double* mu_out, cudaStream_t s) {
  const dim3 blk(32, 8);
  const dim3 grd_r((g.my + 2 + 31) / 32, (g.mx + 2 + 7) / 8);
  k_dphi<N, K1, SMOOTH><<<grd_r, blk, 0, s>>>(m, g, phi, mu, dphi);
  const dim3 grd((g.my + 31) / 32, (g.mx + 7) / 8);
  Geo gu = g;
  gu.gov = nullptr;  // the concentration half step reads refreshed ghosts
  k_update<N, K1, SMOOTH><<<grd, blk, 0, s>>>(m, gu, phi, mu, dphi, phi_out, mu_out);
  return cudaGetLastError();
}

}  // namespace

// Host entry used by the C ABI (gp_capi.cu).  Two launches per step.
cudaError_t gp_f64_step(const gp_model& m, int pitch, int64_t plane, int rpitch, int64_t rplane,
                        const double* phi, const double* mu, double* dphi, double* phi_out, double* mu_out,
                        cudaStream_t s, bool smooth, const double* ghost_rows, const gp_temp_step* temp) {
  if (m.nonisothermal && !temp) return cudaErrorInvalidValue;  // the step needs its temperature
  Geo g;
  g.noniso = m.nonisothermal ? 1 : 0;
  g.t_linear = temp ? temp->linear : 0;
  g.bc_t = m.bc_T[3];
  g.t_bottom = temp ? temp->bottom : 0.0;
  g.t_grad = temp ? temp->grad : 0.0;
  g.mx = (int)m.mesh_x;
  g.my = (int)m.mesh_y;
  g.pitch = pitch;
  g.plane = plane;
  g.rpitch = rpitch;
  g.rplane = rplane;
  g.bc = gp_bc_of(m);
  g.gov = ghost_rows;
#define GP_CASE(NN, KK)                                                                           \
  if (m.N == NN && m.K1 == KK)                                                                    \
    return smooth ? launch_step<NN, KK, true>(m, g, phi, mu, dphi, phi_out, mu_out, s)            \
                  : launch_step<NN, KK, false>(m, g, phi, mu, dphi, phi_out, mu_out, s);
  GP_CASE(2, 1) GP_CASE(2, 2) GP_CASE(2, 3)
  GP_CASE(3, 1) GP_CASE(3, 2) GP_CASE(3, 3)
  GP_CASE(4, 1) GP_CASE(4, 2) GP_CASE(4, 3)
  GP_CASE(5, 1) GP_CASE(5, 2) GP_CASE(5, 3)
  GP_CASE(6, 1) GP_CASE(6, 2) GP_CASE(6, 3)
#undef GP_CASE
  return cudaErrorInvalidValue;
}
