// gp_common.cuh -- shared device helpers of the grand-potential step kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gp_b200.h"

// Ghost layers are not stored.  The reference fills them after every half
// step by plane copies (solverloop/boundary_serial.h:176-203, index tables
// functions/utility_functions.h:471-653): first the x faces over whole
// y-columns, then the y faces over every x.  For the Neumann (1) and periodic
// (3) copies that composition is a pure index map of interior cells:
//   ghost (x, y) == interior (map_x(x), map_y(y)),  x, y in [-3, M+2]
// Neumann mirrors about the first/last interior cell (-1 -> 1, M -> M-2);
// the reference's periodic copy uses period M-1 (-1 -> M-2, M -> 1).
__host__ __device__ __forceinline__ int gp_map(int v, int M, int type) {
  if (v < 0) return type == GP_BC_NEUMANN ? -v : M - 1 + v;
  if (v >= M) return type == GP_BC_NEUMANN ? 2 * M - 2 - v : 1 + v - M;
  return v;
}

// gp_map for coordinates that may lie anywhere beyond the grid (halo cells of
// partial edge tiles, whose values no interior cell uses): clamped into
// [-3, M+2] first so every load stays inside the interior.
__host__ __device__ __forceinline__ int gp_map_any(int v, int M, int type) {
  v = v < -3 ? -3 : (v > M + 2 ? M + 2 : v);
  return gp_map(v, M, type);
}

// Per-field, per-axis copy types.  The reference forces both sides of an axis
// to periodic when either is, and the kernels accept only types 1 and 3, so one
// type per (field, axis) describes the copy.
struct gp_bc {
  int phi_x, phi_y, mu_x, mu_y;
};

static inline gp_bc gp_bc_of(const gp_model &m) {
  gp_bc b;
  b.phi_x = m.bc_phi[0];
  b.phi_y = m.bc_phi[3];
  b.mu_x = m.bc_mu[0];
  b.mu_y = m.bc_mu[3];
  return b;
}

static inline int64_t gp_round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// The frozen temperature gradient of a non-isothermal model at the start of a
// step: T of the reference's ghost-padded row gy = bottom + gy * grad.
struct gp_temp_step {
  double bottom, grad;
  int linear;  // the phase-field half step reads the ghosts' own linear T (every step after the first)
};

// temp_bottom and GRADIENT after step t (t = 0: the initial temperature), microsim_gp.c:77-82 and
// 108-113 in their operation order (no moving frame: shift_OFFSET = 0).
__host__ __device__ inline gp_temp_step gp_temp_after(const gp_model &m, int64_t t) {
  gp_temp_step s;
  const double shift_offset = 0.0;
  const double base_pos = t == 0 ? (m.tg_offset / m.dy) - shift_offset
                                 : (m.tg_offset / m.dy) - shift_offset + ((m.tg_velocity / m.dy) * ((double)t * m.dt));
  s.grad = (m.tg_deltaT) * m.dy / (m.tg_distance);
  s.bottom = m.tg_base - base_pos * s.grad;
  s.linear = t > 0;
  return s;
}

// The temperature a cell sees (functions/Temperature_gradient.h:19): on = 0 for an isothermal model
// (the model's T throughout).
struct Th {
  int on;
  double T;
};

// Beq + dBbdT (T - Teq) of phase a, component k, at the cell's temperature (the model's Beff when
// isothermal: the host folded the same expression at the model's T)
__host__ __device__ __forceinline__ double beff(const gp_model& m, Th t, int a, int k) {
  return t.on ? (m.Beq[a][k] + m.dBbdT[a][k] * (t.T - m.Teq)) : m.Beff[a][k];
}

// c_liq, c_sol of phase a at T (functions/functionF_01.h:70-71, 90-91)
__host__ __device__ __forceinline__ double c_liq_T(const gp_model& m, double T, int a, int k) {
  return m.ceq_l[a][k] - (m.dC[a][k]) * (m.Teq - T) / (m.dT_l[a]);
}
__host__ __device__ __forceinline__ double c_sol_T(const gp_model& m, double T, int a, int k) {
  return m.ceq_s[a][k] - (m.dC[a][k]) * (m.Teq - T) / (m.dT_s[a]);
}

// B(T) of phase a, component i, functions/functionF_01.h:62-80 (the model's B when isothermal)
__host__ __device__ __forceinline__ double B_T(const gp_model& m, Th t, int i, int a) {
  if (!t.on) return m.B[a][i];
  const int N = m.N, K1 = m.K1;
  double sum_c = 0.0, B_ai = 0.0;
  if (a != N - 1) {
    for (int k = 0; k < K1; k++)
      if (k != i) sum_c += m.A[N - 1][k][i] * c_liq_T(m, t.T, a, k) - m.A[a][k][i] * c_sol_T(m, t.T, a, k);
    B_ai = (2.0 * (m.A[N - 1][i][i] * c_liq_T(m, t.T, a, i) - m.A[a][i][i] * c_sol_T(m, t.T, a, i)) + sum_c);
  }
  return B_ai;
}

// C(T) of phase a, functions/functionF_01.h:82-104 (the model's C when isothermal)
__host__ __device__ __forceinline__ double C_T(const gp_model& m, Th t, int a) {
  if (!t.on) return m.C[a];
  const int N = m.N, K1 = m.K1;
  double sum_c = 0.0;
  if (a != N - 1) {
    for (int i = 0; i < K1; i++)
      for (int j = i; j < K1; j++)
        sum_c += (m.A[a][i][j] * c_sol_T(m, t.T, a, i) * c_sol_T(m, t.T, a, j) -
                  m.A[N - 1][i][j] * c_liq_T(m, t.T, a, i) * c_liq_T(m, t.T, a, j));
  }
  return sum_c;
}

// B(T), C(T) with the phase and component counts fixed at compile time (the step kernels)
template <int N, int K1>
__host__ __device__ __forceinline__ double B_Tn(const gp_model& m, Th t, int i, int a) {
  if (!t.on) return m.B[a][i];
  double sum_c = 0.0, B_ai = 0.0;
  if (a != N - 1) {
#pragma unroll
    for (int k = 0; k < K1; k++)
      if (k != i) sum_c += m.A[N - 1][k][i] * c_liq_T(m, t.T, a, k) - m.A[a][k][i] * c_sol_T(m, t.T, a, k);
    B_ai = (2.0 * (m.A[N - 1][i][i] * c_liq_T(m, t.T, a, i) - m.A[a][i][i] * c_sol_T(m, t.T, a, i)) + sum_c);
  }
  return B_ai;
}
template <int N, int K1>
__host__ __device__ __forceinline__ double C_Tn(const gp_model& m, Th t, int a) {
  if (!t.on) return m.C[a];
  double sum_c = 0.0;
  if (a != N - 1) {
#pragma unroll
    for (int i = 0; i < K1; i++)
#pragma unroll
      for (int j = i; j < K1; j++)
        sum_c += (m.A[a][i][j] * c_sol_T(m, t.T, a, i) * c_sol_T(m, t.T, a, j) -
                  m.A[N - 1][i][j] * c_liq_T(m, t.T, a, i) * c_liq_T(m, t.T, a, j));
  }
  return sum_c;
}
