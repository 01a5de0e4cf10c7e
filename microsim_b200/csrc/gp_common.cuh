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
