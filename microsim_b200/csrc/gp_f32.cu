// gp_f32.cu -- the chosen form of the step: FP32 storage and update, one
// fused kernel per time step for a whole batch of independent instances.
//
// Same model as the plain form (gp_f64.cu, reference
// Grand_potential_Finite_difference_2D_serial/solverloop/*), restructured for
// the GPU instead of kept in the reference's evaluation order:
//  * one launch per step covers every tile of every instance of a batch
//    (instances may differ in size and parameters; they share N, K1 and the
//    anisotropy switch, which are template parameters);
//  * a block stages phi for its tile plus a 2-cell halo and mu plus a 1-cell
//    halo in shared memory; ghost cells come from the boundary index map;
//  * anisotropic gradient-energy terms are evaluated once per face and per
//    phase pair and shared by the two cells of the face and by both phases of
//    the pair (q_ba = -q_ab, a_c even, da_c/dq odd in q);
//  * Delta-phi of the tile plus one ring stays in shared memory; the mu update
//    then uses face fluxes (diffusion + antitrapping) computed once per face;
//  * reciprocals of dx, dy, 2dy are folded; the (dc/dmu)^-1 solve of
//    multicomponent cases and all statistics stay FP64.
// The reference's j_at,y skip on row gidy == MESH_Y-2
// (calculate_fluxes_concentration.h:65) is kept: it is part of the model the
// reference integrates.

#include <cuda.h>
#include <stdio.h>
#include <stddef.h>
#include <string.h>

#include <vector>

#include "gp_common.cuh"

extern "C" void gp_set_error(const char* fmt, ...);

namespace gp32 {

constexpr int MP = GP_MAX_PHASES;
constexpr int MK = GP_MAX_K1;

// FP32 model constants of one instance (built on the host from gp_model).
struct alignas(16) Model {
  float dx_inv, dy_inv, half_dy_inv, dt, eps, inv_eps, tau, w_obst, jscale, s_well;
  float hx, hy;    // dt / (2 dx^2), dt / (2 dy^2): face flux (D_c + D_n) * h * (mu_n - mu_c), net = sum of differences
  float jsx, jsy;  // antitrapping scale of an x / y face: jscale / dx, jscale / dy
  int obstacle, mu_solver, skip_row, pad;
  float Gamma[MP][MP];
  float Gabc[MP][MP][MP];
  float tau_ab[MP][MP];
  float dab[MP][MP];
  float R[MP][MP][2][2];
  float Rinv[MP][MP][2][2];
  float cmu[MP][MK][MK];
  float A[MP][MK][MK];
  float Beff[MP][MK];
  float B[MP][MK];
  float C[MP];
  float DC[MP][MK][MK];  // sum_k Diff[b][i][k] * cmu[b][k][j]: D(phi) = sum_b DC_b phi_b
  float atf[MP][MK];     // 1 - Diff[a][k][k] / Diff[N-1][k][k]
  float H[MP][MK][MK];   // d mu / d c of phase b (2 A_kk on the diagonal, A_kl off it): bulk mu += H dc
  int comp;              // compensated flux accumulation (error-free transforms, gp_batch_set_compensated)
  int pad3[3];
  float Gx[MP][MK][MK];  // pure-phase update: mu += Gx Lx + Gy Ly, Gx = H (2 DC) dt / (2 dx^2)
  float Gy[MP][MK][MK];
  float pad2[2];
  double cmu_d[MP][MK][MK];
};
static_assert(sizeof(Model) % 16 == 0, "Model is copied to shared memory as float4");

// One instance of a batch: its buffers and geometry.
struct alignas(16) Inst {
  const float* phi;
  const float* mu;
  float* phi_out;
  float* mu_out;
  int64_t plane;
  int mx, my, pitch;
  int tiles_y;     // tiles along y
  int tile_begin;  // first global tile index of this instance
  int model;       // index into the model array
  int tiles_x;     // tiles along x
  gp_bc bc;
  // non-isothermal frozen gradient (nullptr when isothermal): the instance's FP64 model and the
  // batch's step counter (the step the kernels compute; advanced after every full-kernel pass)
  const gp_model* gm;
  const long long* tstep;
};

template <int N>
struct Pairs {
  static constexpr int P = N * (N - 1) / 2;
  static __host__ __device__ constexpr int index(int a, int b) {  // a < b
    return a * N - a * (a + 1) / 2 + (b - a - 1);
  }
};

// ---------------------------------------------------------------- device helpers

template <int N>
__device__ __forceinline__ float hphi(const float* p, int a) {
  float s1 = 0.f;
#pragma unroll
  for (int b = 0; b < N; b++)
#pragma unroll
    for (int c = b + 1; c < N; c++)
      if (b != a && c != a) s1 += p[b] * p[c];
  return p[a] * p[a] * (3.f - 2.f * p[a]) + 2.f * p[a] * s1;
}

// dh_b / dphi_a
template <int N>
__device__ __forceinline__ float dhphi(const float* p, int b, int a) {
  float s = 0.f;
  if (a == b) {
#pragma unroll
    for (int e = 0; e < N; e++)
#pragma unroll
      for (int f = e + 1; f < N; f++)
        if (e != b && f != b) s += p[e] * p[f];
    return 6.f * p[a] * (1.f - p[a]) + 2.f * s;
  }
#pragma unroll
  for (int e = 0; e < N; e++)
    if (e != b && e != a) s += p[e];
  return 2.f * s * p[b];
}

template <int K1>
__device__ __forceinline__ float c_mu(const Model& m, const float* mu, int a, int i) {
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < K1; k++) s += m.cmu[a][i][k] * (mu[k] - m.Beff[a][k]);
  return s;
}

// c_mu at a cell's temperature: beff = the Beff(T)[N][K1] block of the cell's row of the tile's
// temperature table, or nullptr (isothermal: the model's Beff)
template <int K1>
__device__ __forceinline__ float c_mu_t(const Model& m, const float* mu, int a, int i, const float* beff) {
  if (!beff) return c_mu<K1>(m, mu, a, i);
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < K1; k++) s += m.cmu[a][i][k] * (mu[k] - beff[a * K1 + k]);
  return s;
}

__device__ __forceinline__ float aniso_ac(float dab, float q0, float q1) {
  const float q2 = q0 * q0 + q1 * q1;
  if (q2 > 1.0e-15f) {
    const float inv = 1.f / q2;
    const float x2 = q0 * q0 * inv, y2 = q1 * q1 * inv;
    return 1.f - dab * (3.f - 4.f * (x2 * x2 + y2 * y2));
  }
  return 1.f;
}

// a_c and |q|^2 * d a_c / d q (the combination every caller uses)
__device__ __forceinline__ void aniso_terms(float dab, float q0, float q1, float& ac, float& q2, float& e0,
                                            float& e1) {
  q2 = q0 * q0 + q1 * q1;
  if (q2 > 1.0e-15f) {
    const float inv = 1.f / q2;
    const float x2 = q0 * q0 * inv, y2 = q1 * q1 * inv;
    const float s4 = x2 * x2 + y2 * y2;  // sum q_i^4 / |q|^4
    ac = 1.f - dab * (3.f - 4.f * s4);
    // |q|^2 * 16 dab (q_i^3/|q|^4 - q_i sum q^4/|q|^6) = 16 dab q_i (q_i^2/|q|^2 - s4)
    e0 = 16.f * dab * q0 * (x2 - s4);
    e1 = 16.f * dab * q1 * (y2 - s4);
  } else {
    ac = 1.f;
    e0 = e1 = 0.f;
  }
}

// ---------------------------------------------------------------- shared pieces of the update

// The pieces below are shared by the pure-tile path and the full path.  They
// are written with explicit round-to-nearest intrinsics (never contracted or
// re-associated by the compiler), so a cell gets the same bits whichever path
// its tile takes -- the result does not depend on the tile shape.

// Diffusion flux of every component through one face, scaled by the face's
// 1/dx of the divergence: sum_l (D_c + D_n)_kl * dt/(2 dx^2) * (mu_n - mu_c)_l
// (calculate_gradients.h:132-185 with functionD.h; hh = Model::hx or hy).
template <int K1>
__device__ __forceinline__ void diff_flux(const float (&Dc)[MK][MK], const float (&Dn)[MK][MK],
                                          const float* muc, const float* mun, float hh, float* out) {
#pragma unroll
  for (int k = 0; k < K1; k++) {
    float jd = __fmul_rn(__fmul_rn(__fadd_rn(Dc[k][0], Dn[k][0]), hh), __fsub_rn(mun[0], muc[0]));
#pragma unroll
    for (int l = 1; l < K1; l++)
      jd = __fmaf_rn(__fmul_rn(__fadd_rn(Dc[k][l], Dn[k][l]), hh), __fsub_rn(mun[l], muc[l]), jd);
    out[k] = jd;
  }
}

// phi-weighted mobility D = sum_b DC_b phi_b (functionD.h:1-16)
template <int N, int K1>
__device__ __forceinline__ void mobility(const Model& m, const float* ph, float (&D)[MK][MK]) {
#pragma unroll
  for (int k = 0; k < K1; k++)
#pragma unroll
    for (int l = 0; l < K1; l++) {
      float s = 0.f;
#pragma unroll
      for (int b = 0; b < N; b++) s = __fmaf_rn(m.DC[b][k][l], ph[b], s);
      D[k][l] = s;
    }
}

// net face flux into a cell (the fluxes carry the 1/dx of the divergence)
__device__ __forceinline__ float flux_div(float fxp, float fxm, float fyp, float fym) {
  return __fadd_rn(__fsub_rn(fxp, fxm), __fsub_rn(fyp, fym));
}

// Error-free transforms (Knuth's TwoSum; TwoProduct with the fused multiply-add), explicit
// round-to-nearest: s + e == a + b and p + e == a * b exactly.
__device__ __forceinline__ float two_sum(float a, float b, float& e) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}
__device__ __forceinline__ float two_prod(float a, float b, float& e) {
  const float p = __fmul_rn(a, b);
  e = __fmaf_rn(a, b, -p);
  return p;
}

// Compensated flux accumulation: the net face flux with the rounding errors of its three
// additions summed separately and added once (the flux differences cancel in smooth fields).
__device__ __forceinline__ float flux_div_c(float fxp, float fxm, float fyp, float fym) {
  float e1, e2, e3;
  const float a = two_sum(fxp, -fxm, e1), b = two_sum(fyp, -fym, e2);
  const float s = two_sum(a, b, e3);
  return __fadd_rn(s, __fadd_rn(__fadd_rn(e1, e2), e3));
}

// Bulk cell of phase b whose face fluxes dc were evaluated (a neighbour is not
// pure b): c -> c + dc, mu = dF/dc (calculate_divergence_concentration.h:216-224)
// is, for quadratic free energies, mu + H dc with H = d mu / d c of the phase;
// the FP32 form evaluates it that way (one rounding at mu's scale).
template <int K1>
__device__ __forceinline__ void bulk_update_h(const float (&H)[MK][MK], const float* mu, const float* dc,
                                              float* mnew, bool comp = false) {
#pragma unroll
  for (int k = 0; k < K1; k++) {
    float s, c = 0.f;
    if (comp) {  // compensated dot product (Dot2): products and sums error-free, errors summed apart
      float ep, es;
      s = two_prod(H[k][0], dc[0], ep);
      c = ep;
#pragma unroll
      for (int l = 1; l < K1; l++) {
        const float p = two_prod(H[k][l], dc[l], ep);
        s = two_sum(s, p, es);
        c = __fadd_rn(c, __fadd_rn(ep, es));
      }
      s = __fadd_rn(s, c);
    } else {
      s = __fmul_rn(H[k][0], dc[0]);
#pragma unroll
      for (int l = 1; l < K1; l++) s = __fmaf_rn(H[k][l], dc[l], s);
    }
    mnew[k] = __fadd_rn(mu[k], s);
  }
}

// Pure-phase update of a cell whose 3x3 neighbourhood is the one-hot field of
// phase b: diffusion of mu inside b, mu + Gx Lx + Gy Ly (the face fluxes with
// both mobilities D_b and the bulk update folded into Gx = H (2 D_b) dt/(2 dx^2),
// Gy likewise).  Lx = dxp - dxm from the face differences dxp = mu(x+1) - mu,
// dxm = mu - mu(x-1), which are exact in floating point for neighbouring values
// (Sterbenz), so the increment is formed at its own scale and added once.  Every
// kernel uses this for every such cell, so a cell gets the same bits whichever
// kernel or tile shape updates it.
template <int K1>
__device__ __forceinline__ void pure_update(const float (&gx)[MK][MK], const float (&gy)[MK][MK], const float* mu,
                                            const float* dxp, const float* dxm, const float* dyp, const float* dym,
                                            float* mnew, bool comp = false) {
  float Lx[K1], Ly[K1];
  if (comp) {
    // compensated: the Laplacians' rounding errors and the increment's products and sums are
    // carried separately (TwoSum, TwoProduct) and added to the increment once
    float eLx[K1], eLy[K1];
#pragma unroll
    for (int k = 0; k < K1; k++) {
      Lx[k] = two_sum(dxp[k], -dxm[k], eLx[k]);
      Ly[k] = two_sum(dyp[k], -dym[k], eLy[k]);
    }
#pragma unroll
    for (int k = 0; k < K1; k++) {
      float ep, es, c;
      float s = two_prod(gy[k][0], Ly[0], ep);
      c = __fmaf_rn(gy[k][0], eLy[0], ep);
      float p = two_prod(gx[k][0], Lx[0], ep);
      s = two_sum(s, p, es);
      c = __fadd_rn(c, __fadd_rn(__fmaf_rn(gx[k][0], eLx[0], ep), es));
#pragma unroll
      for (int l = 1; l < K1; l++) {
        p = two_prod(gy[k][l], Ly[l], ep);
        s = two_sum(s, p, es);
        c = __fadd_rn(c, __fadd_rn(__fmaf_rn(gy[k][l], eLy[l], ep), es));
        p = two_prod(gx[k][l], Lx[l], ep);
        s = two_sum(s, p, es);
        c = __fadd_rn(c, __fadd_rn(__fmaf_rn(gx[k][l], eLx[l], ep), es));
      }
      mnew[k] = __fadd_rn(mu[k], __fadd_rn(s, c));
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < K1; k++) {
    Lx[k] = __fsub_rn(dxp[k], dxm[k]);
    Ly[k] = __fsub_rn(dyp[k], dym[k]);
  }
#pragma unroll
  for (int k = 0; k < K1; k++) {
    float s = __fmul_rn(gy[k][0], Ly[0]);
    s = __fmaf_rn(gx[k][0], Lx[0], s);
#pragma unroll
    for (int l = 1; l < K1; l++) {
      s = __fmaf_rn(gy[k][l], Ly[l], s);
      s = __fmaf_rn(gx[k][l], Lx[l], s);
    }
    mnew[k] = __fadd_rn(mu[k], s);
  }
}

// the (K1 x K1) block of phase b of a per-phase constant array
template <int N, int K1>
__device__ __forceinline__ void phase_mat(const float (&src)[MP][MK][MK], int b, float (&out)[MK][MK]) {
#pragma unroll
  for (int a = 0; a < N; a++)
    if (a == b) {
#pragma unroll
      for (int k = 0; k < K1; k++)
#pragma unroll
        for (int l = 0; l < K1; l++) out[k][l] = src[a][k][l];
    }
}

// ---------------------------------------------------------------- the fused step

template <int N, int K1, bool ANISO, int TX, int TY>
struct Tile {
  static_assert(TY % 32 == 0, "a tile row is a whole number of warps");
  static constexpr int P = Pairs<N>::P;
  static constexpr int X2 = TX + 4, Y2 = TY + 4;  // phi region: tile +- 2
  static constexpr int X1 = TX + 2, Y1 = TY + 2;  // mu / Delta-phi region: tile +- 1
  static constexpr int W = TY + 8;                 // staged row: y0-4 .. y0+TY+3 (16-byte aligned)
  static constexpr int Q = W / 4;                  // float4 per staged row
  // shared-memory layout (floats)
  static constexpr int o_phi = 0;                                 // [N][X2][W]
  static constexpr int o_mu = o_phi + N * X2 * W;                 // [K1][X1][W]
  static constexpr int o_dphi = o_mu + K1 * X1 * W;               // [N][X1][Y1]
  static constexpr int o_bx = o_dphi + N * X1 * Y1;               // x-face brackets [P][TX+3][TY+2]
  static constexpr int o_by = o_bx + P * (TX + 3) * (TY + 2);     // y-face brackets [P][TX+2][TY+3]
  static constexpr int o_fx = o_by + P * (TX + 2) * (TY + 3);     // mu-update x-face fluxes [K1][TX+1][TY]
  static constexpr int o_fy = o_fx + K1 * (TX + 1) * TY;          // mu-update y-face fluxes [K1][TX][TY+1]
  static constexpr int o_list = o_fy + K1 * TX * (TY + 1);        // active ring cells (ints) [X1*Y1]
  static constexpr int o_act = o_list + X1 * Y1;                  // active flags (ints) [X1*Y1]
  static constexpr int total = o_act + X1 * Y1;
  static constexpr size_t bytes = total * sizeof(float);
  // non-isothermal instances only (added to the launch's dynamic shared memory): the
  // T-dependent constants of the tile's columns y0-1 .. y0+TY, [2][Y1][RT] -- variant 0 for the
  // phase-field half step, 1 for the concentration half step (they differ on ghost columns) --
  // a row holding Beff(T)[N][K1], B(T)[N][K1], C(T)[N]
  static constexpr int RT = 2 * N * K1 + N;
  static constexpr int o_temp = total;
  static constexpr size_t bytes_temp = (size_t)2 * Y1 * RT * sizeof(float);
};

// Asynchronous global -> shared copies (cp.async), completed per thread by
// wait_group / wait_all and published to the block by a barrier.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------- narrow band
//
// Far from every interface a cell's phi is the one-hot field of one phase and
// its update is diffusion of mu inside that phase.  Each step writes, per tile,
// a purity word describing its output: five 4-bit fields, each 1 + b when every
// in-grid cell of that part of the tile holds the one-hot field of phase b
// (exactly 1.0f and +0.0f), else 0.  The parts: the whole tile, its first and
// last two rows (x) and its first and last two columns (y).
enum { PF_CORE = 0, PF_XLO = 4, PF_XHI = 8, PF_YLO = 12, PF_YHI = 16 };
__host__ __device__ __forceinline__ int pf(uint32_t w, int f) { return (int)((w >> f) & 15u); }
__host__ __device__ __forceinline__ uint32_t pf_all(int c) { return (uint32_t)c * 0x11111u; }

// Static facts of tile t used by lean_phase, one word: tiles along y (the
// index stride of the x-neighbours), which of the four neighbours exist, and
// whether the tile is never lean (its two-cell ring leaves the grid where it
// is not a trusted mirror: a periodic wrap, or fewer than 3 cells on that axis).
// TG_REJECT2: the tile never takes the two-step lean update, because its two-cell
// ring leaves the grid across a periodic boundary of phi or mu (the ring's purity
// and the partner cells of the intermediate step are not known there).
enum : uint32_t { TG_NY = 0xFFFFFFu, TG_XM = 1u << 24, TG_XP = 1u << 25, TG_YM = 1u << 26, TG_YP = 1u << 27,
                  TG_REJECT = 1u << 28, TG_REJECT2 = 1u << 29 };

inline uint32_t tile_geo(const Inst& I, int t, int TX, int TY) {
  const int ny = I.tiles_y, lt = t - I.tile_begin, tx = lt / ny, ty = lt % ny;
  const int ex = I.mx - tx * TX < TX ? I.mx - tx * TX : TX, ey = I.my - ty * TY < TY ? I.my - ty * TY : TY;
  const bool xm = tx > 0, xp = tx + 1 < I.tiles_x, ym = ty > 0, yp = ty + 1 < ny;
  const bool reject = ((!xm || !xp) && !(I.bc.phi_x == GP_BC_NEUMANN && ex >= 3)) ||
                      ((!ym || !yp) && !(I.bc.phi_y == GP_BC_NEUMANN && ey >= 3));
  const int x0 = tx * TX, y0 = ty * TY;
  const bool cross_x = x0 - 2 < 0 || x0 + TX + 2 > I.mx, cross_y = y0 - 2 < 0 || y0 + TY + 2 > I.my;
  const bool reject2 = (cross_x && (I.bc.phi_x != GP_BC_NEUMANN || I.bc.mu_x != GP_BC_NEUMANN)) ||
                       (cross_y && (I.bc.phi_y != GP_BC_NEUMANN || I.bc.mu_y != GP_BC_NEUMANN));
  return (uint32_t)ny | (xm ? TG_XM : 0u) | (xp ? TG_XP : 0u) | (ym ? TG_YM : 0u) | (yp ? TG_YP : 0u) |
         (reject ? TG_REJECT : 0u) | (reject2 ? TG_REJECT2 : 0u);
}

// Phase b >= 0 when tile t may take the lean update: in the input, the tile
// and the two-cell ring the full update reads around it (tile +- 2, the phi
// region it stages) hold the one-hot field of phase b, known from the purity
// words of the tile and its eight neighbours.  Where the ring leaves the grid
// it is the Neumann mirror of the tile's own cells (rows 1, 2 and M-2, M-3:
// the tile needs 3 cells on that axis); a periodic wrap is not trusted.
// The full update of such a tile is its pure-phase path, so the lean update
// gives the same bits.  -1 otherwise.  The nine words are loaded at once (a
// missing neighbour reads the tile's own word, unused).
__host__ __device__ __forceinline__ int lean_phase(const uint32_t* __restrict__ F, uint32_t geo, int t) {
  if (geo & TG_REJECT) return -1;
  const int ny = (int)(geo & TG_NY);
  const bool xm = geo & TG_XM, xp = geo & TG_XP, ym = geo & TG_YM, yp = geo & TG_YP;
  const uint32_t w = F[t];
  const uint32_t wxm = F[xm ? t - ny : t], wxp = F[xp ? t + ny : t], wym = F[ym ? t - 1 : t],
                 wyp = F[yp ? t + 1 : t];
  const uint32_t wmm = F[xm && ym ? t - ny - 1 : t], wmp = F[xm && yp ? t - ny + 1 : t],
                 wpm = F[xp && ym ? t + ny - 1 : t], wpp = F[xp && yp ? t + ny + 1 : t];
  const int c = pf(w, PF_CORE);
  bool ok = c != 0;
  ok &= !xm || pf(wxm, PF_XHI) == c;
  ok &= !xp || pf(wxp, PF_XLO) == c;
  ok &= !ym || pf(wym, PF_YHI) == c;
  ok &= !yp || pf(wyp, PF_YLO) == c;
  ok &= !(xm && ym) || pf(wmm, PF_XHI) == c || pf(wmm, PF_YHI) == c;
  ok &= !(xm && yp) || pf(wmp, PF_XHI) == c || pf(wmp, PF_YLO) == c;
  ok &= !(xp && ym) || pf(wpm, PF_XLO) == c || pf(wpm, PF_YHI) == c;
  ok &= !(xp && yp) || pf(wpp, PF_XLO) == c || pf(wpp, PF_YLO) == c;
  return ok ? c - 1 : -1;
}

// Full update of the tiles.  With glist == nullptr block k takes tile k (grid
// = all tiles).  Otherwise the blocks are persistent and take the entries of
// glist: first the cnt[0] tiles with interface cells of their own (glist[0..]),
// then the cnt[3] tiles that are pure inside and only border an interface
// (stored from glist[total - 1] down), cheaper, so that they fill the second
// round; block k takes entry k first, then entries grid + (queue head
// cnt[1]); the last block to finish resets the counters (cnt[2] counts
// finished blocks) for the next step.
// Every tile writes the purity word of its output.
// THREADS per block (one tile): 256, or 512 for binary alloys (shorter per-thread chains, half
// the resident blocks: faster when there are few interface tiles); the autotuner picks.
template <int N, int K1, bool ANISO, int TX, int TY, int THREADS = 256>
__global__ void __launch_bounds__(THREADS, (N == 2 && K1 == 1) ? 1024 / THREADS
                                                              : (K1 >= 3 || N >= 5 || THREADS > 256 ? 1 : 2))
    k_step32(const Inst* __restrict__ insts, const Model* __restrict__ models, const int* __restrict__ tile_inst,
             const int2* __restrict__ glist, int* __restrict__ cnt, uint32_t* __restrict__ flags_out, int total,
             const int4* __restrict__ tile_desc, const uint32_t* __restrict__ flags_in, int keep_list) {
  using T = Tile<N, K1, ANISO, TX, TY>;
  constexpr int X2 = T::X2, Y2 = T::Y2, X1 = T::X1, Y1 = T::Y1, W = T::W, Q = T::Q;
  constexpr int L = N - 1;
  extern __shared__ __align__(16) float sm[];
  float* sphi = sm + T::o_phi;
  float* smu = sm + T::o_mu;
  float* sdp = sm + T::o_dphi;
  __shared__ __align__(16) Model sModel;
  __shared__ __align__(16) Inst sInst;
  __shared__ int s_tile, s_model, s_reload;
  __shared__ unsigned s_bad;
  // scan mode (tile_desc given): the block's own tiles blockIdx.x + grid * j, scanned THREADS
  // candidates at a time; the ones lean_phase rejects are listed here and updated in turn
  __shared__ int2 s_scan[THREADS];
  __shared__ int s_scan_n, s_scan_k, s_chunk, s_scan_done;
  const int nt = blockDim.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = nt >> 5;
  if (threadIdx.x == 0) {
    s_model = -1;
    s_scan_n = s_scan_k = s_chunk = 0;
    s_scan_done = (int)blockIdx.x >= total;
  }
  // Launched as a programmatic dependent of the tile list (the blocks start while the list kernel
  // runs): nothing an earlier kernel wrote is read before this wait, which returns once the list
  // kernel and everything before it have completed.  Without that launch attribute it returns at once.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");

  for (int iter = 0;; iter++) {
  __syncthreads();  // the previous tile's shared state is no longer read
  if (tile_desc) {
    while (s_scan_k >= s_scan_n && !s_scan_done) {  // block-uniform: shared values read after a barrier
      __syncthreads();
      if (threadIdx.x == 0) s_scan_n = s_scan_k = 0;
      __syncthreads();
      const int64_t t = blockIdx.x + (int64_t)gridDim.x * ((int64_t)s_chunk * nt + threadIdx.x);
      int4 d = make_int4(0, 0, 0, 0);
      if (t < total) d = tile_desc[t];
      const bool gen = t < total && lean_phase(flags_in, (uint32_t)d.w, (int)t) < 0;
      const unsigned bal = __ballot_sync(0xffffffffu, gen);
      int base = 0;
      if (lane == 0 && bal) base = atomicAdd(&s_scan_n, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (gen) s_scan[base + __popc(bal & ((1u << lane) - 1u))] = make_int2((int)t, d.x);
      __syncthreads();
      if (threadIdx.x == 0) {
        s_chunk++;
        s_scan_done = blockIdx.x + (int64_t)gridDim.x * ((int64_t)s_chunk * nt) >= total;
      }
      __syncthreads();
    }
    // every warp has evaluated the loop condition before thread 0 below advances s_scan_k
    // (a warp reading it late would otherwise see the list exhausted and scan alone)
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int2 e = make_int2(-1, 0);
    if (tile_desc) {
      if (s_scan_k < s_scan_n) e = s_scan[s_scan_k++];
    } else if (glist) {  // block k starts with entry k, then takes entries grid, grid + 1, ... from the queue
      // (claimed when the block is free: the blocks whose first tiles finish early take the rest)
      const int i = iter == 0 ? (int)blockIdx.x : (int)gridDim.x + atomicAdd(&cnt[1], 1);
      // the front entry is read together with the counts (an in-bounds read, used only when the
      // count covers it), so the common case waits for one round trip instead of two
      const int2 front = i < total ? glist[i] : make_int2(-1, 0);
      const int n0 = cnt[0];
      if (i < n0) e = front;
      else if (i < n0 + cnt[3]) e = glist[total - 1 - (i - n0)];
    } else if (iter == 0) {
      e = make_int2((int)blockIdx.x, tile_inst[blockIdx.x]);
    }
    s_tile = e.x;
    if (e.x >= 0) {
      sInst = insts[e.y];
      s_reload = sInst.model != s_model;
      s_model = sInst.model;
      s_bad = 0u;
    }
  }
  __syncthreads();
  const int tile = s_tile;
  if (tile < 0) break;
  if (s_reload) {  // the instance's model constants into shared memory, loaded with the staged fields
    const float4* src = reinterpret_cast<const float4*>(models + sInst.model);
    float4* dst = reinterpret_cast<float4*>(&sModel);
    for (int e = threadIdx.x; e < (int)(sizeof(Model) / 16); e += nt) cp_async16(dst + e, src + e);
  }
  const Inst& I = sInst;
  const Model& m = sModel;
  const int lt = tile - I.tile_begin;
  const int x0 = (lt / I.tiles_y) * TX, y0 = (lt % I.tiles_y) * TY;
  const int mx = I.mx, my = I.my;

  auto PH = [&](int a, int i, int j) -> float { return sphi[(a * X2 + i) * W + j + 2]; };  // region-2 coords
  auto MU = [&](int k, int i, int j) -> float { return smu[(k * X1 + i) * W + j + 3]; };   // region-1 coords

  // ---- stage phi (tile +- 2) and mu (tile +- 1)
  const bool inner = x0 >= 2 && x0 + TX + 2 <= mx && y0 >= 4 && y0 + TY + 4 <= my;
  // (asynchronous copies: every load of the tile is in flight at once)
  if (inner) {
    // whole 16-byte aligned rows y0-4 .. y0+TY+3, no boundary maps needed
    for (int e = threadIdx.x; e < N * X2 * Q; e += nt) {
      const int a = e / (X2 * Q), r = (e / Q) % X2, q = e % Q;
      cp_async16(sphi + (a * X2 + r) * W + 4 * q, I.phi + a * I.plane + (int64_t)(x0 - 2 + r) * I.pitch + (y0 - 4) + 4 * q);
    }
    for (int e = threadIdx.x; e < K1 * X1 * Q; e += nt) {
      const int k = e / (X1 * Q), r = (e / Q) % X1, q = e % Q;
      cp_async16(smu + (k * X1 + r) * W + 4 * q, I.mu + k * I.plane + (int64_t)(x0 - 1 + r) * I.pitch + (y0 - 4) + 4 * q);
    }
  } else {
    for (int e = threadIdx.x; e < X2 * Y2; e += nt) {
      const int i = e / Y2, j = e % Y2;
      const int gx = gp_map_any(x0 - 2 + i, mx, I.bc.phi_x), gy = gp_map_any(y0 - 2 + j, my, I.bc.phi_y);
      const float* p = I.phi + (int64_t)gx * I.pitch + gy;
#pragma unroll
      for (int a = 0; a < N; a++) cp_async4(sphi + (a * X2 + i) * W + j + 2, p + a * I.plane);
    }
    for (int e = threadIdx.x; e < X1 * Y1; e += nt) {
      const int i = e / Y1, j = e % Y1;
      const int gx = gp_map_any(x0 - 1 + i, mx, I.bc.mu_x), gy = gp_map_any(y0 - 1 + j, my, I.bc.mu_y);
      const float* p = I.mu + (int64_t)gx * I.pitch + gy;
#pragma unroll
      for (int k = 0; k < K1; k++) cp_async4(smu + (k * X1 + i) * W + j + 3, p + k * I.plane);
    }
  }
  cp_async_wait_all();
  __syncthreads();

  // ---- pure-tile test: when every staged cell is the same pure phase, Delta-phi
  // is exactly zero on the ring (divphi = 0) and so is every antitrapping
  // current (zero gradients): the tile's update is diffusion in one phase.
  int b0 = -1;
#pragma unroll
  for (int a = N - 1; a >= 0; a--)
    if (PH(a, 0, 0) == 1.f) b0 = a;
  bool ok = b0 >= 0;
  for (int e = threadIdx.x; ok && e < X2 * Y2; e += nt) {
    const int i = e / Y2, j = e % Y2;
#pragma unroll
    for (int a = 0; a < N; a++) ok &= (PH(a, i, j) == (a == b0 ? 1.f : 0.f));
  }
  const bool pure = __syncthreads_and(ok) != 0;

  if (pure) {
    float gx[MK][MK], gy[MK][MK];
    phase_mat<N, K1>(m.Gx, b0, gx);
    phase_mat<N, K1>(m.Gy, b0, gy);
    for (int r = warp; r < TX; r += nw) {
      const int x = x0 + r;
      if (x >= mx) break;
#pragma unroll
      for (int c0 = 0; c0 < TY; c0 += 32) {
        const int c = c0 + lane, y = y0 + c;
        if (y >= my) continue;
        const int i1 = r + 1, j1 = c + 1;
        float mc[K1], mb[K1], mf[K1], ml[K1], mr[K1];
#pragma unroll
        for (int k = 0; k < K1; k++) {
          mc[k] = MU(k, i1, j1);
          mb[k] = MU(k, i1 - 1, j1);
          mf[k] = MU(k, i1 + 1, j1);
          ml[k] = MU(k, i1, j1 - 1);
          mr[k] = MU(k, i1, j1 + 1);
        }
        float dxp[K1], dxm[K1], dyp[K1], dym[K1], mnew[K1];
#pragma unroll
        for (int k = 0; k < K1; k++) {
          dxp[k] = __fsub_rn(mf[k], mc[k]);
          dxm[k] = __fsub_rn(mc[k], mb[k]);
          dyp[k] = __fsub_rn(mr[k], mc[k]);
          dym[k] = __fsub_rn(mc[k], ml[k]);
        }
        pure_update<K1>(gx, gy, mc, dxp, dxm, dyp, dym, mnew, m.comp);
        const int64_t o = (int64_t)x * I.pitch + y;
#pragma unroll
        for (int k = 0; k < K1; k++) I.mu_out[o + k * I.plane] = mnew[k];
#pragma unroll
        for (int a = 0; a < N; a++) I.phi_out[o + a * I.plane] = (a == b0) ? 1.f : 0.f;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) flags_out[tile] = pf_all(1 + b0);
    continue;
  }

  // ---- tile touches an interface.  Active ring cells (some divphi != 0) are
  // flagged and compacted into a list; gradient-energy brackets are evaluated
  // only on faces next to an active cell; Delta-phi is computed for the listed
  // cells (calculate_divergence_phasefield.h:4-62).
  // Non-isothermal instances first tabulate the T-dependent constants of the tile's columns:
  // T of ghost-padded column gy = bottom + gy * grad at the step being computed, the ghost
  // columns' own linear T in the phase-field half step after the first step and their boundary
  // copy otherwise (Temperature_gradient.h:19, microsim_gp.c:77-82, 108-113); Beff, B(T), C(T) in
  // FP64 in the reference's order (functionF_01.h:62-104), stored as FP32.  Read after the
  // barriers below.
  float* const ttab = I.gm ? sm + T::o_temp : nullptr;
  if (ttab) {
    const gp_model& g = *I.gm;
    const gp_temp_step ts = gp_temp_after(g, __ldcg(I.tstep));
    for (int e = threadIdx.x; e < 2 * Y1 * N; e += nt) {
      const int v = e / (Y1 * N), j = (e / N) % Y1, a = e % N, y = y0 - 1 + j;
      const bool linear = v == 0 && ts.linear;
      const int yy = (linear || !g.bc_T[3] || (y >= 0 && y < my)) ? y : gp_map(y, my, g.bc_T[3]);
      Th th;
      th.on = 1;
      th.T = ts.bottom + (double)(yy + 3) * ts.grad;
      float* r = ttab + (v * Y1 + j) * T::RT;
#pragma unroll
      for (int k = 0; k < K1; k++) {
        r[a * K1 + k] = (float)beff(g, th, a, k);
        r[N * K1 + a * K1 + k] = (float)B_Tn<N, K1>(g, th, k, a);
      }
      r[2 * N * K1 + a] = (float)C_Tn<N, K1>(g, th, a);
    }
  }
  // the table row of region-1 column j: v = 0 phase-field half step, 1 concentration half step
  auto trow = [&](int v, int j) -> const float* { return ttab ? ttab + (v * Y1 + j) * T::RT : nullptr; };
  int* s_list = reinterpret_cast<int*>(sm + T::o_list);
  int* s_act = reinterpret_cast<int*>(sm + T::o_act);
  float* sbx = sm + T::o_bx;
  float* sby = sm + T::o_by;
  float* sfx = sm + T::o_fx;
  float* sfy = sm + T::o_fy;
  __shared__ int s_nact;
  if (threadIdx.x == 0) s_nact = 0;
  __syncthreads();
  for (int e0 = 0; e0 < X1 * Y1; e0 += nt) {
    const int e = e0 + threadIdx.x;
    bool act = false;
    if (e < X1 * Y1) {
      const int i1 = e / Y1, j1 = e % Y1;
      const int i = i1 + 1, j = j1 + 1;
#pragma unroll
      for (int a = 0; a < N; a++) {
        const float pc = PH(a, i, j);
        const float gf = (PH(a, i + 1, j) - pc) * m.dx_inv, gb = (pc - PH(a, i - 1, j)) * m.dx_inv;
        const float gr = (PH(a, i, j + 1) - pc) * m.dy_inv, gl = (pc - PH(a, i, j - 1)) * m.dy_inv;
        act |= ((gf - gb) * m.dx_inv + (gr - gl) * m.dy_inv) != 0.f;
        sdp[a * X1 * Y1 + e] = 0.f;
      }
      s_act[e] = act;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, act);
    int base = 0;
    if (lane == 0 && bal) base = atomicAdd(&s_nact, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (act) s_list[base + __popc(bal & ((1u << lane) - 1u))] = e;
  }
  __syncthreads();

  // gradient-energy bracket of pair (a, b) on the x-face between region-2 rows
  // i and i+1 at column j (and on the y-face between columns j and j+1 at row i):
  //   Bk = a_c^2 Q_n + a_c |q|^2 (Rinv dadq)_n (anisotropic), Bk = Q_n (isotropic),
  //   Q_n = s_a g_b - s_b g_a; the flux of phase a (pair b) through the face is
  //   -Bk s_b, that of b (pair a) +Bk s_a (function_A_0x divdAdgradphi).
  auto bk_x = [&](int i, int j, int a, int b) -> float {
    const float pa = PH(a, i, j), pfa = PH(a, i + 1, j), pb = PH(b, i, j), pfb = PH(b, i + 1, j);
    const float sa = 0.5f * (pa + pfa), sb = 0.5f * (pb + pfb);
    const float Qx = sa * ((pfb - pb) * m.dx_inv) - sb * ((pfa - pa) * m.dx_inv);
    if (!ANISO) return Qx;
    const float cya = (PH(a, i, j + 1) - PH(a, i, j - 1)) * m.half_dy_inv +
                      (PH(a, i + 1, j + 1) - PH(a, i + 1, j - 1)) * m.half_dy_inv;
    const float cyb = (PH(b, i, j + 1) - PH(b, i, j - 1)) * m.half_dy_inv +
                      (PH(b, i + 1, j + 1) - PH(b, i + 1, j - 1)) * m.half_dy_inv;
    const float Qy = 0.5f * (sa * cyb - sb * cya);
    const float q0 = m.R[a][b][0][0] * Qx + m.R[a][b][0][1] * Qy;
    const float q1 = m.R[a][b][1][0] * Qx + m.R[a][b][1][1] * Qy;
    float ac, q2, e0, e1;
    aniso_terms(m.dab[a][b], q0, q1, ac, q2, e0, e1);
    return ac * ac * Qx + ac * (m.Rinv[a][b][0][0] * e0 + m.Rinv[a][b][0][1] * e1);
  };
  auto bk_y = [&](int i, int j, int a, int b) -> float {
    const float pa = PH(a, i, j), pra = PH(a, i, j + 1), pb = PH(b, i, j), prb = PH(b, i, j + 1);
    const float sa = 0.5f * (pa + pra), sb = 0.5f * (pb + prb);
    const float Qy = sa * ((prb - pb) * m.dy_inv) - sb * ((pra - pa) * m.dy_inv);
    if (!ANISO) return Qy;
    const float cxa = 0.5f * (PH(a, i + 1, j) - PH(a, i - 1, j)) * m.dx_inv +
                      0.5f * (PH(a, i + 1, j + 1) - PH(a, i - 1, j + 1)) * m.dx_inv;
    const float cxb = 0.5f * (PH(b, i + 1, j) - PH(b, i - 1, j)) * m.dx_inv +
                      0.5f * (PH(b, i + 1, j + 1) - PH(b, i - 1, j + 1)) * m.dx_inv;
    const float Qx = 0.5f * (sa * cxb - sb * cxa);
    const float q0 = m.R[a][b][0][0] * Qx + m.R[a][b][0][1] * Qy;
    const float q1 = m.R[a][b][1][0] * Qx + m.R[a][b][1][1] * Qy;
    float ac, q2, e0, e1;
    aniso_terms(m.dab[a][b], q0, q1, ac, q2, e0, e1);
    return ac * ac * Qy + ac * (m.Rinv[a][b][1][0] * e0 + m.Rinv[a][b][1][1] * e1);
  };

  // x-face between region-2 rows i and i+1 (i in [0, TX+2]) at region-2 columns
  // j in [1, TY+2]; read by ring cell (i-1, j-1) as its +x face and by ring cell
  // (i, j-1) as its -x face (region-1 coordinates)
  for (int e = threadIdx.x; e < (TX + 3) * (TY + 2); e += nt) {
    const int i = e / (TY + 2), j = 1 + e % (TY + 2);
    const bool need = (i >= 1 && s_act[(i - 1) * Y1 + (j - 1)]) || (i <= TX + 1 && s_act[i * Y1 + (j - 1)]);
    if (!need) continue;
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
      for (int b = a + 1; b < N; b++)
        sbx[(Pairs<N>::index(a, b) * (TX + 3) + i) * (TY + 2) + (j - 1)] = bk_x(i, j, a, b);
  }
  // y-face between region-2 columns j and j+1 (j in [0, TY+2]) at rows i in [1, TX+2]
  for (int e = threadIdx.x; e < (TX + 2) * (TY + 3); e += nt) {
    const int i = 1 + e / (TY + 3), j = e % (TY + 3);
    const bool need = (j >= 1 && s_act[(i - 1) * Y1 + (j - 1)]) || (j <= TY + 1 && s_act[(i - 1) * Y1 + j]);
    if (!need) continue;
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
      for (int b = a + 1; b < N; b++)
        sby[(Pairs<N>::index(a, b) * (TX + 2) + (i - 1)) * (TY + 3) + j] = bk_y(i, j, a, b);
  }
  __syncthreads();

  const int nact = s_nact;
  for (int idx = threadIdx.x; idx < nact; idx += nt) {
    const int e = s_list[idx];
    const int i1 = e / Y1, j1 = e % Y1;  // region-1 coordinates
    const int i = i1 + 1, j = j1 + 1;    // region-2 coordinates
    float ph[N], cx[N], cy[N], divphi[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      ph[a] = PH(a, i, j);
      const float gf = (PH(a, i + 1, j) - ph[a]) * m.dx_inv, gb = (ph[a] - PH(a, i - 1, j)) * m.dx_inv;
      const float gr = (PH(a, i, j + 1) - ph[a]) * m.dy_inv, gl = (ph[a] - PH(a, i, j - 1)) * m.dy_inv;
      divphi[a] = (gf - gb) * m.dx_inv + (gr - gl) * m.dy_inv;
      cx[a] = 0.5f * (gf + gb);
      cy[a] = (PH(a, i, j + 1) - PH(a, i, j - 1)) * m.half_dy_inv;
    }
    // -dA/dphi_a + div dA/dgrad phi_a, accumulated per phase over pairs (one
    // copy of the pair code: the loops below are not unrolled, keeping the
    // register count of the fused kernel low)
    float gterm[N];
#pragma unroll
    for (int a = 0; a < N; a++) gterm[a] = 0.f;
#pragma unroll 1
    for (int p = 0; p < Pairs<N>::P; p++) {
      int a = 0, b = 1;
#pragma unroll
      for (int aa = 0; aa < N; aa++)
#pragma unroll
        for (int bb = aa + 1; bb < N; bb++)
          if (Pairs<N>::index(aa, bb) == p) { a = aa; b = bb; }
      float pha = 0.f, phb = 0.f, cxa = 0.f, cxb = 0.f, cya = 0.f, cyb = 0.f;
#pragma unroll
      for (int aa = 0; aa < N; aa++) {
        if (aa == a) { pha = ph[aa]; cxa = cx[aa]; cya = cy[aa]; }
        if (aa == b) { phb = ph[aa]; cxb = cx[aa]; cyb = cy[aa]; }
      }
      const float g2 = 2.f * m.Gamma[a][b];
      const float bxf = sbx[(p * (TX + 3) + i) * (TY + 2) + (j - 1)];
      const float bxb = sbx[(p * (TX + 3) + i - 1) * (TY + 2) + (j - 1)];
      const float byr = sby[(p * (TX + 2) + (i - 1)) * (TY + 3) + j];
      const float byl = sby[(p * (TX + 2) + (i - 1)) * (TY + 3) + j - 1];
      const float sxa_f = 0.5f * (pha + PH(a, i + 1, j)), sxb_f = 0.5f * (phb + PH(b, i + 1, j));
      const float sxa_b = 0.5f * (pha + PH(a, i - 1, j)), sxb_b = 0.5f * (phb + PH(b, i - 1, j));
      const float sya_r = 0.5f * (pha + PH(a, i, j + 1)), syb_r = 0.5f * (phb + PH(b, i, j + 1));
      const float sya_l = 0.5f * (pha + PH(a, i, j - 1)), syb_l = 0.5f * (phb + PH(b, i, j - 1));
      const float div_ab = (-bxf * sxb_f + bxb * sxb_b) * m.dx_inv + (-byr * syb_r + byl * syb_l) * m.dy_inv;
      const float div_ba = (bxf * sxa_f - bxb * sxa_b) * m.dx_inv + (byr * sya_r - byl * sya_l) * m.dy_inv;
      // dA/dphi part at the centre
      const float Qx = pha * cxb - phb * cxa;
      const float Qy = pha * cyb - phb * cya;
      float dA_a, dA_b;
      if (ANISO) {
        const float q0 = m.R[a][b][0][0] * Qx + m.R[a][b][0][1] * Qy;
        const float q1 = m.R[a][b][1][0] * Qx + m.R[a][b][1][1] * Qy;
        float ac, q2, e0, e1;
        aniso_terms(m.dab[a][b], q0, q1, ac, q2, e0, e1);
        const float rb0 = m.R[a][b][0][0] * cxb + m.R[a][b][0][1] * cyb;
        const float rb1 = m.R[a][b][1][0] * cxb + m.R[a][b][1][1] * cyb;
        const float ra0 = m.R[a][b][0][0] * cxa + m.R[a][b][0][1] * cya;
        const float ra1 = m.R[a][b][1][0] * cxa + m.R[a][b][1][1] * cya;
        const float ac2 = ac * ac;
        dA_a = ac2 * (q0 * rb0 + q1 * rb1) + ac * (e0 * rb0 + e1 * rb1);
        dA_b = -(ac2 * (q0 * ra0 + q1 * ra1) + ac * (e0 * ra0 + e1 * ra1));
      } else {
        dA_a = Qx * cxb + Qy * cyb;
        dA_b = -(Qx * cxa + Qy * cya);
      }
      const float ta = g2 * (div_ab - dA_a), tb = g2 * (div_ba - dA_b);
#pragma unroll
      for (int aa = 0; aa < N; aa++) {
        if (aa == a) gterm[aa] += ta;
        if (aa == b) gterm[aa] += tb;
      }
    }
    // grand potentials of the phases at this cell's mu
    float mu[K1];
#pragma unroll
    for (int k = 0; k < K1; k++) mu[k] = MU(k, i1, j1);
    float psi[N];
    const float* tp = trow(0, j1);
#pragma unroll
    for (int b = 0; b < N; b++) {
      float c[K1], sv = 0.f;
#pragma unroll
      for (int k = 0; k < K1; k++) c[k] = c_mu_t<K1>(m, mu, b, k, tp);
#pragma unroll
      for (int k = 0; k < K1; k++) {
#pragma unroll
        for (int l = k; l < K1; l++) sv += m.A[b][k][l] * c[k] * c[l];
        sv += ((tp ? tp[N * K1 + b * K1 + k] : m.B[b][k]) - mu[k]) * c[k];
      }
      psi[b] = sv + (tp ? tp[2 * N * K1 + b] : m.C[b]);
    }
    float lambda[N], dp[N], sum_l = 0.f;
    int active = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      lambda[a] = 0.f;
      dp[a] = 0.f;
      if (divphi[a] != 0.f) {
        // obstacle / well potential (functionW_01.h, functionW_02.h)
        float w = 0.f;
#pragma unroll
        for (int b = 0; b < N; b++) {
          if (b == a || divphi[b] == 0.f) continue;
          if (m.obstacle) w += (ph[a] * ph[b] >= 0.f ? m.Gamma[a][b] : -m.Gamma[a][b]) * ph[b];
          else w += 2.f * m.Gamma[a][b] * ph[b] * ph[b] * ph[a];
        }
        w *= m.obstacle ? m.w_obst : 9.f;
#pragma unroll
        for (int b = 0; b < N; b++)
#pragma unroll
          for (int c = b + 1; c < N; c++) {
            if (b == a || c == a || divphi[b] == 0.f || divphi[c] == 0.f) continue;
            const float pbc = ph[b] * ph[c];
            w += (ph[a] * pbc >= 0.f ? m.Gabc[a][b][c] : -m.Gabc[a][b][c]) * pbc;
          }
        float dpsi = 0.f;
#pragma unroll
        for (int b = 0; b < N; b++) dpsi += psi[b] * dhphi<N>(ph, b, a);
        lambda[a] = m.eps * gterm[a] - m.inv_eps * w - dpsi;
        sum_l += lambda[a];
        active++;
      }
    }
    sum_l /= (float)active;
    float st = 0.f, st1 = 0.f;
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
      for (int b = a + 1; b < N; b++) {
        const float pp = ph[a] * ph[b];
        st += m.tau_ab[a][b] * pp;
        st1 += pp;
      }
    const float tphi = st1 != 0.f ? st / st1 : m.tau;
    const float f = m.dt / (tphi * m.eps);
#pragma unroll
    for (int a = 0; a < N; a++)
      if (divphi[a] != 0.f) dp[a] = f * (lambda[a] - sum_l);
    // projection onto the Gibbs simplex (simplex_projection.h:1-49)
    float over = 0.f, sum_in = 0.f;
    int count = 0;
#pragma unroll
    for (int a = 0; a < N; a++) {
      const float v = ph[a] + dp[a];
      if (divphi[a] != 0.f && v > 0.f && v < 1.f) {
        count++;
        sum_in += ph[a];
      }
    }
#pragma unroll
    for (int a = 0; a < N; a++) {
      const float v = ph[a] + dp[a];
      if (v < 0.f) {
        dp[a] -= v;
        over -= v;
      }
    }
    if (over > 0.f) {
#pragma unroll
      for (int b = 0; b < N; b++) {
        const float v = ph[b] + dp[b];
        if (divphi[b] != 0.f && v > 0.f && v < 1.f) dp[b] -= sum_in != 0.f ? over * ph[b] / sum_in : over / (float)count;
      }
    }
    int hit = -1;
#pragma unroll
    for (int a = 0; a < N; a++)
      if (hit < 0 && divphi[a] != 0.f && ph[a] + dp[a] > 1.f) hit = a;
    if (hit >= 0) {
#pragma unroll
      for (int a = 0; a < N; a++)
        if (divphi[a] != 0.f) dp[a] = (a == hit) ? 1.f - ph[a] : -ph[a];
    }
#pragma unroll
    for (int a = 0; a < N; a++) sdp[(a * X1 + i1) * Y1 + j1] = dp[a];
  }
  __syncthreads();

  // ---- face flux of the mu update: dt * D grad mu - jscale * j_at through the
  // face between region-1 cells c and its +x / +y neighbour n
  // (calculate_gradients.h:132-185, calculate_fluxes_concentration.h:4-145).
  // Both cells of a face evaluate it with the same code and inputs.
  auto face_flux = [&](int ic, int jc, bool xface, bool skip_at, float* out) {
    const int in = xface ? ic + 1 : ic, jn = xface ? jc : jc + 1;
    float pc[N], pn[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      pc[a] = PH(a, ic + 1, jc + 1);
      pn[a] = PH(a, in + 1, jn + 1);
    }
    float muc[K1], mun[K1];
#pragma unroll
    for (int k = 0; k < K1; k++) {
      muc[k] = MU(k, ic, jc);
      mun[k] = MU(k, in, jn);
    }
    float Dc[MK][MK], Dn[MK][MK];
    mobility<N, K1>(m, pc, Dc);
    mobility<N, K1>(m, pn, Dn);
    diff_flux<K1>(Dc, Dn, muc, mun, xface ? m.hx : m.hy, out);
    if (skip_at) return;
    float tc[N], tn[N], gn[N];
    bool any = false;
#pragma unroll
    for (int a = 0; a < N; a++) {
      gn[a] = (pn[a] - pc[a]) * (xface ? m.dx_inv : m.dy_inv);
      if (xface) {  // tangential: centred y gradient of each cell
        tc[a] = (PH(a, ic + 1, jc + 2) - PH(a, ic + 1, jc)) * m.half_dy_inv;
        tn[a] = (PH(a, in + 1, jn + 2) - PH(a, in + 1, jn)) * m.half_dy_inv;
      } else {  // centred x gradient (average of the two one-sided ones)
        tc[a] = 0.5f * (PH(a, ic + 2, jc + 1) - PH(a, ic, jc + 1)) * m.dx_inv;
        tn[a] = 0.5f * (PH(a, in + 2, jn + 1) - PH(a, in, jn + 1)) * m.dx_inv;
      }
      any |= (gn[a] != 0.f) | (tc[a] != 0.f) | (tn[a] != 0.f);
    }
    if (!any) return;
    const float* trc = trow(1, jc);  // the two cells' temperatures (concentration half step)
    const float* trn = trow(1, jn);
    const float tl = 0.5f * (tc[L] + tn[L]);
    const float norm_l = sqrtf(tl * tl + gn[L] * gn[L]);
#pragma unroll
    for (int a = 0; a < N - 1; a++) {
      const float ta = 0.5f * (tc[a] + tn[a]);
      const float n2 = ta * ta + gn[a] * gn[a];
      if (n2 == 0.f) continue;
      const float rn = rsqrtf(n2);
      float sp = gn[a] * gn[L] + ta * tl;
      if (norm_l > 0.f) sp *= rn / norm_l;
      float sc = 1.f, sn = 1.f;
      if (m.obstacle) {
        const float uc = pc[a] * (1.f - pc[a]), un = pn[a] * (1.f - pn[a]);
        sc = uc > 0.f ? pc[a] * (1.f - hphi<N>(pc, a)) * rsqrtf(uc) : 0.f;
        sn = un > 0.f ? pn[a] * (1.f - hphi<N>(pn, a)) * rsqrtf(un) : 0.f;
      }
      const float dpc = sdp[(a * X1 + ic) * Y1 + jc], dpn = sdp[(a * X1 + in) * Y1 + jn];
      const float pref = fabsf(sp) * (m.obstacle ? 0.5f : m.s_well) * gn[a] * rn;
#pragma unroll
      for (int k = 0; k < K1; k++) {
        const float dcn = c_mu_t<K1>(m, mun, L, k, trn) - c_mu_t<K1>(m, mun, a, k, trn);
        const float dcc = c_mu_t<K1>(m, muc, L, k, trc) - c_mu_t<K1>(m, muc, a, k, trc);
        const float jt = m.atf[a][k] * pref * (sn * dcn * dpn + sc * dcc * dpc);
        out[k] = __fsub_rn(out[k], __fmul_rn(xface ? m.jsx : m.jsy, jt));
      }
    }
  };

  // x-faces between region-1 rows i and i+1, i in [0, TX], tile columns
  for (int e = threadIdx.x; e < (TX + 1) * TY; e += nt) {
    const int i = e / TY, j = 1 + e % TY;
    float f[K1];
    face_flux(i, j, true, false, f);
#pragma unroll
    for (int k = 0; k < K1; k++) sfx[(k * (TX + 1) + i) * TY + (j - 1)] = f[k];
  }
  // y-faces between region-1 columns j and j+1, j in [0, TY], tile rows; the face whose
  // lower cell sits on interior row mesh_y-5 (gidy == MESH_Y-2) carries no antitrapping
  // current (calculate_fluxes_concentration.h:65)
  for (int e = threadIdx.x; e < TX * (TY + 1); e += nt) {
    const int i = 1 + e / (TY + 1), j = e % (TY + 1);
    float f[K1];
    face_flux(i, j, false, y0 - 1 + j == m.skip_row, f);
#pragma unroll
    for (int k = 0; k < K1; k++) sfy[(k * TX + (i - 1)) * (TY + 1) + j] = f[k];
  }
  __syncthreads();

  // ---- mu and phi update of the tile (calculate_divergence_concentration.h:4-153)
  uint8_t* s_cls = reinterpret_cast<uint8_t*>(sm + T::o_list);  // [TX][TY] one-hot phase of the output, or 0xFF
  for (int ti = warp; ti < TX; ti += nw) {
    const int x = x0 + ti;
    if (x >= mx) break;
#pragma unroll
    for (int c0 = 0; c0 < TY; c0 += 32) {
      const int tj = c0 + lane, y = y0 + tj;
      if (y >= my) continue;
      const int i1 = ti + 1, j1 = tj + 1;
      float ph[N], dp[N], mu[K1], dc[K1];
#pragma unroll
      for (int a = 0; a < N; a++) {
        ph[a] = PH(a, i1 + 1, j1 + 1);
        dp[a] = sdp[(a * X1 + i1) * Y1 + j1];
      }
#pragma unroll
      for (int k = 0; k < K1; k++) {
        mu[k] = MU(k, i1, j1);
        const float fxp_ = sfx[(k * (TX + 1) + ti + 1) * TY + tj], fxm_ = sfx[(k * (TX + 1) + ti) * TY + tj];
        const float fyp_ = sfy[(k * TX + ti) * (TY + 1) + tj + 1], fym_ = sfy[(k * TX + ti) * (TY + 1) + tj];
        dc[k] = m.comp ? flux_div_c(fxp_, fxm_, fyp_, fym_) : flux_div(fxp_, fxm_, fyp_, fym_);
      }
      int bulk = -1;
#pragma unroll
      for (int a = 0; a < N; a++)
        if (bulk < 0 && ph[a] == 1.f) bulk = a;
      float mnew[K1];
      if (bulk >= 0) {
        // phi one-hot `bulk` on the 3x3 neighbourhood: the pure-phase update (the lean kernels' arithmetic)
        bool p3 = true;
#pragma unroll
        for (int di = -1; di <= 1; di++)
#pragma unroll
          for (int dj = -1; dj <= 1; dj++)
#pragma unroll
            for (int a = 0; a < N; a++) p3 &= PH(a, i1 + 1 + di, j1 + 1 + dj) == (a == bulk ? 1.f : 0.f);
        if (p3) {
          float gx[MK][MK], gy[MK][MK], dxp[K1], dxm[K1], dyp[K1], dym[K1];
          phase_mat<N, K1>(m.Gx, bulk, gx);
          phase_mat<N, K1>(m.Gy, bulk, gy);
#pragma unroll
          for (int k = 0; k < K1; k++) {
            dxp[k] = __fsub_rn(MU(k, i1 + 1, j1), mu[k]);
            dxm[k] = __fsub_rn(mu[k], MU(k, i1 - 1, j1));
            dyp[k] = __fsub_rn(MU(k, i1, j1 + 1), mu[k]);
            dym[k] = __fsub_rn(mu[k], MU(k, i1, j1 - 1));
          }
          pure_update<K1>(gx, gy, mu, dxp, dxm, dyp, dym, mnew, m.comp);
        } else {
          float hb[MK][MK];
          phase_mat<N, K1>(m.H, bulk, hb);
          bulk_update_h<K1>(hb, mu, dc, mnew, m.comp);
        }
      } else {
        float hh[N], dce[K1];
        const float* tu = trow(1, j1);
#pragma unroll
        for (int k = 0; k < K1; k++) dce[k] = 0.f;
#pragma unroll
        for (int a = 0; a < N; a++) hh[a] = hphi<N>(ph, a);
        // dc -= sum_a c_a(mu) * dh_a/dt
#pragma unroll
        for (int a = 0; a < N; a++) {
          float sdh = 0.f;
#pragma unroll
          for (int b = 0; b < N; b++) sdh += dhphi<N>(ph, a, b) * dp[b];
#pragma unroll
          for (int k = 0; k < K1; k++) {
            if (m.comp) {  // compensated: the product and the difference error-free, errors kept in dce
              float ep, es;
              const float pr = two_prod(c_mu_t<K1>(m, mu, a, k, tu), sdh, ep);
              dc[k] = two_sum(dc[k], -pr, es);
              dce[k] = __fadd_rn(dce[k], __fsub_rn(es, ep));
            } else {
              dc[k] -= c_mu_t<K1>(m, mu, a, k, tu) * sdh;
            }
          }
        }
        if (m.comp)
#pragma unroll
          for (int k = 0; k < K1; k++) dc[k] = __fadd_rn(dc[k], dce[k]);
        if (K1 == 1) {
          float d = 0.f;
#pragma unroll
          for (int a = 0; a < N; a++) d += m.cmu[a][0][0] * hh[a];
          mnew[0] = mu[0] + dc[0] / d;
        } else {
          // (dc/dmu) = sum_a cmu_a h_a, inverted in FP64
          double D[MK][MK];
#pragma unroll
          for (int k = 0; k < K1; k++)
#pragma unroll
            for (int l = 0; l < K1; l++) {
              double sv = 0.0;
#pragma unroll
              for (int a = 0; a < N; a++) sv += m.cmu_d[a][k][l] * (double)hh[a];
              D[k][l] = sv;
            }
          double dm[K1];
          if (m.mu_solver == GP_MU_BINARY) {  // BINARY = 1 updates the first potential only
#pragma unroll
            for (int k = 0; k < K1; k++) dm[k] = k == 0 ? (double)dc[0] / D[0][0] : 0.0;
          } else if (m.mu_solver == GP_MU_DILUTE) {
#pragma unroll
            for (int k = 0; k < K1; k++) dm[k] = (double)dc[k] / D[k][k];
          } else if (K1 == 2) {
            const double det = D[0][0] * D[K1 - 1][K1 - 1] - D[0][K1 - 1] * D[K1 - 1][0];
            dm[0] = (D[K1 - 1][K1 - 1] * dc[0] - D[0][K1 - 1] * dc[K1 - 1]) / det;
            dm[K1 - 1] = (D[0][0] * dc[K1 - 1] - D[K1 - 1][0] * dc[0]) / det;
          } else {
            // Gauss-Jordan with partial pivoting, K1 <= 3
            double Aug[MK][MK + 1];
#pragma unroll
            for (int k = 0; k < K1; k++) {
#pragma unroll
              for (int l = 0; l < K1; l++) Aug[k][l] = D[k][l];
              Aug[k][K1] = dc[k];
            }
#pragma unroll
            for (int c = 0; c < K1; c++) {
              int piv = c;
#pragma unroll
              for (int r = c + 1; r < K1; r++)
                if (fabs(Aug[r][c]) > fabs(Aug[piv][c])) piv = r;
#pragma unroll
              for (int r = 0; r < K1; r++)
                if (r == piv && piv != c) {
#pragma unroll
                  for (int l = 0; l <= K1; l++) {
                    const double t = Aug[c][l];
                    Aug[c][l] = Aug[r][l];
                    Aug[r][l] = t;
                  }
                }
              const double inv = 1.0 / Aug[c][c];
#pragma unroll
              for (int r = 0; r < K1; r++) {
                if (r == c) continue;
                const double f = Aug[r][c] * inv;
#pragma unroll
                for (int l = 0; l <= K1; l++) Aug[r][l] -= f * Aug[c][l];
              }
            }
#pragma unroll
            for (int k = 0; k < K1; k++) dm[k] = Aug[k][K1] / Aug[k][k];
          }
#pragma unroll
          for (int k = 0; k < K1; k++) mnew[k] = mu[k] + (float)dm[k];
        }
      }
      const int64_t o = (int64_t)x * I.pitch + y;
#pragma unroll
      for (int k = 0; k < K1; k++) I.mu_out[o + k * I.plane] = mnew[k];
      int hot = -1;
      bool onehot = true;
#pragma unroll
      for (int a = 0; a < N; a++) {
        const float v = __fadd_rn(ph[a], dp[a]);
        I.phi_out[o + a * I.plane] = v;
        if (v == 1.f && hot < 0) hot = a;
        else if (__float_as_uint(v) != 0u) onehot = false;  // -0 is not the pure field's +0
      }
      s_cls[ti * TY + tj] = (onehot && hot >= 0) ? (uint8_t)hot : (uint8_t)0xFF;
    }
  }
  __syncthreads();
  // purity word of the output tile (whole tile, first/last two rows, first/last two columns)
  {
    const int ex = min(TX, mx - x0), ey = min(TY, my - y0);
    const int r0 = s_cls[0], rxh = s_cls[(ex - 1) * TY], ryh = s_cls[ey - 1];
    unsigned bad = 0u;
    for (int e = threadIdx.x; e < TX * TY; e += nt) {
      const int i = e / TY, j = e % TY;
      if (i >= ex || j >= ey) continue;
      const int v = s_cls[e];
      if (v != r0) bad |= (i < 2 ? 3u : 1u) | (j < 2 ? 8u : 0u);
      if (i >= ex - 2 && v != rxh) bad |= 4u;
      if (j >= ey - 2 && v != ryh) bad |= 16u;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicOr(&s_bad, bad);
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned B = s_bad;
      uint32_t w = 0u;
      if (!(B & 1u) && r0 != 0xFF) w |= (uint32_t)(1 + r0) << PF_CORE;
      if (!(B & 2u) && r0 != 0xFF) w |= (uint32_t)(1 + r0) << PF_XLO;
      if (!(B & 4u) && rxh != 0xFF) w |= (uint32_t)(1 + rxh) << PF_XHI;
      if (!(B & 8u) && r0 != 0xFF) w |= (uint32_t)(1 + r0) << PF_YLO;
      if (!(B & 16u) && ryh != 0xFF) w |= (uint32_t)(1 + ryh) << PF_YHI;
      flags_out[tile] = w;
    }
  }
  }  // tile loop
  if (glist && threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&cnt[2], 1) == (int)gridDim.x - 1) {
      if (!keep_list) {  // keep_list: a second pass over the same list follows (two-step blocking)
        cnt[0] = 0;
        cnt[3] = 0;
      }
      cnt[1] = 0;
      cnt[2] = 0;
    }
  }
}

// Lean update of the tiles lean_phase accepts (phase b): diffusion of mu
// inside phase b; phi stays the one-hot field of b and is written only when
// the output buffer does not hold it already (its purity word says so).
//
// A warp updates TPW tiles at a time, LP = 32 / TPW lanes per tile.  A tile's
// mu rows x0-1 .. x0+TX, columns y0-4 .. y0+TY+3, every plane, arrive in
// shared memory as one TMA box (a tensor map per instance and buffer; cells
// outside the grid read as zero, and the ghost row/column of a tile at the
// grid edge is then written from the boundary map).  Each warp keeps a ring
// of STAGES stages of TPW boxes: while one stage is computed the next
// STAGES - 1 are loading.
//
// A row of a tile is G = TY/4 lanes of four cells each; the tile's LP/G lane
// groups take RG consecutive rows each and stream them along x: each x-face
// flux is evaluated once and carried to the next row, the y-faces from the
// lane's own cells and the neighbouring float4s of the staged row -- the same
// helper calls on the same operands as the full update's pure path, hence the
// same bits.
#ifndef GP_LEAN_STAGES
#define GP_LEAN_STAGES 2
#endif
#ifndef GP_LEAN_WARPS
#define GP_LEAN_WARPS 4
#endif
#ifndef GP_LEAN_TPW
#define GP_LEAN_TPW 2
#endif

template <int N, int K1, int TX, int TY>
struct Lean {
  static constexpr int G = TY / 4;                                      // lanes per tile row
  static constexpr int TPW = GP_LEAN_TPW < 32 / G ? GP_LEAN_TPW : 32 / G;  // tiles per warp
  static constexpr int LP = 32 / TPW;                                   // lanes per tile
  static constexpr int NG = LP / G;                                     // row groups per tile
  static constexpr int RG = TX / NG;                                    // rows per group
  static constexpr int R = TX + 2;                                      // staged rows: x0-1 .. x0+TX
  static constexpr int W = TY + 8;                                      // staged row: y0-4 .. y0+TY+3
  static constexpr int BYTES = K1 * R * W * 4;                          // one box
  static constexpr int SLOT = (BYTES + 127) / 128 * 128;
  static constexpr int STAGES = GP_LEAN_STAGES;
  static constexpr int WARPS = GP_LEAN_WARPS;                           // warps per block
  static constexpr int ENT = (8 * STAGES + 15) / 16 * 16;              // ring entries after the barriers
  static constexpr int CTRL = (ENT + 16 * STAGES * TPW + 127) / 128 * 128;
  static constexpr int WARP_BYTES = STAGES * TPW * SLOT + CTRL;
  static constexpr size_t smem = (size_t)WARPS * WARP_BYTES + 128;
  static_assert(G * NG == LP && RG * NG == TX && TPW * LP == 32, "tile shape");
  static_assert(W <= 256 && R <= 256 && W * 4 % 16 == 0, "TMA box");
};

// Constants of the lean update of one phase of one instance.
struct alignas(16) LeanConst {
  float gx[MK][MK], gy[MK][MK];  // Model::Gx, Gy of the phase
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of the barrier to complete; false after one second.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > 1000000000ull) return false;
  return true;
}

// One 3-D box (columns, rows, planes) from the tensor map into shared memory,
// completing on the barrier.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Write the ghost row/column of a tile at the grid edge into its staged box:
// the boundary map's source cell, from the box when it lies there, else from
// global memory (periodic partners).  Called by the whole warp; `on` says
// whether the lane's tile needs it, `sub` is the lane's index in its tile.
template <int N, int K1, int TX, int TY>
__device__ __forceinline__ void lean_ghosts(bool on, const Inst& I, int x0, int y0, float* buf, int sub) {
  using S = Lean<N, K1, TX, TY>;
  constexpr int R = S::R, W = S::W, LP = S::LP;
  const int mx = I.mx, my = I.my;
  const int ex = min(TX, mx - x0), ey = min(TY, my - y0);
  // ghost rows x0 - 1 (box row 0) and x0 + ex (box row ex + 1), over the tile's columns
  for (int side = 0; side < 2; side++) {
    const int gx = side ? x0 + ex : x0 - 1;
    if (on && (side ? gx >= mx : gx < 0)) {
      const int src = gp_map_any(gx, mx, I.bc.mu_x), sr = src - x0 + 1, dr = gx - x0 + 1;
      const bool in_box = sr >= 1 && sr <= ex;
      for (int c = sub; c < ey; c += LP)
#pragma unroll
        for (int k = 0; k < K1; k++)
          buf[(k * R + dr) * W + 4 + c] =
              in_box ? buf[(k * R + sr) * W + 4 + c] : I.mu[k * I.plane + (int64_t)src * I.pitch + y0 + c];
    }
  }
  __syncwarp();
  // ghost columns y0 - 1 (box column 3) and y0 + ey (box column ey + 4), over the tile's rows
  for (int side = 0; side < 2; side++) {
    const int gy = side ? y0 + ey : y0 - 1;
    if (on && (side ? gy >= my : gy < 0)) {
      const int src = gp_map_any(gy, my, I.bc.mu_y), sc = src - y0 + 4, dc = gy - y0 + 4;
      const bool in_box = sc >= 4 && sc < 4 + ey;
      for (int r = sub; r < ex; r += LP)
#pragma unroll
        for (int k = 0; k < K1; k++)
          buf[(k * R + r + 1) * W + dc] =
              in_box ? buf[(k * R + r + 1) * W + sc] : I.mu[k * I.plane + (int64_t)(x0 + r) * I.pitch + src];
    }
  }
  __syncwarp();
}

// Update tile (x0, y0) of instance I from its staged box (`sub`: the lane's
// index in the tile).  A tile inside the grid stores its rows without bounds
// tests; an edge tile tests rows and columns.  The phi of a tile whose output
// buffer does not hold the one-hot field of b yet is written in a second pass.
template <int N, int K1, int TX, int TY, bool COMP>
__device__ __forceinline__ void lean_compute(const Inst& I, const LeanConst& C, bool write_phi, int b, int x0, int y0,
                                             const float* buf, int sub) {
  using S = Lean<N, K1, TX, TY>;
  constexpr int G = S::G, RG = S::RG, R = S::R, W = S::W;
  const int lg = sub % G, grp = sub / G, xs = x0 + grp * RG, yb = y0 + 4 * lg;
  const int mx = I.mx, my = I.my;
  const bool full = x0 + TX <= mx && y0 + TY <= my;
  const int64_t pitch = I.pitch, plane = I.plane;
  float* const out = I.mu_out + (int64_t)xs * pitch + yb;
  const float* const sb = buf + grp * RG * W + 4 + 4 * lg;  // the group's first staged row, the lane's first cell
  float gx[MK][MK], gy[MK][MK];
#pragma unroll
  for (int k = 0; k < K1; k++)
#pragma unroll
    for (int l = 0; l < K1; l++) {
      gx[k][l] = C.gx[k][l];
      gy[k][l] = C.gy[k][l];
    }
  auto row = [&](int r, float (&v)[4][K1]) {
#pragma unroll
    for (int k = 0; k < K1; k++) {
      const float4 q = *reinterpret_cast<const float4*>(sb + (k * R + r) * W);
      v[0][k] = q.x;
      v[1][k] = q.y;
      v[2][k] = q.z;
      v[3][k] = q.w;
    }
  };
  float cur[4][K1], dxm[4][K1];  // dxm: the difference across each cell's lower x-face
  {
    float prev[4][K1];
    row(0, prev);
    row(1, cur);
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < K1; k++) dxm[j][k] = __fsub_rn(cur[j][k], prev[j][k]);
  }
  // the new mu of the lane's four cells in group row r (box row r + 1); advances cur and dxm
  auto step = [&](int r, float (&mnew)[4][K1]) {
    float nx[4][K1], dy[5][K1];
    row(r + 2, nx);
#pragma unroll
    for (int k = 0; k < K1; k++) {
      dy[0][k] = __fsub_rn(cur[0][k], sb[(k * R + r + 1) * W - 1]);
#pragma unroll
      for (int j = 1; j < 4; j++) dy[j][k] = __fsub_rn(cur[j][k], cur[j - 1][k]);
      dy[4][k] = __fsub_rn(sb[(k * R + r + 1) * W + 4], cur[3][k]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float dxp[K1];
#pragma unroll
      for (int k = 0; k < K1; k++) dxp[k] = __fsub_rn(nx[j][k], cur[j][k]);
      pure_update<K1>(gx, gy, cur[j], dxp, dxm[j], dy[j + 1], dy[j], mnew[j], COMP);
#pragma unroll
      for (int k = 0; k < K1; k++) dxm[j][k] = dxp[k];
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < K1; k++) cur[j][k] = nx[j][k];
  };
  if (full) {
#pragma unroll
    for (int r = 0; r < RG; r++) {
      float mnew[4][K1];
      step(r, mnew);
#pragma unroll
      for (int k = 0; k < K1; k++)
        __stwb(reinterpret_cast<float4*>(out + r * pitch + k * plane),
               make_float4(mnew[0][k], mnew[1][k], mnew[2][k], mnew[3][k]));
    }
  } else {
    const bool vec = yb + 3 < my;
#pragma unroll
    for (int r = 0; r < RG; r++) {
      float mnew[4][K1];
      step(r, mnew);
      if (xs + r < mx) {
        if (vec) {
#pragma unroll
          for (int k = 0; k < K1; k++)
            __stwb(reinterpret_cast<float4*>(out + r * pitch + k * plane),
                   make_float4(mnew[0][k], mnew[1][k], mnew[2][k], mnew[3][k]));
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (yb + j < my) {
#pragma unroll
              for (int k = 0; k < K1; k++) out[r * pitch + k * plane + j] = mnew[j][k];
            }
        }
      }
    }
  }
  if (write_phi) {
    float* const po = I.phi_out + (int64_t)xs * pitch + yb;
    for (int r = 0; r < RG && xs + r < mx; r++)
#pragma unroll
      for (int a = 0; a < N; a++) {
        const float v = a == b ? 1.f : 0.f;
        if (yb + 3 < my) {
          *reinterpret_cast<float4*>(po + r * pitch + a * plane) = make_float4(v, v, v, v);
        } else {
          for (int j = 0; j < 4 && yb + j < my; j++) po[r * pitch + a * plane + j] = v;
        }
      }
  }
}

// The lean tiles of one step.  Warps scan the tiles w, w + W, w + 2W, ...
// (W = warps of the grid), 32 candidates per ballot, and update the accepted
// ones TPW at a time through the ring of staged boxes.  With `reverse` the
// scan runs from the last tile down: steps alternate the direction, so a step
// starts on the tiles the previous step wrote last, whose mu is still in L2.  A stage whose boxes
// have not arrived after one second sets *err; the warp then waits (bounded)
// for its other boxes and returns.
template <int N, int K1, int TX, int TY, bool COMP>
__global__ void __launch_bounds__(32 * GP_LEAN_WARPS)
    k_lean32(const Inst* __restrict__ insts, const LeanConst* __restrict__ lconst,
             const CUtensorMap* __restrict__ tmaps, const int4* __restrict__ tile_desc,
             const uint32_t* __restrict__ flags_in, uint32_t* __restrict__ flags_out, int total, int reverse,
             int lose_box, int* __restrict__ err) {
  using S = Lean<N, K1, TX, TY>;
  constexpr int STAGES = S::STAGES, TPW = S::TPW, LP = S::LP;
  static_assert(STAGES >= 2, "a stage loads while another is computed");
  extern __shared__ __align__(16) unsigned char lsm_raw[];
  unsigned char* lsm = lsm_raw + ((128 - (smem_u32(lsm_raw) & 127)) & 127);
  const int lane = threadIdx.x & 31, q = lane / LP, sub = lane % LP;
  unsigned char* wsm = lsm + (threadIdx.x >> 5) * S::WARP_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsm);          // [STAGES]
  int4* ent = reinterpret_cast<int4*>(wsm + S::ENT);         // [STAGES][TPW] {tile, inst * 8 + phase, x0, y0}
  float* slots = reinterpret_cast<float*>(wsm + S::CTRL);    // [STAGES][TPW][SLOT / 4]
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) - 32 * nwarp;
  unsigned todo = 0;
  int mine = -1, mx0 = 0, my0 = 0;  // this lane's candidate: inst * 8 + phase (or -1), its origin
  if (lane == 0) {
    for (int s = 0; s < STAGES; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  // the next accepted tile of this warp (warp-uniform), tile -1 when none is left
  auto next = [&]() -> int4 {
    while (!todo) {
      base += 32 * nwarp;
      if (base >= total) return make_int4(-1, 0, 0, 0);
      int64_t tc = base + lane * nwarp;
      if (reverse) tc = total - 1 - tc;
      mine = -1;
      if (tc >= 0 && tc < total) {
        const int4 d = tile_desc[tc];  // {instance, x0, y0, tile_geo}
        const int bc = lean_phase(flags_in, (uint32_t)d.w, (int)tc);
        if (bc >= 0) {
          mine = d.x * 8 + bc;
          mx0 = d.y;
          my0 = d.z;
        }
      }
      todo = __ballot_sync(0xffffffffu, mine >= 0);
    }
    const int src = __ffs(todo) - 1;
    todo &= todo - 1;
    const int t = (int)(base + src * nwarp);
    return make_int4(reverse ? total - 1 - t : t, __shfl_sync(0xffffffffu, mine, src),
                     __shfl_sync(0xffffffffu, mx0, src), __shfl_sync(0xffffffffu, my0, src));
  };
  // record the next TPW tiles in stage s and start their boxes
  // failure-detection test: the first warp to take the token err[1] issues none of that
  // stage's boxes, so its wait expires
  auto fill = [&](int s) {
    int4 e[TPW];
    int nv = 0;
#pragma unroll
    for (int j = 0; j < TPW; j++) {
      e[j] = next();
      nv += e[j].x >= 0;
    }
    if (lane == 0) {
#pragma unroll
      for (int j = 0; j < TPW; j++) ent[s * TPW + j] = e[j];
      if (nv) {
        const bool lose = lose_box && atomicExch(&err[1], 0) != 0;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[s], nv * S::BYTES);
#pragma unroll
        for (int j = 0; j < TPW; j++)
          if (e[j].x >= 0 && !lose)
            tma_load_3d(slots + (s * TPW + j) * (S::SLOT / 4), &tmaps[e[j].y >> 3], &bar[s], e[j].w - 4,
                        e[j].z - 1, 0);
      }
    }
  };
  for (int s = 0; s < STAGES - 1; s++) fill(s);
  __syncwarp();
  uint32_t phase = 0;  // bit s: parity of stage s's next completion
  for (int s = 0;; s = s + 1 == STAGES ? 0 : s + 1) {
    if (ent[s * TPW].x < 0) break;  // stages fill in order: nothing is left
    const int4 e = ent[s * TPW + q];
    fill(s == 0 ? STAGES - 1 : s - 1);  // the stage computed in the previous pass
    const bool own = e.x >= 0;
    const int inst = own ? e.y >> 3 : 0, b = e.y & 7;
    const Inst I = insts[inst];
    const LeanConst C = lconst[inst * N + b];
    const bool write_phi = own && pf(flags_out[e.x], PF_CORE) != 1 + b;
    if (!mbar_wait(&bar[s], (phase >> s) & 1)) {
      if (lane == 0) atomicExch(err, 1);
      __syncwarp();
      for (int j = 0; j < STAGES; j++)  // every stage with boxes in flight
        if (ent[j * TPW].x >= 0) mbar_wait(&bar[j], (phase >> j) & 1);
      return;
    }
    phase ^= 1u << s;
    float* buf = slots + (s * TPW + q) * (S::SLOT / 4);
    const bool edge = own && (e.z == 0 || e.z + TX >= I.mx || e.w == 0 || e.w + TY >= I.my);
    if (__any_sync(0xffffffffu, edge)) lean_ghosts<N, K1, TX, TY>(edge, I, e.z, e.w, buf, sub);
    if (own) lean_compute<N, K1, TX, TY, COMP>(I, C, write_phi, b, e.z, e.w, buf, sub);
    __syncwarp();
    if (own && sub == 0) flags_out[e.x] = pf_all(1 + b);
  }
}

// ---------------------------------------------------------------- two steps per staged box (depth 2)

// Floats per staged row of the two-step lean kernel's box and intermediate rows: the W = TY + 8
// columns it computes, padded for 16x32 tiles to 44 (eleven 16-byte quads).  There a warp's
// sweep puts three row segments of six rows side by side in its lanes (ten float4 column groups
// each); with 40-float rows the segments' quads overlap inside an 8-lane phase of a float4
// access (bank-conflict replays), with 44 the segments' quads are offset by 2 (11 x 6 = 66 = 2
// mod 8) and each phase touches eight distinct quads.  The TMA box loads the padding columns
// too (unused).
__host__ __device__ constexpr int lean2_stride(int tx, int ty) { return (tx == 16 && ty == 32) ? ty + 12 : ty + 8; }

// A cell's update is the pure-phase one (pure_update: diffusion of mu in phase
// b, phi kept) when phi is the one-hot field of b on the cell's 3x3
// neighbourhood, and then its phi stays one-hot: the pure region shrinks by at
// most one cell per step.  So a tile lean_phase accepts (phi one-hot b on the
// tile and its two-cell ring) has its cells and its ring's first row/column pure
// for two steps, and one box of mu -- rows x0-2 .. x0+TX+1, columns y0-4 ..
// y0+TY+3, at step t -- gives the tile at t+2: sub-step 1 computes rows x0-1 ..
// x0+TX of step t+1 into a second shared array (over the box's columns; of
// those only the tile's columns and the ring column beside them are used),
// sub-step 2 the tile.  Each cell and face goes through the same helper calls
// on the same operands as two single steps, so the results are the same bits.
//
// One tile per warp; a ring of two stages (one box loading while the other is
// computed).  Lanes own a float4 column group and stream a segment of rows
// along x, carrying the x-face difference from row to row; y-neighbours come
// from the neighbouring lanes by shuffles (only the tile's outermost groups
// read the ring column from shared memory in sub-step 2).
template <int N, int K1, int TX, int TY>
struct Lean2 {
  static constexpr int R2 = TX + 4;                        // box rows x0-2 .. x0+TX+1
  static constexpr int R1 = TX + 2;                        // intermediate rows x0-1 .. x0+TX
  static constexpr int W = TY + 8;                         // columns y0-4 .. y0+TY+3
  static constexpr int WS = lean2_stride(TX, TY);          // floats per staged row (box and intermediate)
  static constexpr int Q1 = W / 4;                         // column groups of sub-step 1
  static constexpr int Q2 = TY / 4;                        // column groups of sub-step 2 (the tile)
  static constexpr int S1 = 32 / Q1 > 0 ? 32 / Q1 : 1;     // row segments of sub-step 1
  static constexpr int RS1 = (R1 + S1 - 1) / S1;           // rows per segment
  static constexpr int S2 = 32 / Q2;
  static constexpr int RS2 = (TX + S2 - 1) / S2;
  static constexpr int BYTES = K1 * R2 * WS * 4;           // one box
  static constexpr int SLOT = (BYTES + 127) / 128 * 128;
  static constexpr int MID = (K1 * R1 * WS * 4 + 127) / 128 * 128;
  static constexpr int STAGES = 2;
  static constexpr int WARPS = 4;
  static constexpr int CTRL = 128;                         // barriers, ring entries
  static constexpr int WARP_BYTES = CTRL + STAGES * SLOT + MID;
  static constexpr size_t smem = (size_t)WARPS * WARP_BYTES + 128;
  static_assert(Q1 <= 32 && Q2 * S2 <= 32 && S2 >= 1, "tile shape");
  static_assert(W <= 256 && R2 <= 256 && W * 4 % 16 == 0, "TMA box");
};

// One lane's diffusion sweep over output rows [r0, r1) of a staged array with
// R rows of W columns per plane: output row r comes from source rows r, r+1,
// r+2 (the source starts one row earlier) at columns c0 .. c0+3.  The
// y-neighbours c0-1 and c0+4 come from the lanes holding them (shuffles: the
// warp's lanes hold consecutive groups of a segment; a segment's outermost
// lanes get an unused value) or, where ld_left / ld_right, from the array.
// Every lane runs RS rows (the shuffles need the whole warp); rows at or past
// r1 are computed from clamped rows and not stored.  put(r, mnew) stores a
// row's four new cells.
template <int K1, int R, int W, int WS, int RS, bool COMP, typename Put>
__device__ __forceinline__ void lean_sweep(const float* __restrict__ src, int c0, int r0, int r1, bool ld_left,
                                           bool ld_right, const float (&gx)[MK][MK], const float (&gy)[MK][MK],
                                           Put put) {
  const int cl = c0 > 0 ? c0 - 1 : 0, cr = c0 + 4 < W ? c0 + 4 : W - 1;
  auto row = [&](int r, float (&v)[4][K1]) {
    r = r < R - 1 ? r : R - 1;
#pragma unroll
    for (int k = 0; k < K1; k++) {
      const float4 q = *reinterpret_cast<const float4*>(src + (k * R + r) * WS + c0);
      v[0][k] = q.x;
      v[1][k] = q.y;
      v[2][k] = q.z;
      v[3][k] = q.w;
    }
  };
  float cur[4][K1], dxm[4][K1];
  {
    float prev[4][K1];
    row(r0, prev);
    row(r0 + 1, cur);
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < K1; k++) dxm[j][k] = __fsub_rn(cur[j][k], prev[j][k]);
  }
#pragma unroll
  for (int i = 0; i < RS; i++) {
    const int r = r0 + i;
    const int rr = r + 1 < R - 1 ? r + 1 : R - 1;
    float nx[4][K1], dy[5][K1], mnew[4][K1];
    row(r + 2, nx);
#pragma unroll
    for (int k = 0; k < K1; k++) {
      float left = __shfl_up_sync(0xffffffffu, cur[3][k], 1), right = __shfl_down_sync(0xffffffffu, cur[0][k], 1);
      if (ld_left) left = src[(k * R + rr) * WS + cl];
      if (ld_right) right = src[(k * R + rr) * WS + cr];
      dy[0][k] = __fsub_rn(cur[0][k], left);
#pragma unroll
      for (int j = 1; j < 4; j++) dy[j][k] = __fsub_rn(cur[j][k], cur[j - 1][k]);
      dy[4][k] = __fsub_rn(right, cur[3][k]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      float dxp[K1];
#pragma unroll
      for (int k = 0; k < K1; k++) dxp[k] = __fsub_rn(nx[j][k], cur[j][k]);
      pure_update<K1>(gx, gy, cur[j], dxp, dxm[j], dy[j + 1], dy[j], mnew[j], COMP);
#pragma unroll
      for (int k = 0; k < K1; k++) dxm[j][k] = dxp[k];
    }
    if (r < r1) put(r, mnew);
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < K1; k++) cur[j][k] = nx[j][k];
  }
}

// Cells of a staged mu array (rows gx0 .. gx0+R-1, columns gy0 .. gy0+W-1 of
// instance I, K1 planes, WS floats per stored row) on the grid's first ghost row or column (-1, M) get
// their boundary-map source: from the array when the source lies in it, else
// from `gmu` (the state the array holds; the periodic partner of a row or
// column the array crosses).  Ghost rows over the grid's columns first, then
// ghost columns over the grid's rows.  Called by the whole warp.
template <int K1, int R, int W, int WS>
__device__ __forceinline__ void lean2_ghosts(const Inst& I, int gx0, int gy0, float* buf, const float* gmu,
                                             int lane) {
  const int mx = I.mx, my = I.my;
  const int ylo = max(0, gy0), yhi = min(my, gy0 + W), xlo = max(0, gx0), xhi = min(mx, gx0 + R);
  for (int side = 0; side < 2; side++) {
    const int gx = side ? mx : -1, dr = gx - gx0;
    if (dr < 0 || dr >= R) continue;
    const int src = gp_map(gx, mx, I.bc.mu_x), sr = src - gx0;
    const bool in_buf = sr >= 0 && sr < R;
    if (!in_buf && !gmu) continue;
    for (int gy = ylo + lane; gy < yhi; gy += 32)
#pragma unroll
      for (int k = 0; k < K1; k++)
        buf[(k * R + dr) * WS + (gy - gy0)] =
            in_buf ? buf[(k * R + sr) * WS + (gy - gy0)] : gmu[k * I.plane + (int64_t)src * I.pitch + gy];
  }
  __syncwarp();
  for (int side = 0; side < 2; side++) {
    const int gy = side ? my : -1, dc = gy - gy0;
    if (dc < 0 || dc >= W) continue;
    const int src = gp_map(gy, my, I.bc.mu_y), sc = src - gy0;
    const bool in_buf = sc >= 0 && sc < W;
    if (!in_buf && !gmu) continue;
    for (int gx = xlo + lane; gx < xhi; gx += 32)
#pragma unroll
      for (int k = 0; k < K1; k++)
        buf[(k * R + (gx - gx0)) * WS + dc] =
            in_buf ? buf[(k * R + (gx - gx0)) * WS + sc] : gmu[k * I.plane + (int64_t)gx * I.pitch + src];
  }
  __syncwarp();
}

// Some existing neighbour of tile t is listed for the full kernel (gen[] from k_general_list).
__device__ __forceinline__ bool next_to_full(const uint8_t* __restrict__ gen, uint32_t geo, int t) {
  const int ny = (int)(geo & TG_NY);
  const bool xm = geo & TG_XM, xp = geo & TG_XP, ym = geo & TG_YM, yp = geo & TG_YP;
  bool f = false;
  f |= xm && gen[t - ny];
  f |= xp && gen[t + ny];
  f |= ym && gen[t - 1];
  f |= yp && gen[t + 1];
  f |= xm && ym && gen[t - ny - 1];
  f |= xm && yp && gen[t - ny + 1];
  f |= xp && ym && gen[t + ny - 1];
  f |= xp && yp && gen[t + ny + 1];
  return f;
}

// The frozen temperature gradient's clock, one step on: launched after every full-kernel pass of
// a non-isothermal batch (that pass read the step it computed at its tiles' start).
__global__ void k_tick(long long* t) { *t += 1; }

// The lean tiles of a blocked pair that border a tile of the full kernel's list,
// as entries {tile, inst * 8 + phase, x0, y0} (count in cnt[4]).
__global__ void __launch_bounds__(256) k_adj_list(const int4* __restrict__ tile_desc,
                                                  const uint32_t* __restrict__ flags_in,
                                                  const uint8_t* __restrict__ gen, int total,
                                                  int4* __restrict__ alist, int* __restrict__ cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int4 d = make_int4(0, 0, 0, 0);
  bool adj = false;
  int b = -1;
  if (t < total && !gen[t]) {
    d = tile_desc[t];
    b = lean_phase(flags_in, (uint32_t)d.w, t);
    adj = b >= 0 && next_to_full(gen, (uint32_t)d.w, t);
  }
  const unsigned bal = __ballot_sync(0xffffffffu, adj);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && bal) base = atomicAdd(&cnt[4], __popc(bal));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (adj) alist[base + __popc(bal & ((1u << lane) - 1u))] = make_int4(t, d.x * 8 + b, d.y, d.z);
}

// Two steps of the lean tiles of a blocked pair.  alist given (adjacent mode):
// the listed tiles (lean tiles next to the full kernel's tiles), warp w taking
// entries w, w + warps, ...; they also store their step t+1 (mu, and phi unless
// the buffer holds it) into the intermediate buffer X (insts_x[i].phi_out /
// mu_out, purity words flags_x) for the full kernel's second pass.  Otherwise
// the lean tiles not next to the list, found by scanning.  Bounded waits as
// k_lean32.
template <int N, int K1, int TX, int TY, bool COMP>
__global__ void __launch_bounds__(32 * Lean2<N, K1, TX, TY>::WARPS)
    k_lean2(const Inst* __restrict__ insts, const Inst* __restrict__ insts_x, const LeanConst* __restrict__ lconst,
            const CUtensorMap* __restrict__ tmaps, const int4* __restrict__ tile_desc,
            const uint32_t* __restrict__ flags_in, uint32_t* __restrict__ flags_out, uint32_t* __restrict__ flags_x,
            const uint8_t* __restrict__ gen, int total, int reverse, const int4* __restrict__ alist,
            const int* __restrict__ acnt, int* __restrict__ err) {
  using S = Lean2<N, K1, TX, TY>;
  constexpr int R1 = S::R1, R2 = S::R2, W = S::W, WS = S::WS, STAGES = S::STAGES, Q1 = S::Q1, Q2 = S::Q2;
  extern __shared__ __align__(16) unsigned char lsm_raw[];
  unsigned char* lsm = lsm_raw + ((128 - (smem_u32(lsm_raw) & 127)) & 127);
  const int lane = threadIdx.x & 31;
  unsigned char* wsm = lsm + (threadIdx.x >> 5) * S::WARP_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsm);                    // [STAGES]
  int4* ent = reinterpret_cast<int4*>(wsm + 64);                       // [STAGES] {tile, inst * 8 + phase, x0, y0}
  float* slots = reinterpret_cast<float*>(wsm + S::CTRL);              // [STAGES][SLOT / 4]
  float* mid = reinterpret_cast<float*>(wsm + S::CTRL + STAGES * S::SLOT);  // [K1][R1][W]
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int64_t base = wid - 32 * nwarp;
  int64_t ai = wid - nwarp;  // adjacent mode: the last list entry taken
  const int na = alist ? *acnt : 0;
  unsigned todo = 0;
  int mine = -1, mx0 = 0, my0 = 0;
  if (lane == 0) {
    for (int s = 0; s < STAGES; s++) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  auto next = [&]() -> int4 {
    if (alist) {
      ai += nwarp;
      return ai < na ? alist[ai] : make_int4(-1, 0, 0, 0);
    }
    while (!todo) {
      base += 32 * nwarp;
      if (base >= total) return make_int4(-1, 0, 0, 0);
      int64_t tc = base + lane * nwarp;
      if (reverse) tc = total - 1 - tc;
      mine = -1;
      if (tc >= 0 && tc < total && !gen[tc]) {
        const int4 d = tile_desc[tc];
        const uint32_t geo = (uint32_t)d.w;
        const int bc = lean_phase(flags_in, geo, (int)tc);
        if (bc >= 0 && !next_to_full(gen, geo, (int)tc)) {
          mine = d.x * 8 + bc;
          mx0 = d.y;
          my0 = d.z;
        }
      }
      todo = __ballot_sync(0xffffffffu, mine >= 0);
    }
    const int src = __ffs(todo) - 1;
    todo &= todo - 1;
    const int t = (int)(base + src * nwarp);
    return make_int4(reverse ? total - 1 - t : t, __shfl_sync(0xffffffffu, mine, src),
                     __shfl_sync(0xffffffffu, mx0, src), __shfl_sync(0xffffffffu, my0, src));
  };
  auto fill = [&](int s) {
    const int4 e = next();
    if (lane == 0) {
      ent[s] = e;
      if (e.x >= 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[s], S::BYTES);
        tma_load_3d(slots + s * (S::SLOT / 4), &tmaps[e.y >> 3], &bar[s], e.w - 4, e.z - 2, 0);
      }
    }
  };
  // lane layouts of the two sub-steps (lanes outside every segment run a dummy sweep: no stores)
  const int seg1 = lane / Q1, g2 = lane % Q2, seg2 = lane / Q2;
  const bool live1 = seg1 < S::S1, live2 = seg2 < S::S2;
  // a dead lane of sub-step 1 reads what the live lane two below it reads (the same 8-lane phase
  // for 16x32 tiles: no extra shared-memory wavefront) and stores nothing (e1 = 0)
  const int l1 = live1 ? lane : (lane >= 2 ? lane - 2 : 0);
  const int a1 = (l1 / Q1) * S::RS1, e1 = live1 ? min(R1, a1 + S::RS1) : 0;
  const int a2 = live2 ? seg2 * S::RS2 : 0, e2 = live2 ? min(TX, a2 + S::RS2) : 0;
  const int c1 = 4 * (l1 % Q1);
  for (int s = 0; s < STAGES - 1; s++) fill(s);
  __syncwarp();
  uint32_t phase = 0;
  for (int s = 0;; s = s + 1 == STAGES ? 0 : s + 1) {
    const int4 e = ent[s];
    if (e.x < 0) break;
    fill(s == 0 ? STAGES - 1 : s - 1);
    const int inst = e.y >> 3, b = e.y & 7, x0 = e.z, y0 = e.w;
    const Inst I = insts[inst];
    const LeanConst C = lconst[inst * N + b];
    const bool adjm = alist != nullptr;
    const bool write_phi = pf(flags_out[e.x], PF_CORE) != 1 + b;
    const bool write_phi_x = adjm && pf(flags_x[e.x], PF_CORE) != 1 + b;
    if (!mbar_wait(&bar[s], (phase >> s) & 1)) {
      if (lane == 0) atomicExch(err, 1);
      __syncwarp();
      for (int j = 0; j < STAGES; j++)
        if (ent[j].x >= 0) mbar_wait(&bar[j], (phase >> j) & 1);
      return;
    }
    phase ^= 1u << s;
    float* box = slots + s * (S::SLOT / 4);
    const int mx = I.mx, my = I.my;
    const int ex = min(TX, mx - x0), ey = min(TY, my - y0);
    // the box's cells on the grid's first ghost row/column: boundary map of step t
    if (x0 - 2 < 0 || x0 + TX + 2 > mx || y0 - 4 < 0 || y0 + TY + 4 > my)
      lean2_ghosts<K1, R2, W, WS>(I, x0 - 2, y0 - 4, box, I.mu, lane);
    float gx[MK][MK], gy[MK][MK];
#pragma unroll
    for (int k = 0; k < K1; k++)
#pragma unroll
      for (int l = 0; l < K1; l++) {
        gx[k][l] = C.gx[k][l];
        gy[k][l] = C.gy[k][l];
      }
    // sub-step 1: rows x0-1 .. x0+TX of step t+1 into mid
    lean_sweep<K1, R2, W, WS, S::RS1, COMP>(box, c1, a1, e1, false, false, gx, gy, [&](int r, const float (&v)[4][K1]) {
#pragma unroll
      for (int k = 0; k < K1; k++)
        *reinterpret_cast<float4*>(mid + (k * R1 + r) * WS + c1) = make_float4(v[0][k], v[1][k], v[2][k], v[3][k]);
    });
    __syncwarp();
    // step t+1 ghosts of a tile at the grid edge (Neumann: sources inside mid)
    if (x0 == 0 || x0 + ex == mx || y0 == 0 || y0 + ey == my)
      lean2_ghosts<K1, R1, W, WS>(I, x0 - 1, y0 - 4, mid, nullptr, lane);
    if (adjm) {  // the tile at step t+1 into X for the full kernel's second pass
      const Inst& X = insts_x[inst];
      for (int e3 = lane; e3 < ex * Q2; e3 += 32) {
        const int r = e3 / Q2, g = e3 % Q2, yb = y0 + 4 * g;
        if (yb >= my) continue;
        const int64_t o = (int64_t)(x0 + r) * X.pitch + yb;
#pragma unroll
        for (int k = 0; k < K1; k++) {
          const float* v = mid + (k * R1 + r + 1) * WS + 4 + 4 * g;
          if (yb + 3 < my) {
            *reinterpret_cast<float4*>(X.mu_out + o + k * X.plane) = *reinterpret_cast<const float4*>(v);
          } else {
            for (int j = 0; j < 4 && yb + j < my; j++) X.mu_out[o + k * X.plane + j] = v[j];
          }
        }
        if (write_phi_x)
#pragma unroll
          for (int aa = 0; aa < N; aa++) {
            const float pv = aa == b ? 1.f : 0.f;
            if (yb + 3 < my) *reinterpret_cast<float4*>(X.phi_out + o + aa * X.plane) = make_float4(pv, pv, pv, pv);
            else
              for (int j = 0; j < 4 && yb + j < my; j++) X.phi_out[o + aa * X.plane + j] = pv;
          }
      }
    }
    __syncwarp();
    // sub-step 2: the tile at step t+2
    {
      const int yb = y0 + 4 * g2;
      const bool full = x0 + TX <= mx && y0 + TY <= my;
      float* const out = I.mu_out + (int64_t)x0 * I.pitch + yb;
      lean_sweep<K1, R1, W, WS, S::RS2, COMP>(
          mid, 4 + 4 * g2, a2, e2, g2 == 0, g2 == Q2 - 1, gx, gy, [&](int r, const float (&v)[4][K1]) {
            if (full) {
#pragma unroll
              for (int k = 0; k < K1; k++)
                __stwb(reinterpret_cast<float4*>(out + r * I.pitch + k * I.plane),
                       make_float4(v[0][k], v[1][k], v[2][k], v[3][k]));
            } else if (x0 + r < mx && yb < my) {
              if (yb + 3 < my) {
#pragma unroll
                for (int k = 0; k < K1; k++)
                  __stwb(reinterpret_cast<float4*>(out + r * I.pitch + k * I.plane),
                         make_float4(v[0][k], v[1][k], v[2][k], v[3][k]));
              } else {
#pragma unroll
                for (int j = 0; j < 4; j++)
                  if (yb + j < my)
#pragma unroll
                    for (int k = 0; k < K1; k++) out[r * I.pitch + k * I.plane + j] = v[j][k];
              }
            }
          });
      if (write_phi) {
        float* const po = I.phi_out + (int64_t)x0 * I.pitch + yb;
        for (int r = a2; r < e2 && x0 + r < mx; r++)
#pragma unroll
          for (int aa = 0; aa < N; aa++) {
            const float v = aa == b ? 1.f : 0.f;
            if (yb + 3 < my) {
              *reinterpret_cast<float4*>(po + r * I.pitch + aa * I.plane) = make_float4(v, v, v, v);
            } else {
              for (int j = 0; j < 4 && yb + j < my; j++) po[r * I.pitch + aa * I.plane + j] = v;
            }
          }
      }
    }
    __syncwarp();
    if (lane == 0) {
      flags_out[e.x] = pf_all(1 + b);
      if (adjm) flags_x[e.x] = pf_all(1 + b);
    }
  }
}

// The tiles of one step that lean_phase rejects, listed for the full kernel:
// tiles whose own cells are not all one pure phase from glist[0] up (count in
// cnt[0]), the others (an interface only in their ring) from glist[total - 1]
// down (count in cnt[3]).  For a two-step blocked pair (depth 2) the tiles
// marked TG_REJECT2 are listed too, and gen[t] records which tiles are listed.
template <int TX, int TY>
__global__ void __launch_bounds__(256) k_general_list(const int4* __restrict__ tile_desc,
                                                      const uint32_t* __restrict__ flags_in, int total,
                                                      int2* __restrict__ glist, int* __restrict__ cnt,
                                                      uint8_t* __restrict__ genb, int depth) {
  // the full kernel that reads this list may start its blocks now; they wait for this kernel's end
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int4 d = make_int4(0, 0, 0, 0);
  if (t < total) d = tile_desc[t];
  const bool gen = t < total && (lean_phase(flags_in, (uint32_t)d.w, t) < 0 ||
                                 (depth > 1 && ((uint32_t)d.w & TG_REJECT2)));
  if (genb && t < total) genb[t] = gen ? 1 : 0;
  if (depth > 1 && t == 0) cnt[4] = 0;  // the adjacency list (k_adj_list) of this pair starts empty
  const bool ring = gen && pf(flags_in[t], PF_CORE) != 0;  // pure inside
  const unsigned bal = __ballot_sync(0xffffffffu, gen && !ring), balr = __ballot_sync(0xffffffffu, ring);
  const int lane = threadIdx.x & 31;
  int base = 0, baser = 0;
  if (lane == 0 && bal) base = atomicAdd(&cnt[0], __popc(bal));
  if (lane == 0 && balr) baser = atomicAdd(&cnt[3], __popc(balr));
  base = __shfl_sync(0xffffffffu, base, 0);
  baser = __shfl_sync(0xffffffffu, baser, 0);
  const unsigned below = (1u << lane) - 1u;
  if (gen && !ring) glist[base + __popc(bal & below)] = make_int2(t, d.x);
  if (ring) glist[total - 1 - (baser + __popc(balr & below))] = make_int2(t, d.x);
}

// ---------------------------------------------------------------- host side

Model make_model(const gp_model& g) {
  Model m;
  memset(&m, 0, sizeof m);
  m.dx_inv = (float)(1.0 / g.dx);
  m.dy_inv = (float)(1.0 / g.dy);
  m.half_dy_inv = (float)(0.5 / g.dy);
  m.dt = (float)g.dt;
  m.eps = (float)g.epsilon;
  m.inv_eps = (float)(1.0 / g.epsilon);
  m.tau = (float)g.tau;
  m.w_obst = (float)g.w_obstacle;
  m.jscale = (float)(g.obstacle ? g.jat_obst : g.jat_well);
  m.hx = (float)(0.5 * g.dt / (g.dx * g.dx));
  m.hy = (float)(0.5 * g.dt / (g.dy * g.dy));
  m.jsx = (float)((g.obstacle ? g.jat_obst : g.jat_well) / g.dx);
  m.jsy = (float)((g.obstacle ? g.jat_obst : g.jat_well) / g.dy);
  m.s_well = (float)g.s_well;
  m.obstacle = g.obstacle;
  m.mu_solver = g.mu_solver;
  m.skip_row = (int)g.mesh_y - 5;
  const int N = g.N, K1 = g.K1;
  for (int a = 0; a < MP; a++)
    for (int b = 0; b < MP; b++) {
      m.Gamma[a][b] = (float)g.Gamma[a][b];
      m.tau_ab[a][b] = (float)g.tau_ab[a][b];
      m.dab[a][b] = g.anisotropy ? (float)g.dab[a][b] : 0.f;  // an isotropic instance of an anisotropic batch: a_c = 1
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
          m.R[a][b][i][j] = (float)g.R[a][b][i][j];
          m.Rinv[a][b][i][j] = (float)g.Rinv[a][b][i][j];
        }
      for (int c = 0; c < MP; c++) m.Gabc[a][b][c] = (float)g.Gamma_abc[a][b][c];
    }
  for (int a = 0; a < N; a++) {
    m.C[a] = (float)g.C[a];
    for (int i = 0; i < K1; i++) {
      m.Beff[a][i] = (float)g.Beff[a][i];
      m.B[a][i] = (float)g.B[a][i];
      m.atf[a][i] = (float)(1.0 - g.Diff[a][i][i] / g.Diff[N - 1][i][i]);
      for (int j = 0; j < K1; j++) {
        m.cmu[a][i][j] = (float)g.cmu[a][i][j];
        m.cmu_d[a][i][j] = g.cmu[a][i][j];
        m.A[a][i][j] = (float)g.A[a][i][j];
        double s = 0.0;
        for (int k = 0; k < K1; k++) s += g.Diff[a][i][k] * g.cmu[a][k][j];
        m.DC[a][i][j] = (float)s;
        m.H[a][i][j] = (float)(i == j ? 2.0 * g.A[a][i][i] : g.A[a][i][j]);
      }
    }
    // Gx = H (2 DC) dt / (2 dx^2), Gy likewise, folded in double
    for (int i = 0; i < K1; i++)
      for (int j = 0; j < K1; j++) {
        double s = 0.0;
        for (int k = 0; k < K1; k++) {
          double dc = 0.0;
          for (int l = 0; l < K1; l++) dc += g.Diff[a][k][l] * g.cmu[a][l][j];
          s += (k == i ? 2.0 * g.A[a][i][i] : g.A[a][i][k]) * 2.0 * dc;
        }
        m.Gx[a][i][j] = (float)(s * 0.5 * g.dt / (g.dx * g.dx));
        m.Gy[a][i][j] = (float)(s * 0.5 * g.dt / (g.dy * g.dy));
      }
  }
  return m;
}

}  // namespace gp32

using namespace gp32;

// Kernels of one (N, K1, anisotropy, tile shape).
struct KernelSet {
  void (*general)(const Inst*, const Model*, const int*, const int2*, int*, uint32_t*, int, const int4*,
                  const uint32_t*, int);
  void (*general_wide)(const Inst*, const Model*, const int*, const int2*, int*, uint32_t*, int, const int4*,
                       const uint32_t*, int);  // 512 threads
  void (*lean)(const Inst*, const LeanConst*, const CUtensorMap*, const int4*, const uint32_t*, uint32_t*, int, int,
               int, int*);
  void (*lean2)(const Inst*, const Inst*, const LeanConst*, const CUtensorMap*, const int4*, const uint32_t*,
                uint32_t*, uint32_t*, const uint8_t*, int, int, const int4*, const int*, int*);
  void (*list)(const int4*, const uint32_t*, int, int2*, int*, uint8_t*, int);
  size_t smem_general, smem_lean, smem_lean2;
  size_t smem_temp;  // the full kernel's temperature table (non-isothermal batches add it to smem_general)
  // the lean kernels with compensated accumulation (a template switch: the plain ones keep
  // their registers)
  decltype(lean) lean_c;
  decltype(lean2) lean2_c;
};

template <int N, int K1, bool AN, int TX, int TY>
static KernelSet make_set() {
  KernelSet k;
  k.general = k_step32<N, K1, AN, TX, TY>;
  k.general_wide = nullptr;
  if constexpr (N == 2 && K1 == 1) k.general_wide = k_step32<N, K1, AN, TX, TY, 512>;
  k.lean = k_lean32<N, K1, TX, TY, false>;
  k.lean2 = k_lean2<N, K1, TX, TY, false>;
  k.lean_c = k_lean32<N, K1, TX, TY, true>;
  k.lean2_c = k_lean2<N, K1, TX, TY, true>;
  k.list = k_general_list<TX, TY>;
  k.smem_general = Tile<N, K1, AN, TX, TY>::bytes;
  k.smem_temp = Tile<N, K1, AN, TX, TY>::bytes_temp;
  k.smem_lean = Lean<N, K1, TX, TY>::smem;
  k.smem_lean2 = Lean2<N, K1, TX, TY>::smem;
  return k;
}

template <int N, int K1, bool AN>
static bool pick_tile(int tx, int ty, KernelSet* k) {
  if (tx == 16 && ty == 32) { *k = make_set<N, K1, AN, 16, 32>(); return true; }
  if (tx == 8 && ty == 32) { *k = make_set<N, K1, AN, 8, 32>(); return true; }
  if constexpr (N <= 4) {  // five or six phases: the larger tiles' shared memory exceeds a block's
    if (tx == 32 && ty == 32) { *k = make_set<N, K1, AN, 32, 32>(); return true; }
    if (tx == 16 && ty == 64) { *k = make_set<N, K1, AN, 16, 64>(); return true; }
  }
  return false;
}

static bool pick(int N, int K1, int an, int tx, int ty, KernelSet* k) {
#define GP_PICK(NN, KK)                                                                        \
  if (N == NN && K1 == KK) return an ? pick_tile<NN, KK, true>(tx, ty, k) : pick_tile<NN, KK, false>(tx, ty, k);
  GP_PICK(2, 1) GP_PICK(2, 2) GP_PICK(3, 1) GP_PICK(3, 2) GP_PICK(4, 1) GP_PICK(4, 2)
  GP_PICK(2, 3) GP_PICK(3, 3) GP_PICK(4, 3) GP_PICK(5, 1) GP_PICK(5, 2) GP_PICK(5, 3)
  GP_PICK(6, 1) GP_PICK(6, 2) GP_PICK(6, 3)
#undef GP_PICK
  return false;
}

int gp_f32_supported(const gp_model& m) {
  KernelSet k;
  return pick(m.N, m.K1, m.anisotropy, 16, 32, &k);
}

// tile shapes offered to the autotuner
static const int kTileShapes[][2] = {{16, 32}, {8, 32}, {32, 32}, {16, 64}};
static const int kNumTileShapes = 4;

int gp_f32_tile_shape_count() { return kNumTileShapes; }
void gp_f32_tile_shape(int i, int* tx, int* ty) {
  *tx = kTileShapes[i][0];
  *ty = kTileShapes[i][1];
}

// A batch of FP32 instances on the current device.
struct gp_f32_batch {
  int n = 0, N = 0, K1 = 0, aniso = 0;
  int tx = 16, ty = 32;  // tile shape (autotuned)
  int narrowband = 1;    // send the tiles lean_phase accepts to the lean kernel
  int depth = 1;         // steps per blocked launch: 1, or 2 (lean tiles two steps per box; needs X)
  int has_x = 0;         // intermediate buffers X bound (gp_f32_batch_bind_x)
  int comp = 0;          // compensated accumulation (Model::comp of every instance, lean_c / lean2_c)
  std::vector<Inst> hinst_x1[2], hinst_x2[2];  // [parity] buffer p -> X, X -> buffer p^1
  Inst* dinst_x1[2] = {nullptr, nullptr};
  Inst* dinst_x2[2] = {nullptr, nullptr};
  CUtensorMap* dtmap2[2] = {nullptr, nullptr};  // [parity][n] mu boxes of the two-step lean kernel
  uint8_t* dgen = nullptr;                      // [total_tiles] tile listed for the full kernel (blocked pairs)
  int4* dalist = nullptr;                       // [total_tiles] lean tiles next to the list (blocked pairs)
  cudaEvent_t ev_list = nullptr, ev_adj = nullptr;
  cudaStream_t side2 = nullptr;  // blocked pairs: the lean tiles next to the full kernel's list
  int grid_lean2 = 0, occ_lean2 = 0;
  int occ_lean_by[2] = {1, 1}, occ_lean2_by[2] = {1, 1};  // plain, compensated lean kernels
  int lose_box = 0;      // failure-detection test: the next lean launch loses one stage's boxes
  std::vector<gp_model> gm;
  std::vector<Inst> hinst[2];  // [buffer parity]
  Inst* dinst[2] = {nullptr, nullptr};
  Model* dmodel = nullptr;
  int noniso = 0;                 // some instance has the frozen temperature gradient
  gp_model* dgm = nullptr;        // [n] the instances' FP64 models (non-isothermal batches)
  long long* dtstep = nullptr;    // the step the next full-kernel pass computes
  LeanConst* dlconst = nullptr;                 // [n][N] lean-update constants of each phase
  CUtensorMap* dtmap[2] = {nullptr, nullptr};  // [parity][n] mu boxes of the lean kernel
  int* derr = nullptr;                          // lean kernel: a staged box did not arrive
  int total_tiles = 0;
  KernelSet ks;
  uint32_t* dflags = nullptr;  // [3][total_tiles] purity words of buffer 0, buffer 1 and X
  int* dtile_inst = nullptr;   // [total_tiles] instance of each tile
  int4* dtile_desc = nullptr;  // [total_tiles] {instance, x0, y0, tile_geo}
  std::vector<int4> htile_desc;
  int2* dglist = nullptr;      // [total_tiles] {tile, instance} of the full kernel's tiles
  int* dcnt = nullptr;         // [8] list count, queue head, finished blocks, ring-only count, adjacency count
  int grid_general = 0, grid_lean = 0;
  int occ_general = 0, occ_lean = 0;         // resident blocks per SM at full occupancy
  int step_threads = 256;                    // full-kernel block size: 256 or 512
  int scan = 0;                              // full-kernel blocks scan their own tiles (no list kernel)
  int occ_general_by[2] = {0, 0};            // occupancy of the 256- and 512-thread full kernels
  int lean_per_sm = 0, general_per_sm = 0;   // blocks per SM of the persistent grids (0: occupancy)
  int sms = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // per-kernel timing (off by default): a ring of event sets, one per step
  static constexpr int kTimingSlots = 64;
  int timing = 0, tn = 0, tdone = 0;
  std::vector<cudaEvent_t> tev;  // [kTimingSlots][kEv]: lean start/end, list start/end, general start/end
  static constexpr int kEv = 6;
  double tms[3] = {0, 0, 0};     // accumulated lean, list, general milliseconds
  int64_t tsteps = 0;
  int tslot_steps[kTimingSlots] = {};  // steps of each slot (negative: narrow band off, no lean/list events)
};

void gp_f32_batch_destroy(gp_f32_batch* b);

static void free_tiles(gp_f32_batch* b) {
  cudaFree(b->dflags);
  cudaFree(b->dtile_inst);
  cudaFree(b->dtile_desc);
  cudaFree(b->dglist);
  cudaFree(b->dgen);
  cudaFree(b->dalist);
  b->dalist = nullptr;
  b->dflags = nullptr;
  b->dtile_inst = nullptr;
  b->dtile_desc = nullptr;
  b->dglist = nullptr;
  b->dgen = nullptr;
}

cudaError_t gp_f32_batch_create(const gp_model* models, int n, gp_f32_batch** out) {
  if (n < 1) return cudaErrorInvalidValue;
  // one kernel set serves the batch: the anisotropic one when any instance is anisotropic (an
  // isotropic instance then runs it with dab = 0, where a_c = 1 and its derivative terms vanish)
  int aniso = 0;
  for (int i = 0; i < n; i++) {
    if (models[i].N != models[0].N || models[i].K1 != models[0].K1) return cudaErrorInvalidValue;
    aniso |= models[i].anisotropy ? 1 : 0;
  }
  KernelSet ks;
  if (!pick(models[0].N, models[0].K1, aniso, 16, 32, &ks)) return cudaErrorNotSupported;
  gp_f32_batch* b = new gp_f32_batch();
  b->n = n;
  b->N = models[0].N;
  b->K1 = models[0].K1;
  b->aniso = aniso;
  b->gm.assign(models, models + n);
  std::vector<Model> hm(n);
  for (int i = 0; i < n; i++) hm[i] = make_model(models[i]);
  std::vector<LeanConst> hl((size_t)n * b->N);
  for (int i = 0; i < n; i++)
    for (int a = 0; a < b->N; a++) {
      LeanConst& L = hl[(size_t)i * b->N + a];
      memset(&L, 0, sizeof L);
      for (int k = 0; k < MK; k++)
        for (int l = 0; l < MK; l++) {
          L.gx[k][l] = hm[i].Gx[a][k][l];
          L.gy[k][l] = hm[i].Gy[a][k][l];
        }
    }
  cudaError_t e = cudaMalloc(&b->dmodel, sizeof(Model) * n);
  if (e == cudaSuccess) e = cudaMemcpy(b->dmodel, hm.data(), sizeof(Model) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->dlconst, sizeof(LeanConst) * hl.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(b->dlconst, hl.data(), sizeof(LeanConst) * hl.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->derr, 2 * sizeof(int));  // error word, test token
  if (e == cudaSuccess) e = cudaMemset(b->derr, 0, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&b->dcnt, 8 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->dcnt, 0, 8 * sizeof(int));
  for (int i = 0; i < n; i++) b->noniso |= models[i].nonisothermal ? 1 : 0;
  if (e == cudaSuccess && b->noniso) {
    e = cudaMalloc(&b->dgm, sizeof(gp_model) * n);
    if (e == cudaSuccess) e = cudaMemcpy(b->dgm, models, sizeof(gp_model) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->dtstep, sizeof(long long));
    if (e == cudaSuccess) e = cudaMemset(b->dtstep, 0, sizeof(long long));
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_list, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_adj, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side2, cudaStreamNonBlocking);
  for (int p = 0; e == cudaSuccess && p < 2; p++) {
    b->hinst[p].resize(n);
    b->hinst_x1[p].resize(n);
    b->hinst_x2[p].resize(n);
    e = cudaMalloc(&b->dinst[p], sizeof(Inst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->dinst_x1[p], sizeof(Inst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->dinst_x2[p], sizeof(Inst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->dtmap[p], sizeof(CUtensorMap) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->dtmap2[p], sizeof(CUtensorMap) * n);
  }
  if (e != cudaSuccess) {
    gp_f32_batch_destroy(b);
    return e;
  }
  *out = b;
  return cudaSuccess;
}

void gp_f32_batch_destroy(gp_f32_batch* b) {
  if (!b) return;
  if (b->side) cudaStreamSynchronize(b->side);
  cudaFree(b->dmodel);
  for (int p = 0; p < 2; p++) {
    cudaFree(b->dinst[p]);
    cudaFree(b->dinst_x1[p]);
    cudaFree(b->dinst_x2[p]);
    cudaFree(b->dtmap[p]);
    cudaFree(b->dtmap2[p]);
  }
  cudaFree(b->dlconst);
  cudaFree(b->dgm);
  cudaFree(b->dtstep);
  cudaFree(b->derr);
  free_tiles(b);
  cudaFree(b->dcnt);
  for (cudaEvent_t ev : b->tev) cudaEventDestroy(ev);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->ev_list) cudaEventDestroy(b->ev_list);
  if (b->ev_adj) cudaEventDestroy(b->ev_adj);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->side2) {
    cudaStreamSynchronize(b->side2);
    cudaStreamDestroy(b->side2);
  }
  delete b;
}

// Bind the two state buffers of instance i (parity 0 reads buffer A, writes B).
void gp_f32_batch_bind(gp_f32_batch* b, int i, float* phiA, float* muA, float* phiB, float* muB, int pitch,
                       int64_t plane) {
  for (int p = 0; p < 2; p++) {
    Inst& I = b->hinst[p][i];
    I.phi = p ? phiB : phiA;
    I.mu = p ? muB : muA;
    I.phi_out = p ? phiA : phiB;
    I.mu_out = p ? muA : muB;
    I.plane = plane;
    I.pitch = pitch;
    I.mx = (int)b->gm[i].mesh_x;
    I.my = (int)b->gm[i].mesh_y;
    I.model = i;
    I.bc = gp_bc_of(b->gm[i]);
    I.gm = b->gm[i].nonisothermal ? b->dgm + i : nullptr;
    I.tstep = b->dtstep;
  }
}

// Bind the intermediate buffers X of instance i (step t+1 of a blocked pair:
// the full kernel's first pass writes it, its second pass reads it).
void gp_f32_batch_bind_x(gp_f32_batch* b, int i, float* phiX, float* muX) {
  for (int p = 0; p < 2; p++) {
    Inst& A = b->hinst_x1[p][i];
    A = b->hinst[p][i];
    A.phi_out = phiX;
    A.mu_out = muX;
    Inst& B = b->hinst_x2[p][i];
    B = b->hinst[p][i];
    B.phi = phiX;
    B.mu = muX;
  }
  b->has_x = 1;
}

// The purity flags describe the buffers' contents; after the state changes
// behind the kernels' back (upload, restore) they are reset to "unknown".
cudaError_t gp_f32_batch_invalidate(gp_f32_batch* b, cudaStream_t s) {
  if (!b->dflags) return cudaSuccess;
  return cudaMemsetAsync(b->dflags, 0, 3 * sizeof(uint32_t) * (size_t)b->total_tiles, s);
}

void gp_f32_batch_set_narrowband(gp_f32_batch* b, int on) { b->narrowband = on ? 1 : 0; }

// cuTensorMapEncodeTiled, from the driver (the runtime does not wrap it).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)f;
  }
  return fn;
}

// The lean kernel's mu box of every instance read at parity p: a 3-D tensor
// (columns, rows, planes) over the instance's input mu, box (TY + 8) x (TX + 2)
// x K1 starting at (y0 - 4, x0 - 1, 0); cells outside the grid read as zero.
// halo = 1: the single-step lean kernel's box (TX + 2 rows); halo = 2: the
// two-step one's (TX + 4 rows from x0 - 2).
static cudaError_t encode_boxes(gp_f32_batch* b, int p, int halo = 1) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  std::vector<CUtensorMap> maps(b->n);
  for (int i = 0; i < b->n; i++) {
    const Inst& I = b->hinst[p][i];
    const cuuint64_t dim[3] = {(cuuint64_t)I.my, (cuuint64_t)I.mx, (cuuint64_t)b->K1};
    const cuuint64_t stride[2] = {(cuuint64_t)I.pitch * 4, (cuuint64_t)I.plane * 4};
    const cuuint32_t box[3] = {(cuuint32_t)(halo == 2 ? lean2_stride(b->tx, b->ty) : b->ty + 8),
                               (cuuint32_t)b->tx + 2 * halo, (cuuint32_t)b->K1};
    const cuuint32_t estride[3] = {1, 1, 1};
    if (enc(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)I.mu, dim, stride, box, estride,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
  }
  return cudaMemcpy(halo == 2 ? b->dtmap2[p] : b->dtmap[p], maps.data(), sizeof(CUtensorMap) * b->n,
                    cudaMemcpyHostToDevice);
}

// Persistent grid sizes: blocks per SM as set (clamped to the occupancy), else the occupancy.
// Fewer lean blocks than fit leave room on every SM for full-kernel blocks to run beside them.
static void set_grids(gp_f32_batch* b) {
  const int l = b->lean_per_sm > 0 && b->lean_per_sm < b->occ_lean ? b->lean_per_sm : b->occ_lean;
  const int l2 = b->lean_per_sm > 0 && b->lean_per_sm < b->occ_lean2 ? b->lean_per_sm : b->occ_lean2;
  const int g = b->general_per_sm > 0 && b->general_per_sm < b->occ_general ? b->general_per_sm : b->occ_general;
  b->grid_lean = b->sms * l;
  b->grid_lean2 = b->sms * l2;
  b->grid_general = b->sms * g;
}

void gp_f32_batch_set_grids(gp_f32_batch* b, int lean_per_sm, int general_per_sm) {
  b->lean_per_sm = lean_per_sm;
  b->general_per_sm = general_per_sm;
  if (b->sms) set_grids(b);
}

// Full-kernel block size (256, or 512 where the 512-thread kernel exists); false if unavailable.
bool gp_f32_batch_set_step_threads(gp_f32_batch* b, int threads) {
  if (threads != 256 && !(threads == 512 && b->ks.general_wide)) return false;
  b->step_threads = threads;
  if (b->sms) {
    b->occ_general = b->occ_general_by[threads == 512];
    set_grids(b);
  }
  return true;
}

int gp_f32_batch_step_threads(const gp_f32_batch* b) { return b->step_threads; }
void gp_f32_batch_set_scan(gp_f32_batch* b, int on) { b->scan = on ? 1 : 0; }
int gp_f32_batch_scan(const gp_f32_batch* b) { return b->scan; }
bool gp_f32_batch_has_wide_step(const gp_f32_batch* b) { return b->ks.general_wide != nullptr; }

void gp_f32_batch_get_grids(const gp_f32_batch* b, int* lean_per_sm, int* general_per_sm, int* occ_lean,
                            int* occ_general) {
  const bool two = b->depth == 2;
  *lean_per_sm = b->sms ? (two ? b->grid_lean2 : b->grid_lean) / b->sms : 0;
  *general_per_sm = b->sms ? b->grid_general / b->sms : 0;
  *occ_lean = two ? b->occ_lean2 : b->occ_lean;
  *occ_general = b->occ_general;
}

// Steps per blocked launch: 1, or 2 (needs the intermediate buffers X and the
// list way of finding the interface tiles).  False if unavailable.
// Compensated accumulation on or off: the comp word of every instance's Model (read by the
// full kernel; synchronous copies: the caller has drained the batch's streams) and the lean
// kernels' template variant (the caller drops graphs captured with the other one).
cudaError_t gp_f32_batch_set_compensated(gp_f32_batch* b, int on) {
  const int v = on ? 1 : 0;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < b->n && e == cudaSuccess; i++)
    e = cudaMemcpy(reinterpret_cast<char*>(b->dmodel + i) + offsetof(Model, comp), &v, sizeof v,
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    b->comp = v;
    b->occ_lean = b->occ_lean_by[v];
    b->occ_lean2 = b->occ_lean2_by[v];
    if (b->sms) set_grids(b);
  }
  return e;
}
int gp_f32_batch_compensated(const gp_f32_batch* b) { return b->comp; }

bool gp_f32_batch_set_depth(gp_f32_batch* b, int depth) {
  if (depth != 1 && !(depth == 2 && b->has_x)) return false;
  b->depth = depth;
  return true;
}
int gp_f32_batch_depth(const gp_f32_batch* b) { return b->depth; }

// Recompute the tile decomposition for shape (tx, ty) and upload the instance tables.
cudaError_t gp_f32_batch_set_tiles(gp_f32_batch* b, int tx, int ty) {
  KernelSet ks;
  if (!pick(b->N, b->K1, b->aniso, tx, ty, &ks)) return cudaErrorInvalidValue;
  b->tx = tx;
  b->ty = ty;
  if (b->noniso) ks.smem_general += ks.smem_temp;
  b->ks = ks;
  int t = 0;
  std::vector<int> tile_inst;
  b->htile_desc.clear();
  for (int i = 0; i < b->n; i++) {
    const int txs = (int)((b->gm[i].mesh_x + tx - 1) / tx), tys = (int)((b->gm[i].mesh_y + ty - 1) / ty);
    for (int p = 0; p < 2; p++) {
      b->hinst[p][i].tiles_x = txs;
      b->hinst[p][i].tiles_y = tys;
      b->hinst[p][i].tile_begin = t;
    }
    for (int k = 0; k < txs * tys; k++)
      b->htile_desc.push_back(make_int4(i, (k / tys) * tx, (k % tys) * ty, (int)tile_geo(b->hinst[0][i], t + k, tx, ty)));
    t += txs * tys;
    tile_inst.insert(tile_inst.end(), (size_t)txs * tys, i);
  }
  b->total_tiles = t;
  for (int p = 0; p < 2; p++) {
    for (int i = 0; i < b->n; i++) {  // the X tables carry the tile decomposition too
      for (Inst* x : {&b->hinst_x1[p][i], &b->hinst_x2[p][i]}) {
        x->tiles_x = b->hinst[p][i].tiles_x;
        x->tiles_y = b->hinst[p][i].tiles_y;
        x->tile_begin = b->hinst[p][i].tile_begin;
      }
    }
    cudaError_t e = cudaMemcpy(b->dinst[p], b->hinst[p].data(), sizeof(Inst) * b->n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b->has_x)
      e = cudaMemcpy(b->dinst_x1[p], b->hinst_x1[p].data(), sizeof(Inst) * b->n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b->has_x)
      e = cudaMemcpy(b->dinst_x2[p], b->hinst_x2[p].data(), sizeof(Inst) * b->n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = encode_boxes(b, p);
    if (e == cudaSuccess) e = encode_boxes(b, p, 2);
    if (e != cudaSuccess) return e;
  }
  free_tiles(b);
  cudaError_t e = cudaMalloc(&b->dflags, 3 * sizeof(uint32_t) * (size_t)t);
  if (e == cudaSuccess) e = cudaMemset(b->dflags, 0, 3 * sizeof(uint32_t) * (size_t)t);
  if (e == cudaSuccess) e = cudaMalloc(&b->dgen, (size_t)t);
  if (e == cudaSuccess) e = cudaMemset(b->dgen, 0, (size_t)t);
  if (e == cudaSuccess) e = cudaMalloc(&b->dalist, sizeof(int4) * (size_t)t);
  if (e == cudaSuccess) e = cudaMalloc(&b->dtile_inst, sizeof(int) * t);
  if (e == cudaSuccess) e = cudaMalloc(&b->dglist, sizeof(int2) * t);
  if (e == cudaSuccess) e = cudaMalloc(&b->dtile_desc, sizeof(int4) * t);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->dtile_desc, b->htile_desc.data(), sizeof(int4) * t, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->dtile_inst, tile_inst.data(), sizeof(int) * t, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  // dynamic shared memory limits and persistent grid sizes
  int dev = 0, sms = 0, occ_g = 0, occ_l = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // one shared-memory carve-out for the three kernels of a step: no L1/shared reconfiguration
  // between them, and lean and full blocks can share an SM
  for (const void* f : {(const void*)ks.general, (const void*)ks.lean, (const void*)ks.lean2, (const void*)ks.list}) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(ks.general, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.smem_general);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_g, ks.general, 256, ks.smem_general);
  int occ_w = 0;
  if (e == cudaSuccess && ks.general_wide) {
    e = cudaFuncSetAttribute(ks.general_wide, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ks.general_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.smem_general);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_w, ks.general_wide, 512, ks.smem_general);
  }
  int occ_l2 = 0;
  for (int c = 0; c < 2 && e == cudaSuccess; c++) {
    const void* fl = c ? (const void*)ks.lean_c : (const void*)ks.lean;
    const void* fl2 = c ? (const void*)ks.lean2_c : (const void*)ks.lean2;
    int ol = 0, ol2 = 0;
    if (c) e = cudaFuncSetAttribute(fl, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (c && e == cudaSuccess)
      e = cudaFuncSetAttribute(fl2, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.smem_lean);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ol, fl, 32 * GP_LEAN_WARPS, ks.smem_lean);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(fl2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ks.smem_lean2);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ol2, fl2, 32 * 4, ks.smem_lean2);
    b->occ_lean_by[c] = ol > 0 ? ol : 1;
    b->occ_lean2_by[c] = ol2 > 0 ? ol2 : 1;
  }
  if (e != cudaSuccess) return e;
  occ_l = b->occ_lean_by[b->comp];
  occ_l2 = b->occ_lean2_by[b->comp];
  b->occ_lean2 = occ_l2 > 0 ? occ_l2 : 1;
  b->sms = sms;
  b->occ_general_by[0] = occ_g > 0 ? occ_g : 1;
  b->occ_general_by[1] = occ_w > 0 ? occ_w : 1;
  if (!ks.general_wide) b->step_threads = 256;
  b->occ_general = b->occ_general_by[b->step_threads == 512];
  b->occ_lean = occ_l > 0 ? occ_l : 1;
  set_grids(b);
  return cudaDeviceSynchronize();  // the flag reset above must land before any stream uses them
}

int gp_f32_batch_tiles(const gp_f32_batch* b) { return b->total_tiles; }

// Fold the event times of timing slot `slot` into the totals.
// Slot layout: [0] lean start, [1] lean end, [2] list start, [3] list end,
// [4] full start, [5] full end, [6] steps the slot covers (as an event count is
// not an event, the step count of each slot is kept in tslot_steps).
static cudaError_t timing_collect(gp_f32_batch* b, int slot) {
  cudaEvent_t* E = &b->tev[gp_f32_batch::kEv * slot];
  cudaError_t e = cudaEventSynchronize(E[5]);
  if (e == cudaSuccess) e = cudaEventSynchronize(E[1]);
  if (e != cudaSuccess) return e;
  float lean = 0.f, list = 0.f, gen = 0.f;
  const int st = b->tslot_steps[slot];
  if (st > 0) {  // narrow band on
    cudaEventElapsedTime(&lean, E[0], E[1]);
    cudaEventElapsedTime(&list, E[2], E[3]);
  }
  cudaEventElapsedTime(&gen, E[4], E[5]);
  b->tms[0] += lean;
  b->tms[1] += list;
  b->tms[2] += gen;
  b->tsteps += st > 0 ? st : -st;
  return cudaSuccess;
}

// Per-kernel timing: while on, every step records events around its kernels.
cudaError_t gp_f32_batch_set_timing(gp_f32_batch* b, int on) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  if (on && b->tev.empty()) {
    b->tev.resize(gp_f32_batch::kEv * gp_f32_batch::kTimingSlots);
    for (cudaEvent_t& ev : b->tev)
      if ((e = cudaEventCreate(&ev)) != cudaSuccess) return e;
  }
  b->timing = on ? 1 : 0;
  b->tn = b->tdone = 0;
  b->tms[0] = b->tms[1] = b->tms[2] = 0.0;
  b->tsteps = 0;
  return cudaSuccess;
}

// Mean milliseconds per step of the lean kernel, the list kernel and the full
// kernel over the steps timed since timing was switched on.
cudaError_t gp_f32_batch_kernel_ms(gp_f32_batch* b, double* ms, int64_t* steps) {
  for (; b->tdone < b->tn; b->tdone++) {
    cudaError_t e = timing_collect(b, b->tdone % gp_f32_batch::kTimingSlots);
    if (e != cudaSuccess) return e;
  }
  for (int i = 0; i < 3; i++) ms[i] = b->tsteps ? b->tms[i] / (double)b->tsteps : 0.0;
  *steps = b->tsteps;
  return cudaSuccess;
}

// The timing slot of the next launch (nullptr when timing is off).
static cudaError_t timing_slot(gp_f32_batch* b, int steps, cudaEvent_t** E) {
  *E = nullptr;
  if (!b->timing) return cudaSuccess;
  if (b->tn - b->tdone == gp_f32_batch::kTimingSlots) {  // ring full: fold the oldest slot first
    cudaError_t e = timing_collect(b, b->tdone % gp_f32_batch::kTimingSlots);
    if (e != cudaSuccess) return e;
    b->tdone++;
  }
  const int slot = b->tn++ % gp_f32_batch::kTimingSlots;
  b->tslot_steps[slot] = steps;
  *E = &b->tev[gp_f32_batch::kEv * slot];
  return cudaSuccess;
}

// The full kernel launched right after the tile list on the same stream, as its programmatic
// dependent: its blocks are scheduled while the list kernel runs and wait in the kernel
// (griddepcontrol.wait) for the list, instead of the launch waiting for the list to finish.
template <typename Fn, typename... Args>
static cudaError_t launch_after_list(Fn fn, int grid, int threads, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fn, args...);
}

// One step of every instance, reading buffer parity `parity`.
cudaError_t gp_f32_batch_launch(gp_f32_batch* b, int parity, cudaStream_t s) {
  const KernelSet& k = b->ks;
  const int p = parity & 1;
  const uint32_t* flags_in = b->dflags + (size_t)p * b->total_tiles;
  uint32_t* flags_out = b->dflags + (size_t)(p ^ 1) * b->total_tiles;
  cudaEvent_t* E = nullptr;
  cudaError_t e;
  if ((e = timing_slot(b, b->narrowband ? 1 : -1, &E)) != cudaSuccess) return e;
  if (!b->narrowband) {
    b->lose_box = 0;  // no lean kernel, no staged boxes to lose
    if (E && ((e = cudaEventRecord(E[4], s)) != cudaSuccess)) return e;
    (b->step_threads == 512 ? k.general_wide : k.general)<<<b->total_tiles, b->step_threads, k.smem_general, s>>>(
        b->dinst[p], b->dmodel, b->dtile_inst, nullptr, nullptr, flags_out, b->total_tiles, nullptr, nullptr, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (b->noniso) {
      k_tick<<<1, 1, 0, s>>>(b->dtstep);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (E) {
      if ((e = cudaEventRecord(E[5], s)) != cudaSuccess) return e;
      if ((e = cudaEventRecord(E[1], s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  // the lean tiles (side stream) and the rest run concurrently: disjoint tiles and words;
  // timed steps run them one after the other on `s` so that each kernel's events bracket it alone
  cudaStream_t ls = E ? s : b->side;
  if (!E) {
    if ((e = cudaEventRecord(b->ev_fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(b->side, b->ev_fork, 0)) != cudaSuccess) return e;
  }
  if (E && ((e = cudaEventRecord(E[0], ls)) != cudaSuccess)) return e;
  if (b->lose_box)  // failure-detection test: a nonzero token, taken by one warp
    if ((e = cudaMemsetAsync(b->derr + 1, 1, sizeof(int), ls)) != cudaSuccess) return e;
  (b->comp ? k.lean_c : k.lean)<<<b->grid_lean, 32 * GP_LEAN_WARPS, k.smem_lean, ls>>>(b->dinst[p], b->dlconst, b->dtmap[p], b->dtile_desc, flags_in,
                                                 flags_out, b->total_tiles, p, b->lose_box, b->derr);
  b->lose_box = 0;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (E && ((e = cudaEventRecord(E[1], ls)) != cudaSuccess)) return e;
  if (E && ((e = cudaEventRecord(E[2], s)) != cudaSuccess)) return e;
  if (!b->scan) {
    k.list<<<(b->total_tiles + 255) / 256, 256, 0, s>>>(b->dtile_desc, flags_in, b->total_tiles, b->dglist,
                                                        b->dcnt, nullptr, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (E && ((e = cudaEventRecord(E[3], s)) != cudaSuccess)) return e;
  if (E && ((e = cudaEventRecord(E[4], s)) != cudaSuccess)) return e;
  auto full = b->step_threads == 512 ? k.general_wide : k.general;
  if (b->scan || E)  // no list kernel before it, or timed launches (events between the two)
    full<<<b->grid_general, b->step_threads, k.smem_general, s>>>(
        b->dinst[p], b->dmodel, b->dtile_inst, b->scan ? nullptr : b->dglist, b->scan ? nullptr : b->dcnt, flags_out,
        b->total_tiles, b->scan ? b->dtile_desc : nullptr, b->scan ? flags_in : nullptr, 0);
  else
    e = launch_after_list(full, b->grid_general, b->step_threads, k.smem_general, s, (const Inst*)b->dinst[p],
                          (const Model*)b->dmodel, (const int*)b->dtile_inst, (const int2*)b->dglist, b->dcnt,
                          flags_out, b->total_tiles, (const int4*)nullptr, (const uint32_t*)nullptr, 0);
  if (e != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) return e;
  if (b->noniso) {
    k_tick<<<1, 1, 0, s>>>(b->dtstep);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (E) return cudaEventRecord(E[5], s);
  if ((e = cudaEventRecord(b->ev_join, b->side)) != cudaSuccess) return e;
  return cudaStreamWaitEvent(s, b->ev_join, 0);
}

// Two steps of every instance (a blocked pair), reading buffer parity `parity`
// and writing parity^1; X holds step t+1 of the tiles that need it.
//   stream s:    list (tiles for the full kernel, gen bytes)  -> full pass 1 (buffer p -> X)
//                -> [lean tiles next to the list done] -> full pass 2 (X -> buffer p^1)
//   second side stream: [list done] -> list of the lean tiles next to the list -> two-step lean
//                kernel on them (also writing their step t+1 into X)
//   side stream: [list done] -> two-step lean kernel on the other lean tiles
// Timed launches run one after the other on s.
cudaError_t gp_f32_batch_launch_pair(gp_f32_batch* b, int parity, cudaStream_t s) {
  if (b->depth != 2 || !b->narrowband || !b->has_x) return cudaErrorInvalidValue;
  const KernelSet& k = b->ks;
  const int p = parity & 1;
  const size_t T = (size_t)b->total_tiles;
  const uint32_t* flags_in = b->dflags + p * T;
  uint32_t* flags_out = b->dflags + (p ^ 1) * T;
  uint32_t* flags_x = b->dflags + 2 * T;
  cudaEvent_t* E = nullptr;
  cudaError_t e;
  if ((e = timing_slot(b, 2, &E)) != cudaSuccess) return e;
  b->lose_box = 0;
  auto full = b->step_threads == 512 ? k.general_wide : k.general;
  if (E && (e = cudaEventRecord(E[2], s)) != cudaSuccess) return e;
  k.list<<<(b->total_tiles + 255) / 256, 256, 0, s>>>(b->dtile_desc, flags_in, b->total_tiles, b->dglist, b->dcnt,
                                                      b->dgen, 2);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (E && (e = cudaEventRecord(E[3], s)) != cudaSuccess) return e;
  cudaStream_t ls = E ? s : b->side, as = E ? s : b->side2;
  if (!E) {
    if ((e = cudaEventRecord(b->ev_list, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(b->side, b->ev_list, 0)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(b->side2, b->ev_list, 0)) != cudaSuccess) return e;
  }
  if (E && (e = cudaEventRecord(E[0], ls)) != cudaSuccess) return e;
  k_adj_list<<<(b->total_tiles + 255) / 256, 256, 0, as>>>(b->dtile_desc, flags_in, b->dgen, b->total_tiles,
                                                           b->dalist, b->dcnt);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  for (int adj = 1; adj >= 0; adj--) {
    (b->comp ? k.lean2_c : k.lean2)<<<b->grid_lean2, 128, k.smem_lean2, adj ? as : ls>>>(
        b->dinst[p], b->dinst_x1[p], b->dlconst, b->dtmap2[p], b->dtile_desc, flags_in, flags_out, flags_x, b->dgen,
        b->total_tiles, p, adj ? b->dalist : nullptr, adj ? b->dcnt + 4 : nullptr, b->derr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (adj && !E && (e = cudaEventRecord(b->ev_adj, as)) != cudaSuccess) return e;
  }
  if (E && (e = cudaEventRecord(E[1], ls)) != cudaSuccess) return e;
  if (E && (e = cudaEventRecord(E[4], s)) != cudaSuccess) return e;
  if (E)
    full<<<b->grid_general, b->step_threads, k.smem_general, s>>>(b->dinst_x1[p], b->dmodel, b->dtile_inst,
                                                                   b->dglist, b->dcnt, flags_x, b->total_tiles,
                                                                   nullptr, nullptr, 1);
  else
    e = launch_after_list(full, b->grid_general, b->step_threads, k.smem_general, s, (const Inst*)b->dinst_x1[p],
                          (const Model*)b->dmodel, (const int*)b->dtile_inst, (const int2*)b->dglist, b->dcnt,
                          flags_x, b->total_tiles, (const int4*)nullptr, (const uint32_t*)nullptr, 1);
  if (e != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) return e;
  if (b->noniso) {
    k_tick<<<1, 1, 0, s>>>(b->dtstep);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (!E && (e = cudaStreamWaitEvent(s, b->ev_adj, 0)) != cudaSuccess) return e;
  full<<<b->grid_general, b->step_threads, k.smem_general, s>>>(b->dinst_x2[p], b->dmodel, b->dtile_inst, b->dglist,
                                                                 b->dcnt, flags_out, b->total_tiles, nullptr, nullptr, 0);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (b->noniso) {
    k_tick<<<1, 1, 0, s>>>(b->dtstep);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (E) return cudaEventRecord(E[5], s);
  if ((e = cudaEventRecord(b->ev_join, b->side)) != cudaSuccess) return e;
  return cudaStreamWaitEvent(s, b->ev_join, 0);
}

int gp_f32_batch_timing(const gp_f32_batch* b) { return b->timing; }

// Tiles the next step (reading buffer parity `parity`) sends to the lean
// kernel: lean_phase evaluated on the host over a copy of the purity words
// (with depth 2, the tiles the two-step lean kernel takes).
cudaError_t gp_f32_batch_lean_tiles(gp_f32_batch* b, int parity, cudaStream_t s, int64_t* lean,
                                    int64_t* lean_cells) {
  std::vector<uint32_t> F(b->total_tiles);
  cudaError_t e = cudaMemcpyAsync(F.data(), b->dflags + (size_t)(parity & 1) * b->total_tiles,
                                  sizeof(uint32_t) * F.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  int64_t n = 0, c = 0;
  for (int i = 0; i < b->n && b->narrowband; i++) {
    const Inst& I = b->hinst[parity & 1][i];
    for (int t = I.tile_begin; t < I.tile_begin + I.tiles_x * I.tiles_y; t++)
      if (lean_phase(F.data(), (uint32_t)b->htile_desc[t].w, t) >= 0 &&
          !(b->depth == 2 && ((uint32_t)b->htile_desc[t].w & TG_REJECT2))) {
        const int lt = t - I.tile_begin, x0 = (lt / I.tiles_y) * b->tx, y0 = (lt % I.tiles_y) * b->ty;
        n++;
        c += (int64_t)(I.mx - x0 < b->tx ? I.mx - x0 : b->tx) * (I.my - y0 < b->ty ? I.my - y0 : b->ty);
      }
  }
  *lean = n;
  *lean_cells = c;
  return cudaSuccess;
}

// Failure-detection test: the next lean-kernel launch leaves one staged box
// unissued, so that its bounded wait expires and the error word is set.
void gp_f32_batch_test_lose_box(gp_f32_batch* b) { b->lose_box = 1; }

// device word set by a lean kernel whose staged box did not arrive (0 = none)
const int* gp_f32_batch_error_word(const gp_f32_batch* b) { return b->derr; }

// kernel launches one gp_f32_batch_launch issues
int gp_f32_batch_launches_per_step(const gp_f32_batch* b) {
  return (b->narrowband ? (b->scan ? 2 : 3) : 1) + (b->noniso ? 1 : 0);
}
// kernel launches one gp_f32_batch_launch_pair issues (two steps)
int gp_f32_batch_launches_per_pair(const gp_f32_batch* b) { return 6 + (b->noniso ? 2 : 0); }

// The step count of the frozen temperature gradient (non-isothermal batches): the step the next
// full-kernel pass computes.  Stream-ordered on s.
cudaError_t gp_f32_batch_set_tstep(gp_f32_batch* b, long long t, cudaStream_t s) {
  if (!b->dtstep) return cudaSuccess;
  static thread_local long long v;
  v = t;
  cudaError_t e = cudaMemcpyAsync(b->dtstep, &v, sizeof v, cudaMemcpyHostToDevice, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
