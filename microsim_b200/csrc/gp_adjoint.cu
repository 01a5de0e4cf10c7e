// gp_adjoint.cu -- hand-written adjoint of the explicit step (binary alloys:
// 2 phases, one independent chemical potential) with sqrt(N) checkpointing.
//
// Forward: the step of gp_adjoint_cell.cuh (the plain step's model) in the
// working precision T (float: the chosen form; double: the reference
// adjoint), two kernels per step like the plain form: Delta-phi on the
// interior plus one ghost ring, then the mu/phi update.  Every
// `every`-th state is kept (checkpoints).
//
// Reverse of one step n (state x_n, adjoint lambda_{n+1} of x_{n+1}):
//   1. recompute Delta-phi of x_n on the ring;
//   2. per interior cell: reverse of its mu/phi update -> its own adjoints
//      and the adjoints of its flux divergences (gdf, gdj);
//   3. per face: reverse of the diffusion flux and the antitrapping current
//      (adjoint = difference of the two cells' gdf, gdj), scattered by atomic
//      adds into phi, mu and Delta-phi of the cells it reads;
//   4. per ring cell with a nonzero Delta-phi adjoint: reverse of Delta-phi,
//      scattered into its 3x3 phi stencil and its mu.
// Ghost reads are boundary index maps, so their adjoints land on the mapped
// interior cells.  Parameter gradients are reduced per block in FP64.
// Backward: segments of `every` steps, last first: the segment is recomputed
// from its checkpoint into a buffer of `every` states, then reversed.
// Memory: ceil(N / every) + every states (every = ceil(sqrt(N)) by default).

#include <math.h>
#include <string.h>

#include <vector>

#include "gp_common.cuh"
#include "gp_adjoint_cell.cuh"

extern "C" void gp_set_error(const char* fmt, ...);

namespace {

using namespace gpadj;

struct Geo {
  int mx, my, pitch, rpitch;
  int64_t plane, rplane;  // elements per state plane / Delta-phi ring plane
  gp_bc bc;
};

// state layout: planes phi_0, phi_1, mu, each [mx][pitch]
template <typename T>
__device__ __forceinline__ T ld_phi(const T* st, const Geo& g, int x, int y, int a) {
  return st[a * g.plane + (int64_t)gp_map(x, g.mx, g.bc.phi_x) * g.pitch + gp_map(y, g.my, g.bc.phi_y)];
}
template <typename T>
__device__ __forceinline__ T ld_mu(const T* st, const Geo& g, int x, int y) {
  return st[2 * g.plane + (int64_t)gp_map(x, g.mx, g.bc.mu_x) * g.pitch + gp_map(y, g.my, g.bc.mu_y)];
}
__device__ __forceinline__ int64_t ix_phi(const Geo& g, int x, int y, int a) {
  return a * g.plane + (int64_t)gp_map(x, g.mx, g.bc.phi_x) * g.pitch + gp_map(y, g.my, g.bc.phi_y);
}
__device__ __forceinline__ int64_t ix_mu(const Geo& g, int x, int y) {
  return 2 * g.plane + (int64_t)gp_map(x, g.mx, g.bc.mu_x) * g.pitch + gp_map(y, g.my, g.bc.mu_y);
}
// Delta-phi ring: cells x in [-1, mx], y in [-1, my]
__device__ __forceinline__ int64_t ix_ring(const Geo& g, int x, int y, int a) {
  return a * g.rplane + (int64_t)(x + 1) * g.rpitch + (y + 1);
}

template <typename T>
__device__ __forceinline__ void load_P(const T* st, const Geo& g, int x, int y, T (&P)[3][3][2]) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int a = 0; a < 2; a++) P[i][j][a] = ld_phi(st, g, x + i - 1, y + j - 1, a);
}

// Face k of interior cell (x, y): 0 = x+, 1 = x-, 2 = y+, 3 = y-; M[5], D[5]:
// mu and Delta-phi (phase 0) of the cell and its x-, x+, y-, y+ neighbours.
template <typename T>
__device__ __forceinline__ Face<T> cell_face(const AM<T>& m, const Geo& g, int y, const T (&P)[3][3][2],
                                             const T (&M)[5], const T (&D)[5], int k) {
  Face<T> f;
  const T ty = (T)2 * m.dy;
  auto cy = [&](int i, int a) { return (P[i][2][a] - P[i][0][a]) / ty; };
  auto cx = [&](int j, int a) {
    return (T)0.5 * ((P[2][j][a] - P[1][j][a]) / m.dx + (P[1][j][a] - P[0][j][a]) / m.dx);
  };
  for (int a = 0; a < 2; a++) {
    if (k == 0) {
      f.pc[a] = P[1][1][a]; f.pn[a] = P[2][1][a]; f.tc[a] = cy(1, a); f.tn[a] = cy(2, a);
    } else if (k == 1) {
      f.pc[a] = P[0][1][a]; f.pn[a] = P[1][1][a]; f.tc[a] = cy(0, a); f.tn[a] = cy(1, a);
    } else if (k == 2) {
      f.pc[a] = P[1][1][a]; f.pn[a] = P[1][2][a]; f.tc[a] = cx(1, a); f.tn[a] = cx(2, a);
    } else {
      f.pc[a] = P[1][0][a]; f.pn[a] = P[1][1][a]; f.tc[a] = cx(0, a); f.tn[a] = cx(1, a);
    }
  }
  // neighbour slots: 0 centre, 1 x-, 2 x+, 3 y-, 4 y+
  const int cs = k == 1 ? 1 : (k == 3 ? 3 : 0), ns = k == 0 ? 2 : (k == 2 ? 4 : 0);
  f.muc = M[cs]; f.mun = M[ns];
  f.dpc = D[cs]; f.dpn = D[ns];
  f.h = (k >> 1) ? m.dy : m.dx;
  const int ylow = k == 3 ? y - 1 : y;  // the face's lower cell
  f.skip = (k >> 1) && (ylow + 3 == g.my - 2);
  return f;
}

template <typename T>
__device__ __forceinline__ void load_MD(const T* st, const T* ring, const Geo& g, int x, int y, T (&M)[5],
                                        T (&D)[5], T (&Dc)[2]) {
  const int dx[5] = {0, -1, 1, 0, 0}, dy[5] = {0, 0, 0, -1, 1};
#pragma unroll
  for (int s = 0; s < 5; s++) {
    M[s] = ld_mu(st, g, x + dx[s], y + dy[s]);
    D[s] = ring[ix_ring(g, x + dx[s], y + dy[s], 0)];
  }
  Dc[0] = D[0];
  Dc[1] = ring[ix_ring(g, x, y, 1)];
}

// ------------------------------------------------------------------ forward

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_dphi(const AM<T> m, Geo g, const T* __restrict__ st,
                                                  T* __restrict__ ring) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x - 1, x = blockIdx.y - 1;
  if (y > g.my) return;
  T P[3][3][2], dp[2];
  load_P(st, g, x, y, P);
  dphi_fwd(m, P, ld_mu(st, g, x, y), dp);
  ring[ix_ring(g, x, y, 0)] = dp[0];
  ring[ix_ring(g, x, y, 1)] = dp[1];
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_update(const AM<T> m, Geo g, const T* __restrict__ st,
                                                    const T* __restrict__ ring, T* __restrict__ out) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  T P[3][3][2], M[5], D[5], Dc[2], F[4], J[4];
  load_P(st, g, x, y, P);
  load_MD(st, ring, g, x, y, M, D, Dc);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const Face<T> f = cell_face(m, g, y, P, M, D, k);
    F[k] = fface(m, f);
    J[k] = jface(m, f);
  }
  const T ph[2] = {P[1][1][0], P[1][1][1]};
  const int64_t o = (int64_t)x * g.pitch + y;
  out[2 * g.plane + o] = mu_new(m, ph, M[0], Dc, F, J);
  out[o] = ph[0] + Dc[0];
  out[g.plane + o] = ph[1] + Dc[1];
}

// ------------------------------------------------------------------ reverse

// block sum of the four parameter adjoints into grad (FP64)
__device__ __forceinline__ void reduce_params(double (&lp)[NPARAM], double* grad) {
  __shared__ double s[NPARAM][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int p = 0; p < NPARAM; p++) {
    double v = lp[p];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s[p][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NPARAM) {
    double v = 0.0;
    for (int i = 0; i < nw; i++) v += s[threadIdx.x][i];
    if (v != 0.0) atomicAdd(grad + threadIdx.x, v);
  }
}

// 2. reverse of the cell update: lam_out (phi, mu of the cell) is written,
// ldphi (ring, zeroed before) receives the cell's own Delta-phi adjoint
template <typename T>
__global__ void __launch_bounds__(256) k_rev_cell(const AM<T> m, Geo g, const T* __restrict__ st,
                                                  const T* __restrict__ ring, const T* __restrict__ lam_in,
                                                  T* __restrict__ lam_out, T* __restrict__ ldphi,
                                                  T* __restrict__ gdf, T* __restrict__ gdj) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
  if (y >= g.my) return;
  const int64_t o = (int64_t)x * g.pitch + y;
  T P[3][3][2], M[5], D[5], Dc[2], F[4], J[4];
  load_P(st, g, x, y, P);
  load_MD(st, ring, g, x, y, M, D, Dc);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const Face<T> f = cell_face(m, g, y, P, M, D, k);
    F[k] = fface(m, f);
    J[k] = jface(m, f);
  }
  const T ph[2] = {P[1][1][0], P[1][1][1]};
  const T lp0 = lam_in[o], lp1 = lam_in[g.plane + o], lmn = lam_in[2 * g.plane + o];
  T lph[2] = {lp0, lp1}, lmu = (T)0, ldp[2] = {lp0, lp1}, df = (T)0, dj = (T)0;
  mu_new_rev(m, ph, M[0], Dc, F, J, lmn, lph, lmu, ldp, df, dj);
  lam_out[o] = lph[0];
  lam_out[g.plane + o] = lph[1];
  lam_out[2 * g.plane + o] = lmu;
  ldphi[ix_ring(g, x, y, 0)] += ldp[0];
  ldphi[ix_ring(g, x, y, 1)] += ldp[1];
  gdf[o] = df;
  gdj[o] = dj;
}

// Scatter of one adjoint contribution; a zero one is skipped (most faces of a bulk region carry no
// antitrapping current, so most of their tangential and Delta-phi adjoints are zero).  The float
// sums are order-dependent anyway (atomics); skipping a +-0 addend changes at most a zero's sign.
template <typename T>
__device__ __forceinline__ void add_nz(T* p, T v) {
  if (v != (T)0) atomicAdd(p, v);
}

// 3. reverse of the face fluxes; thread = one face (lower cell (x, y)):
// x-faces for x in [-1, mx-1], y in [0, my-1]; y-faces for x in [0, mx-1], y in [-1, my-1]
template <typename T>
__global__ void __launch_bounds__(256) k_rev_face(const AM<T> m, Geo g, const T* __restrict__ st,
                                                  const T* __restrict__ ring, const T* __restrict__ gdf,
                                                  const T* __restrict__ gdj, T* __restrict__ lam_out,
                                                  T* __restrict__ ldphi, double* __restrict__ grad) {
  double lpd[NPARAM] = {0, 0, 0, 0};
  const int dir = blockIdx.z;  // 0: x-faces, 1: y-faces
  const int x = blockIdx.y - (dir == 0 ? 1 : 0);
  const int y = blockIdx.x * blockDim.x + threadIdx.x - (dir == 1 ? 1 : 0);
  const bool valid = dir == 0 ? (y < g.my && x <= g.mx - 1) : (y <= g.my - 1 && x < g.mx);
  if (valid) {
    const int xn = dir == 0 ? x + 1 : x, yn = dir == 0 ? y : y + 1;
    const bool cin = x >= 0 && y >= 0, nin = xn < g.mx && yn < g.my;
    const T h = dir == 0 ? m.dx : m.dy;
    const T lF = ((cin ? gdf[(int64_t)x * g.pitch + y] : (T)0) - (nin ? gdf[(int64_t)xn * g.pitch + yn] : (T)0)) / h;
    const T lJ = ((cin ? gdj[(int64_t)x * g.pitch + y] : (T)0) - (nin ? gdj[(int64_t)xn * g.pitch + yn] : (T)0)) *
                 m.jscale / h;
    // the face's operands, as the cells build them
    Face<T> f;
    const T ty = (T)2 * m.dy;
    for (int a = 0; a < 2; a++) {
      f.pc[a] = ld_phi(st, g, x, y, a);
      f.pn[a] = ld_phi(st, g, xn, yn, a);
      if (dir == 0) {
        f.tc[a] = (ld_phi(st, g, x, y + 1, a) - ld_phi(st, g, x, y - 1, a)) / ty;
        f.tn[a] = (ld_phi(st, g, xn, y + 1, a) - ld_phi(st, g, xn, y - 1, a)) / ty;
      } else {
        const T c0 = ld_phi(st, g, x, y, a), n0 = ld_phi(st, g, x, yn, a);
        f.tc[a] = (T)0.5 * ((ld_phi(st, g, x + 1, y, a) - c0) / m.dx + (c0 - ld_phi(st, g, x - 1, y, a)) / m.dx);
        f.tn[a] = (T)0.5 * ((ld_phi(st, g, x + 1, yn, a) - n0) / m.dx + (n0 - ld_phi(st, g, x - 1, yn, a)) / m.dx);
      }
    }
    f.muc = ld_mu(st, g, x, y);
    f.mun = ld_mu(st, g, xn, yn);
    f.dpc = ring[ix_ring(g, x, y, 0)];
    f.dpn = ring[ix_ring(g, xn, yn, 0)];
    f.h = h;
    f.skip = dir == 1 && (y + 3 == g.my - 2);
    FaceAdj<T> L = {};
    T lp[NPARAM] = {(T)0, (T)0, (T)0, (T)0};
    if (lF != (T)0) fface_rev(m, f, lF, L, lp);
    if (lJ != (T)0) jface_rev(m, f, lJ, L, lp);
    for (int p = 0; p < NPARAM; p++) lpd[p] = (double)lp[p];
    for (int a = 0; a < 2; a++) {
      add_nz(lam_out + ix_phi(g, x, y, a), L.pc[a]);
      add_nz(lam_out + ix_phi(g, xn, yn, a), L.pn[a]);
      if (dir == 0) {
        add_nz(lam_out + ix_phi(g, x, y + 1, a), L.tc[a] / ty);
        add_nz(lam_out + ix_phi(g, x, y - 1, a), -L.tc[a] / ty);
        add_nz(lam_out + ix_phi(g, xn, y + 1, a), L.tn[a] / ty);
        add_nz(lam_out + ix_phi(g, xn, y - 1, a), -L.tn[a] / ty);
      } else {
        const T hc = (T)0.5 * L.tc[a] / m.dx, hn = (T)0.5 * L.tn[a] / m.dx;
        add_nz(lam_out + ix_phi(g, x + 1, y, a), hc);
        add_nz(lam_out + ix_phi(g, x - 1, y, a), -hc);
        add_nz(lam_out + ix_phi(g, x + 1, yn, a), hn);
        add_nz(lam_out + ix_phi(g, x - 1, yn, a), -hn);
      }
    }
    add_nz(lam_out + ix_mu(g, x, y), L.muc);
    add_nz(lam_out + ix_mu(g, xn, yn), L.mun);
    add_nz(ldphi + ix_ring(g, x, y, 0), L.dpc);
    add_nz(ldphi + ix_ring(g, xn, yn, 0), L.dpn);
  }
  reduce_params(lpd, grad);
}

// 4. reverse of Delta-phi on the ring
template <typename T>
__global__ void __launch_bounds__(256) k_rev_dphi(const AM<T> m, Geo g, const T* __restrict__ st,
                                                  const T* __restrict__ ldphi, T* __restrict__ lam_out,
                                                  double* __restrict__ grad) {
  double lpd[NPARAM] = {0, 0, 0, 0};
  const int y = blockIdx.x * blockDim.x + threadIdx.x - 1, x = blockIdx.y - 1;
  if (y <= g.my) {
    const T ld[2] = {ldphi[ix_ring(g, x, y, 0)], ldphi[ix_ring(g, x, y, 1)]};
    if (ld[0] != (T)0 || ld[1] != (T)0) {
      T P[3][3][2], LP[3][3][2] = {}, lmu = (T)0, lp[NPARAM] = {(T)0, (T)0, (T)0, (T)0};
      load_P(st, g, x, y, P);
      dphi_rev(m, P, ld_mu(st, g, x, y), ld, LP, lmu, lp);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          for (int a = 0; a < 2; a++)
            if (LP[i][j][a] != (T)0) atomicAdd(lam_out + ix_phi(g, x + i - 1, y + j - 1, a), LP[i][j][a]);
      if (lmu != (T)0) atomicAdd(lam_out + ix_mu(g, x, y), lmu);
      for (int p = 0; p < NPARAM; p++) lpd[p] = (double)lp[p];
    }
  }
  reduce_params(lpd, grad);
}

// ------------------------------------------------------------------ host side

template <typename T>
AM<T> make_am(const gp_model& g) {
  AM<T> m;
  m.dx = (T)g.dx;
  m.dy = (T)g.dy;
  m.dt = (T)g.dt;
  m.eps = (T)g.epsilon;
  m.inv_eps = (T)g.inv_eps;
  m.mob = (T)(1.0 / g.tau_ab[0][1]);
  m.tau_ratio = (T)(g.tau / g.tau_ab[0][1]);
  m.gam = (T)g.Gamma[0][1];
  m.dab = g.anisotropy ? (T)g.dab[0][1] : (T)0;
  m.wobs = (T)g.w_obstacle;
  m.jscale = (T)(g.obstacle ? g.jat_obst : g.jat_well);
  m.swell = (T)g.s_well;
  for (int a = 0; a < 2; a++)
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        m.R[a][i][j] = g.anisotropy ? (T)g.R[a][1 - a][i][j] : (T)(i == j);
        m.Ri[a][i][j] = g.anisotropy ? (T)g.Rinv[a][1 - a][i][j] : (T)(i == j);
      }
  for (int a = 0; a < 2; a++) {
    m.cmu[a] = (T)g.cmu[a][0][0];
    m.A[a] = (T)g.A[a][0][0];
    m.B[a] = (T)g.B[a][0];
    m.C[a] = (T)g.C[a];
    m.Beff[a] = (T)g.Beff[a][0];
  }
  m.Ds = (T)g.Diff[0][0][0];
  m.Dl = (T)g.Diff[1][0][0];
  m.obstacle = g.obstacle ? 1 : 0;
  m.skip_row = (int)g.mesh_y - 5;
  return m;
}

struct AdjBase {
  virtual ~AdjBase() {}
  virtual int forward(const double* phi0, const double* mu0, int64_t nsteps, int64_t every, double* phi_out,
                      double* mu_out) = 0;
  virtual int backward(const double* lphi, const double* lmu, double* grad, double* lphi0, double* lmu0) = 0;
  int64_t stored = 0;
};

#define ADJ_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      gp_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));  \
      return GP_E_CUDA;                                                                 \
    }                                                                                   \
  } while (0)

template <typename T>
struct Adj : AdjBase {
  gp_model gm;
  AM<T> m;
  Geo g;
  cudaStream_t s = nullptr;
  T *ckpt = nullptr, *seg = nullptr, *cur = nullptr, *nxt = nullptr, *ring = nullptr;
  T *lam[2] = {nullptr, nullptr}, *ldphi = nullptr, *gdf = nullptr, *gdj = nullptr;
  double* dgrad = nullptr;
  int64_t nsteps = 0, every = 0, nck = 0;
  bool have = false;

  int64_t state() const { return 3 * g.plane; }

  ~Adj() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(ckpt);
    cudaFree(seg);
    cudaFree(cur);
    cudaFree(nxt);
    cudaFree(ring);
    cudaFree(lam[0]);
    cudaFree(lam[1]);
    cudaFree(ldphi);
    cudaFree(gdf);
    cudaFree(gdj);
    cudaFree(dgrad);
    if (s) cudaStreamDestroy(s);
  }

  int init(const gp_model& model) {
    gm = model;
    m = make_am<T>(model);
    g.mx = (int)model.mesh_x;
    g.my = (int)model.mesh_y;
    g.pitch = (int)gp_round_up(g.my, 32);
    g.plane = (int64_t)g.pitch * g.mx;
    g.rpitch = (int)gp_round_up(g.my + 2, 32);
    g.rplane = (int64_t)g.rpitch * (g.mx + 2);
    g.bc = gp_bc_of(model);
    ADJ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    ADJ_CUDA(cudaMalloc(&cur, sizeof(T) * state()));
    ADJ_CUDA(cudaMalloc(&nxt, sizeof(T) * state()));
    ADJ_CUDA(cudaMalloc(&ring, sizeof(T) * 2 * g.rplane));
    ADJ_CUDA(cudaMalloc(&lam[0], sizeof(T) * state()));
    ADJ_CUDA(cudaMalloc(&lam[1], sizeof(T) * state()));
    ADJ_CUDA(cudaMalloc(&ldphi, sizeof(T) * 2 * g.rplane));
    ADJ_CUDA(cudaMalloc(&gdf, sizeof(T) * g.plane));
    ADJ_CUDA(cudaMalloc(&gdj, sizeof(T) * g.plane));
    ADJ_CUDA(cudaMalloc(&dgrad, sizeof(double) * NPARAM));
    ADJ_CUDA(cudaMemsetAsync(cur, 0, sizeof(T) * state(), s));
    ADJ_CUDA(cudaMemsetAsync(nxt, 0, sizeof(T) * state(), s));
    return GP_OK;
  }

  cudaError_t step(const T* in, T* out) {
    const dim3 b(256), gr((g.my + 2 + 255) / 256, g.mx + 2), gu((g.my + 255) / 256, g.mx);
    k_fwd_dphi<T><<<gr, b, 0, s>>>(m, g, in, ring);
    k_fwd_update<T><<<gu, b, 0, s>>>(m, g, in, ring, out);
    return cudaGetLastError();
  }

  // lam_in = adjoint of the state after x, lam_out = adjoint of x
  cudaError_t rev_step(const T* x, const T* lin, T* lout) {
    const dim3 b(256), gr((g.my + 2 + 255) / 256, g.mx + 2), gu((g.my + 255) / 256, g.mx);
    k_fwd_dphi<T><<<gr, b, 0, s>>>(m, g, x, ring);
    cudaError_t e = cudaMemsetAsync(ldphi, 0, sizeof(T) * 2 * g.rplane, s);
    if (e != cudaSuccess) return e;
    k_rev_cell<T><<<gu, b, 0, s>>>(m, g, x, ring, lin, lout, ldphi, gdf, gdj);
    const dim3 gf((g.my + 1 + 255) / 256, g.mx + 1, 2);
    k_rev_face<T><<<gf, b, 0, s>>>(m, g, x, ring, gdf, gdj, lout, ldphi, dgrad);
    k_rev_dphi<T><<<gr, b, 0, s>>>(m, g, x, ldphi, lout, dgrad);
    return cudaGetLastError();
  }

  // host [planes][mx][my] doubles <-> device [planes][mx][pitch] T
  int upload(T* dst, const double* phi, const double* mu) {
    std::vector<T> h(state(), (T)0);
    for (int a = 0; a < 3; a++) {
      const double* src = a < 2 ? (phi ? phi + (int64_t)a * g.mx * g.my : nullptr) : mu;
      if (!src) continue;
      for (int x = 0; x < g.mx; x++)
        for (int y = 0; y < g.my; y++) h[a * g.plane + (int64_t)x * g.pitch + y] = (T)src[(int64_t)x * g.my + y];
    }
    ADJ_CUDA(cudaMemcpyAsync(dst, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    ADJ_CUDA(cudaStreamSynchronize(s));
    return GP_OK;
  }
  int download(const T* src, double* phi, double* mu) {
    std::vector<T> h(state());
    ADJ_CUDA(cudaMemcpyAsync(h.data(), src, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, s));
    ADJ_CUDA(cudaStreamSynchronize(s));
    for (int a = 0; a < 3; a++) {
      double* dst = a < 2 ? (phi ? phi + (int64_t)a * g.mx * g.my : nullptr) : mu;
      if (!dst) continue;
      for (int x = 0; x < g.mx; x++)
        for (int y = 0; y < g.my; y++) dst[(int64_t)x * g.my + y] = (double)h[a * g.plane + (int64_t)x * g.pitch + y];
    }
    return GP_OK;
  }

  int forward(const double* phi0, const double* mu0, int64_t n, int64_t ev, double* phi_out,
              double* mu_out) override {
    if (n < 1 || !phi0 || !mu0) return GP_E_ARG;
    if (ev <= 0) ev = (int64_t)ceil(sqrt((double)n));
    if (ev > n) ev = n;
    const int64_t nc = (n + ev - 1) / ev;
    cudaFree(ckpt);
    cudaFree(seg);
    ckpt = seg = nullptr;
    have = false;
    if (cudaMalloc(&ckpt, sizeof(T) * state() * nc) != cudaSuccess ||
        cudaMalloc(&seg, sizeof(T) * state() * ev) != cudaSuccess) {
      cudaGetLastError();
      gp_set_error("adjoint: %lld checkpoints + %lld segment states do not fit", (long long)nc, (long long)ev);
      return GP_E_NOMEM;
    }
    nsteps = n;
    every = ev;
    nck = nc;
    stored = nc + ev;
    int rc = upload(cur, phi0, mu0);
    if (rc != GP_OK) return rc;
    for (int64_t i = 0; i < n; i++) {
      if (i % ev == 0)
        ADJ_CUDA(cudaMemcpyAsync(ckpt + (i / ev) * state(), cur, sizeof(T) * state(), cudaMemcpyDeviceToDevice, s));
      ADJ_CUDA(step(cur, nxt));
      T* t = cur;
      cur = nxt;
      nxt = t;
    }
    have = true;
    return download(cur, phi_out, mu_out);
  }

  int backward(const double* lphi, const double* lmu, double* grad, double* lphi0, double* lmu0) override {
    if (!have) {
      gp_set_error("adjoint: backward before forward");
      return GP_E_ARG;
    }
    if (!grad) return GP_E_ARG;
    int rc = upload(lam[0], lphi, lmu);
    if (rc != GP_OK) return rc;
    ADJ_CUDA(cudaMemsetAsync(dgrad, 0, sizeof(double) * NPARAM, s));
    int li = 0;
    for (int64_t k = nck - 1; k >= 0; k--) {
      const int64_t start = k * every, len = (nsteps - start < every) ? nsteps - start : every;
      ADJ_CUDA(cudaMemcpyAsync(seg, ckpt + k * state(), sizeof(T) * state(), cudaMemcpyDeviceToDevice, s));
      for (int64_t i = 1; i < len; i++) ADJ_CUDA(step(seg + (i - 1) * state(), seg + i * state()));
      for (int64_t i = len - 1; i >= 0; i--) {
        ADJ_CUDA(rev_step(seg + i * state(), lam[li], lam[li ^ 1]));
        li ^= 1;
      }
    }
    ADJ_CUDA(cudaMemcpyAsync(grad, dgrad, sizeof(double) * NPARAM, cudaMemcpyDeviceToHost, s));
    ADJ_CUDA(cudaStreamSynchronize(s));
    if (lphi0 || lmu0) return download(lam[li], lphi0, lmu0);
    return GP_OK;
  }
};

}  // namespace

struct gp_adj {
  AdjBase* impl;
};

extern "C" int gp_adj_create(const gp_model* m, int precision, gp_adj** out) {
  if (!m || !out) return GP_E_ARG;
  *out = nullptr;
  if (m->N != 2 || m->K1 != 1) {
    gp_set_error("adjoint: binary alloys only (N = 2, K-1 = 1), got N = %d, K-1 = %d", m->N, m->K1);
    return GP_E_UNSUPPORTED;
  }
  if (m->mesh_x < 4 || m->mesh_y < 4) return GP_E_ARG;
  if (m->nonisothermal) {
    gp_set_error("adjoint: isothermal models only");
    return GP_E_UNSUPPORTED;
  }
  gp_adj* a = new gp_adj();
  int rc;
  if (precision == GP_FP32) {
    Adj<float>* p = new Adj<float>();
    a->impl = p;
    rc = p->init(*m);
  } else {
    Adj<double>* p = new Adj<double>();
    a->impl = p;
    rc = p->init(*m);
  }
  if (rc != GP_OK) {
    delete a->impl;
    delete a;
    return rc;
  }
  *out = a;
  return GP_OK;
}

extern "C" int gp_adj_forward(gp_adj* a, const double* phi0, const double* mu0, int64_t nsteps,
                              int64_t checkpoint_every, double* phi_out, double* mu_out) {
  if (!a) return GP_E_ARG;
  return a->impl->forward(phi0, mu0, nsteps, checkpoint_every, phi_out, mu_out);
}

extern "C" int gp_adj_backward(gp_adj* a, const double* lam_phi, const double* lam_mu, double* grad,
                               double* lam_phi0, double* lam_mu0) {
  if (!a) return GP_E_ARG;
  return a->impl->backward(lam_phi, lam_mu, grad, lam_phi0, lam_mu0);
}

extern "C" int gp_adj_stored_states(const gp_adj* a, int64_t* states) {
  if (!a || !states) return GP_E_ARG;
  *states = a->impl->stored;
  return GP_OK;
}

extern "C" int gp_adj_destroy(gp_adj* a) {
  if (!a) return GP_OK;
  delete a->impl;
  delete a;
  return GP_OK;
}
