// gp_capi.cu -- the C ABI of include/gp_b200.h: device contexts, copies,
// the step loop and the FP64 statistics reduction.
//
// Reference entry points this replaces (Grand_potential_Finite_difference_2D_serial/):
//   solverloop_phasefield / apply_boundary_conditions / solverloop_concentration
//   called from microsim_gp.c:103-106, and the progress statistics of
//   microsim_gp.c:139-148 (global_max_min, updated in
//   calculate_divergence_concentration.h:272-296).

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "gp_common.cuh"

extern "C" void gp_set_error(const char* fmt, ...);

cudaError_t gp_f64_step(const gp_model& m, int pitch, int64_t plane, int rpitch, int64_t rplane, const double* phi,
                        const double* mu, double* dphi, double* phi_out, double* mu_out, cudaStream_t s);
cudaError_t gp_f32_step(const gp_model& m, int pitch, int64_t plane, const float* phi, const float* mu,
                        float* phi_out, float* mu_out, cudaStream_t s, int* launches);
int gp_f32_supported(const gp_model& m);

#define GP_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      gp_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));     \
      return GP_E_CUDA;                                                                    \
    }                                                                                      \
  } while (0)

struct gp_ctx {
  gp_model m;
  int precision;
  int device;
  cudaStream_t stream;
  int pitch;       // elements per x-row of a state plane
  int64_t plane;   // elements per plane
  int rpitch;      // Delta-phi ring array (FP64 form)
  int64_t rplane;
  size_t esize;    // bytes per element of the state
  void* phi[2];
  void* mu[2];
  double* dphi;    // FP64 form: Delta-phi of the last phase-field half step
  int cur;         // which buffer holds the current state
  int have_prev;   // buffer 1-cur holds the previous step's state
  double* partials;  // statistics: per-block partial results
  double* reduced;   // statistics: final values (device)
  int red_blocks;
  int64_t launches;
  // running extrema (microsim_gp.c prints running values since t = 0)
  double run_phi_max[GP_MAX_PHASES], run_phi_min[GP_MAX_PHASES];
  double run_mu_max[GP_MAX_K1], run_mu_min[GP_MAX_K1];
};

static int check_model(const gp_model* m) {
  if (!m) return GP_E_ARG;
  if (m->N < 2 || m->N > GP_MAX_PHASES || m->K1 < 1 || m->K1 > GP_MAX_K1) {
    gp_set_error("N=%d, K1=%d outside the supported 2..%d, 1..%d", m->N, m->K1, GP_MAX_PHASES, GP_MAX_K1);
    return GP_E_UNSUPPORTED;
  }
  if (m->mesh_x < 4 || m->mesh_y < 4 || m->mesh_x > (1 << 20) || m->mesh_y > (1 << 20)) {
    gp_set_error("mesh %lld x %lld outside 4..2^20", (long long)m->mesh_x, (long long)m->mesh_y);
    return GP_E_SIZE;
  }
  for (int i = 0; i < 4; i++) {
    int a = m->bc_phi[i], b = m->bc_mu[i];
    if ((a != GP_BC_NEUMANN && a != GP_BC_PERIODIC) || (b != GP_BC_NEUMANN && b != GP_BC_PERIODIC)) {
      gp_set_error("boundary types must be Neumann (1) or periodic (3)");
      return GP_E_UNSUPPORTED;
    }
  }
  if (m->bc_phi[0] != m->bc_phi[1] || m->bc_phi[2] != m->bc_phi[3] || m->bc_mu[0] != m->bc_mu[1] ||
      m->bc_mu[2] != m->bc_mu[3]) {
    gp_set_error("both sides of an axis must share a boundary type (the reference forces periodic pairs)");
    return GP_E_UNSUPPORTED;
  }
  if (m->mu_solver == GP_MU_TERNARY && m->K1 != 2) return GP_E_UNSUPPORTED;
  if (!(m->dt > 0) || !(m->dx > 0) || !(m->dy > 0) || !(m->epsilon > 0)) {
    gp_set_error("dt, dx, dy, epsilon must be positive");
    return GP_E_ARG;
  }
  return GP_OK;
}

extern "C" int gp_create(const gp_model* m, int precision, gp_ctx** out) {
  int rc = check_model(m);
  if (rc != GP_OK) return rc;
  if (!out) return GP_E_ARG;
  if (precision != GP_FP64 && precision != GP_FP32) return GP_E_ARG;
  if (precision == GP_FP32 && !gp_f32_supported(*m)) {
    gp_set_error("FP32 form not available for N=%d, K1=%d", m->N, m->K1);
    return GP_E_UNSUPPORTED;
  }
  gp_ctx* c = new (std::nothrow) gp_ctx();
  if (!c) return GP_E_NOMEM;
  memset(c, 0, sizeof *c);
  c->m = *m;
  c->precision = precision;
  cudaError_t e = cudaGetDevice(&c->device);
  if (e != cudaSuccess) {
    gp_set_error("no CUDA device: %s", cudaGetErrorString(e));
    delete c;
    return GP_E_CUDA;
  }
  c->esize = precision == GP_FP64 ? sizeof(double) : sizeof(float);
  c->pitch = (int)gp_round_up(m->mesh_y, 32);
  c->plane = (int64_t)m->mesh_x * c->pitch;
  c->rpitch = (int)gp_round_up(m->mesh_y + 2, 32);
  c->rplane = (int64_t)(m->mesh_x + 2) * c->rpitch;
  c->red_blocks = 296;
  for (int a = 0; a < GP_MAX_PHASES; a++) { c->run_phi_max[a] = 1.0; c->run_phi_min[a] = 0.0; }
  for (int k = 0; k < GP_MAX_K1; k++) { c->run_mu_max[k] = 1.0; c->run_mu_min[k] = 1.0; }
  size_t nphi = (size_t)m->N * c->plane * c->esize, nmu = (size_t)m->K1 * c->plane * c->esize;
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess;
  for (int i = 0; ok && i < 2; i++) {
    ok = cudaMalloc(&c->phi[i], nphi) == cudaSuccess && cudaMalloc(&c->mu[i], nmu) == cudaSuccess;
    if (ok) ok = cudaMemset(c->phi[i], 0, nphi) == cudaSuccess && cudaMemset(c->mu[i], 0, nmu) == cudaSuccess;
  }
  if (ok && precision == GP_FP64) {
    ok = cudaMalloc(&c->dphi, (size_t)m->N * c->rplane * sizeof(double)) == cudaSuccess &&
         cudaMemset(c->dphi, 0, (size_t)m->N * c->rplane * sizeof(double)) == cudaSuccess;
  }
  if (ok) ok = cudaMalloc(&c->partials, (size_t)c->red_blocks * 64 * sizeof(double)) == cudaSuccess &&
               cudaMalloc(&c->reduced, 64 * sizeof(double)) == cudaSuccess;
  if (!ok) {
    gp_set_error("device allocation failed: %s", cudaGetErrorString(cudaGetLastError()));
    gp_destroy(c);
    return GP_E_NOMEM;
  }
  *out = c;
  return GP_OK;
}

extern "C" int gp_destroy(gp_ctx* c) {
  if (!c) return GP_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int i = 0; i < 2; i++) {
    if (c->phi[i]) cudaFree(c->phi[i]);
    if (c->mu[i]) cudaFree(c->mu[i]);
  }
  if (c->dphi) cudaFree(c->dphi);
  if (c->partials) cudaFree(c->partials);
  if (c->reduced) cudaFree(c->reduced);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return GP_OK;
}

// dense host planes [n][mx][my] (double) -> pitched device planes
template <typename T>
__global__ void k_pack(const double* __restrict__ src, T* __restrict__ dst, int mx, int my, int pitch,
                       int64_t plane, int nplanes) {
  const int64_t n = (int64_t)mx * my * nplanes;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / ((int64_t)mx * my), r = i % ((int64_t)mx * my);
    const int x = (int)(r / my), y = (int)(r % my);
    dst[p * plane + (int64_t)x * pitch + y] = (T)src[i];
  }
}

template <typename T>
__global__ void k_unpack(const T* __restrict__ src, double* __restrict__ dst, int mx, int my, int pitch,
                         int64_t plane, int nplanes) {
  const int64_t n = (int64_t)mx * my * nplanes;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / ((int64_t)mx * my), r = i % ((int64_t)mx * my);
    const int x = (int)(r / my), y = (int)(r % my);
    dst[i] = (double)src[p * plane + (int64_t)x * pitch + y];
  }
}

static int copy_planes(gp_ctx* c, const double* host, void* dev, int nplanes, bool up) {
  const int64_t mx = c->m.mesh_x, my = c->m.mesh_y;
  if (c->precision == GP_FP64) {
    for (int p = 0; p < nplanes; p++) {
      double* d = (double*)dev + p * c->plane;
      const double* h = host + p * mx * my;
      if (up)
        GP_CUDA(cudaMemcpy2DAsync(d, c->pitch * sizeof(double), h, my * sizeof(double), my * sizeof(double), mx,
                                  cudaMemcpyHostToDevice, c->stream));
      else
        GP_CUDA(cudaMemcpy2DAsync((void*)h, my * sizeof(double), d, c->pitch * sizeof(double), my * sizeof(double),
                                  mx, cudaMemcpyDeviceToHost, c->stream));
    }
    return GP_OK;
  }
  // FP32: stage doubles on the device, convert with a kernel
  double* stage = nullptr;
  const size_t bytes = (size_t)nplanes * mx * my * sizeof(double);
  GP_CUDA(cudaMallocAsync((void**)&stage, bytes, c->stream));
  if (up) {
    GP_CUDA(cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, c->stream));
    k_pack<float><<<592, 256, 0, c->stream>>>(stage, (float*)dev, (int)mx, (int)my, c->pitch, c->plane, nplanes);
  } else {
    k_unpack<float><<<592, 256, 0, c->stream>>>((const float*)dev, stage, (int)mx, (int)my, c->pitch, c->plane,
                                                nplanes);
    GP_CUDA(cudaMemcpyAsync((void*)host, stage, bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  c->launches++;
  GP_CUDA(cudaGetLastError());
  GP_CUDA(cudaFreeAsync(stage, c->stream));
  return GP_OK;
}

extern "C" int gp_upload(gp_ctx* c, const double* phi, const double* mu) {
  if (!c || !phi || !mu) return GP_E_ARG;
  int rc = copy_planes(c, phi, c->phi[c->cur], c->m.N, true);
  if (rc == GP_OK) rc = copy_planes(c, mu, c->mu[c->cur], c->m.K1, true);
  if (rc == GP_OK) GP_CUDA(cudaStreamSynchronize(c->stream));
  c->have_prev = 0;
  return rc;
}

extern "C" int gp_download(gp_ctx* c, double* phi, double* mu) {
  if (!c || !phi || !mu) return GP_E_ARG;
  int rc = copy_planes(c, phi, c->phi[c->cur], c->m.N, false);
  if (rc == GP_OK) rc = copy_planes(c, mu, c->mu[c->cur], c->m.K1, false);
  if (rc == GP_OK) GP_CUDA(cudaStreamSynchronize(c->stream));
  return rc;
}

extern "C" int gp_download_dphi(gp_ctx* c, double* dphi) {
  if (!c || !dphi) return GP_E_ARG;
  if (c->precision != GP_FP64) return GP_E_UNSUPPORTED;
  const int64_t rx = c->m.mesh_x + 2, ry = c->m.mesh_y + 2;
  for (int a = 0; a < c->m.N; a++)
    GP_CUDA(cudaMemcpy2DAsync(dphi + a * rx * ry, ry * sizeof(double), c->dphi + a * c->rplane,
                              c->rpitch * sizeof(double), ry * sizeof(double), rx, cudaMemcpyDeviceToHost, c->stream));
  GP_CUDA(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

extern "C" int gp_step(gp_ctx* c, int64_t nsteps) {
  if (!c || nsteps < 0) return GP_E_ARG;
  for (int64_t t = 0; t < nsteps; t++) {
    const int nxt = 1 - c->cur;
    if (c->precision == GP_FP64) {
      GP_CUDA(gp_f64_step(c->m, c->pitch, c->plane, c->rpitch, c->rplane, (const double*)c->phi[c->cur],
                          (const double*)c->mu[c->cur], c->dphi, (double*)c->phi[nxt], (double*)c->mu[nxt],
                          c->stream));
      c->launches += 2;
    } else {
      int nl = 0;
      GP_CUDA(gp_f32_step(c->m, c->pitch, c->plane, (const float*)c->phi[c->cur], (const float*)c->mu[c->cur],
                          (float*)c->phi[nxt], (float*)c->mu[nxt], c->stream, &nl));
      c->launches += nl;
    }
    c->cur = nxt;
    c->have_prev = 1;
  }
  return GP_OK;
}

extern "C" int gp_sync(gp_ctx* c) {
  if (!c) return GP_E_ARG;
  GP_CUDA(cudaStreamSynchronize(c->stream));
  return GP_OK;
}

extern "C" size_t gp_model_sizeof(void) { return sizeof(gp_model); }

extern "C" void* gp_stream(gp_ctx* c) { return c ? (void*)c->stream : nullptr; }
extern "C" int64_t gp_launch_count(const gp_ctx* c) { return c ? c->launches : 0; }

// ------------------------------------------------------------------ statistics

// slots of the reduction vector
struct StatLayout {
  int N, K1;
  __host__ __device__ int phi_max(int a) const { return a; }
  __host__ __device__ int phi_min(int a) const { return N + a; }
  __host__ __device__ int rel_phi(int a) const { return 2 * N + a; }
  __host__ __device__ int phase(int a) const { return 3 * N + a; }
  __host__ __device__ int mu_max(int k) const { return 4 * N + k; }
  __host__ __device__ int mu_min(int k) const { return 4 * N + K1 + k; }
  __host__ __device__ int rel_mu(int k) const { return 4 * N + 2 * K1 + k; }
  __host__ __device__ int solute(int k) const { return 4 * N + 3 * K1 + k; }
  __host__ __device__ int nonfinite() const { return 4 * N + 4 * K1; }
  __host__ __device__ int count() const { return 4 * N + 4 * K1 + 1; }
  __host__ __device__ bool is_max(int s) const { return s < N || (s >= 4 * N && s < 4 * N + K1); }
  __host__ __device__ bool is_min(int s) const {
    return (s >= N && s < 2 * N) || (s >= 4 * N + K1 && s < 4 * N + 2 * K1);
  }
};

__device__ __forceinline__ double combine(const StatLayout& L, int s, double a, double b) {
  if (L.is_max(s)) return fmax(a, b);
  if (L.is_min(s)) return fmin(a, b);
  return a + b;
}

__device__ __forceinline__ double ident(const StatLayout& L, int s) {
  if (L.is_max(s)) return -1.0e308;
  if (L.is_min(s)) return 1.0e308;
  return 0.0;
}

// One pass over the interior: each block writes its partial vector.
// The solute integrand is sum_a c_a(mu) h_a(phi) (file_writer.h:203-235).
template <typename T>
__global__ void __launch_bounds__(256) k_stats(const __grid_constant__ gp_model m, const T* __restrict__ phi, const T* __restrict__ mu,
                                               const T* __restrict__ phi_prev, const T* __restrict__ mu_prev,
                                               int have_prev, int pitch, int64_t plane, double* __restrict__ partials) {
  const StatLayout L{m.N, m.K1};
  const int S = L.count();
  double acc[4 * GP_MAX_PHASES + 4 * GP_MAX_K1 + 1];
  for (int s = 0; s < S; s++) acc[s] = ident(L, s);
  const int64_t ncell = (int64_t)m.mesh_x * m.mesh_y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncell; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i / m.mesh_y), y = (int)(i % m.mesh_y);
    const int64_t o = (int64_t)x * pitch + y;
    double ph[GP_MAX_PHASES], mm[GP_MAX_K1];
    bool bad = false;
    for (int a = 0; a < m.N; a++) {
      ph[a] = (double)phi[o + a * plane];
      bad |= !isfinite(ph[a]);
      acc[L.phi_max(a)] = fmax(acc[L.phi_max(a)], ph[a]);
      acc[L.phi_min(a)] = fmin(acc[L.phi_min(a)], ph[a]);
      acc[L.phase(a)] += ph[a];
      if (have_prev) {
        const double d = ph[a] - (double)phi_prev[o + a * plane];
        acc[L.rel_phi(a)] += d * d;
      }
    }
    for (int k = 0; k < m.K1; k++) {
      mm[k] = (double)mu[o + k * plane];
      bad |= !isfinite(mm[k]);
      acc[L.mu_max(k)] = fmax(acc[L.mu_max(k)], mm[k]);
      acc[L.mu_min(k)] = fmin(acc[L.mu_min(k)], mm[k]);
      if (have_prev) {
        const double d = mm[k] - (double)mu_prev[o + k * plane];
        acc[L.rel_mu(k)] += d * d;
      }
    }
    for (int k = 0; k < m.K1; k++) {
      double comp = 0.0;
      for (int a = 0; a < m.N; a++) {
        double cm = 0.0;
        for (int l = 0; l < m.K1; l++) cm += m.cmu[a][k][l] * (mm[l] - m.Beff[a][l]);
        double h = 3.0 * ph[a] * ph[a] - 2.0 * ph[a] * ph[a] * ph[a], s1 = 0.0;
        for (int b = 0; b < m.N; b++)
          for (int c = b + 1; c < m.N; c++)
            if (b != a && c != a) s1 += ph[b] * ph[c];
        s1 *= 2.0 * ph[a];
        comp += cm * (h + s1);
      }
      acc[L.solute(k)] += comp;
    }
    if (bad) acc[L.nonfinite()] += 1.0;
  }
  __shared__ double red[8][4 * GP_MAX_PHASES + 4 * GP_MAX_K1 + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = 0; s < S; s++) {
    double v = acc[s];
    for (int off = 16; off > 0; off >>= 1) v = combine(L, s, v, __shfl_down_sync(0xffffffffu, v, off));
    if (lane == 0) red[warp][s] = v;
  }
  __syncthreads();
  if (threadIdx.x < S) {
    const int s = threadIdx.x;
    double v = red[0][s];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = combine(L, s, v, red[w][s]);
    partials[(int64_t)blockIdx.x * 64 + s] = v;
  }
}

// Fixed-order final combine of the block partials (deterministic).
__global__ void k_stats_final(int N, int K1, const double* __restrict__ partials, int nblocks,
                              double* __restrict__ out) {
  const StatLayout L{N, K1};
  const int s = threadIdx.x;
  if (s >= L.count()) return;
  double v = partials[s];
  for (int b = 1; b < nblocks; b++) v = combine(L, s, v, partials[(int64_t)b * 64 + s]);
  out[s] = v;
}

extern "C" int gp_get_stats(gp_ctx* c, gp_stats* out) {
  if (!c || !out) return GP_E_ARG;
  const gp_model& m = c->m;
  const int cur = c->cur, prv = 1 - c->cur;
  if (c->precision == GP_FP64)
    k_stats<double><<<c->red_blocks, 256, 0, c->stream>>>(m, (const double*)c->phi[cur], (const double*)c->mu[cur],
                                                         (const double*)c->phi[prv], (const double*)c->mu[prv],
                                                         c->have_prev, c->pitch, c->plane, c->partials);
  else
    k_stats<float><<<c->red_blocks, 256, 0, c->stream>>>(m, (const float*)c->phi[cur], (const float*)c->mu[cur],
                                                        (const float*)c->phi[prv], (const float*)c->mu[prv],
                                                        c->have_prev, c->pitch, c->plane, c->partials);
  GP_CUDA(cudaGetLastError());
  k_stats_final<<<1, 64, 0, c->stream>>>(m.N, m.K1, c->partials, c->red_blocks, c->reduced);
  GP_CUDA(cudaGetLastError());
  c->launches += 2;
  double v[64];
  GP_CUDA(cudaMemcpyAsync(v, c->reduced, sizeof v, cudaMemcpyDeviceToHost, c->stream));
  GP_CUDA(cudaStreamSynchronize(c->stream));
  const StatLayout L{m.N, m.K1};
  memset(out, 0, sizeof *out);
  for (int a = 0; a < m.N; a++) {
    if (v[L.phi_max(a)] > c->run_phi_max[a]) c->run_phi_max[a] = v[L.phi_max(a)];
    if (v[L.phi_min(a)] < c->run_phi_min[a]) c->run_phi_min[a] = v[L.phi_min(a)];
    out->phi_max[a] = c->run_phi_max[a];
    out->phi_min[a] = c->run_phi_min[a];
    out->rel_change_phi[a] = v[L.rel_phi(a)];
    out->phase_fraction[a] = v[L.phase(a)];
  }
  for (int k = 0; k < m.K1; k++) {
    if (v[L.mu_max(k)] > c->run_mu_max[k]) c->run_mu_max[k] = v[L.mu_max(k)];
    if (v[L.mu_min(k)] < c->run_mu_min[k]) c->run_mu_min[k] = v[L.mu_min(k)];
    out->mu_max[k] = c->run_mu_max[k];
    out->mu_min[k] = c->run_mu_min[k];
    out->rel_change_mu[k] = v[L.rel_mu(k)];
    out->solute[k] = v[L.solute(k)];
  }
  out->nonfinite = (int64_t)v[L.nonfinite()];
  return out->nonfinite ? GP_E_NONFINITE : GP_OK;
}
