// gp_noalloc.cu -- one plain (FP64) step for callers that cannot allocate
// device memory.
//
// Who needs it: host codes that hand us device buffers they already own and
// that are not allowed to call cudaMalloc themselves or through us -- for
// example a solver embedded in a framework whose memory pool owns the whole
// device (every allocation must go through that pool), or a code whose device
// memory budget is fixed at start-up.  The regular entry points (gp_create /
// gp_step) allocate the state buffers and the Delta-phi ring array the step
// needs between its two kernels.  This entry point takes the state buffers
// from the caller and keeps the ring array in a file-scope device array of
// fixed size, so a call allocates nothing.
//
// Facts a caller must know:
//  * The scratch array is GP_NOALLOC_SCRATCH_BYTES (8 MiB) per GPU.  It is
//    reserved on every GPU that loads this library and held until the process
//    exits.  A grid needs N * (mesh_x + 2) * round_up(mesh_y + 2, 32) doubles of
//    it; larger grids are rejected with GP_E_SIZE before anything is launched.
//  * Every call on a device shares that one array and it keeps the contents of
//    the last call.  Nothing in it has to start at zero: the first kernel writes
//    every ring cell the second kernel reads.  Calls whose kernels overlap on
//    the GPU (different streams without ordering) race on the array.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make that
//    first call before any stream capture.
//  * The device is this library's current device, the one gp_set_device chose
//    (device 0 unless it was called): the library carries its own CUDA
//    runtime, so the host program's own device choice does not reach it.  The
//    four buffers and the stream must belong to that device; a call with any of
//    them elsewhere is rejected with GP_E_ARG, as is an output whose bytes
//    overlap an input or the other output.
//  * Host code cannot use the array's name as a device address: the symbol
//    seen by host code is a host-side stand-in.  Only the address returned by
//    cudaGetSymbolAddress is passed to the kernels.

#include <stdint.h>

#include <mutex>

#include "gp_common.cuh"

extern "C" void gp_set_error(const char* fmt, ...);

cudaError_t gp_f64_step(const gp_model& m, int pitch, int64_t plane, int rpitch, int64_t rplane,
                        const double* phi, const double* mu, double* dphi, double* phi_out, double* mu_out,
                        cudaStream_t s, bool smooth = false, const double* ghost_rows = nullptr,
                        const gp_temp_step* temp = nullptr);

static __device__ __align__(256) double g_noalloc_dphi[GP_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_lock;
double* g_scratch[kMaxDevices];  // device address of g_noalloc_dphi, per device
}  // namespace

extern "C" int gp_step_f64_noalloc(const gp_model* m, const double* phi, const double* mu, double* phi_out,
                                   double* mu_out, int64_t pitch, void* stream) {
  if (!m || !phi || !mu || !phi_out || !mu_out) {
    gp_set_error("gp_step_f64_noalloc: NULL argument");
    return GP_E_ARG;
  }
  if (phi == phi_out || mu == mu_out) {
    gp_set_error("gp_step_f64_noalloc: input and output buffers must differ (the step reads neighbours of "
                 "the old state while it writes the new one)");
    return GP_E_ARG;
  }
  if (m->N < 2 || m->N > GP_MAX_PHASES || m->K1 < 1 || m->K1 > GP_MAX_K1 || m->mesh_x < 4 || m->mesh_y < 4 ||
      pitch < m->mesh_y || pitch > (int64_t)1 << 30 || m->mesh_x > (1 << 20)) {
    gp_set_error("gp_step_f64_noalloc: N=%d K1=%d mesh %lld x %lld pitch %lld outside the supported ranges", m->N,
                 m->K1, (long long)m->mesh_x, (long long)m->mesh_y, (long long)pitch);
    return GP_E_ARG;
  }
  for (int i = 0; i < 4; i++) {
    const int a = m->bc_phi[i], b = m->bc_mu[i];
    if ((a != GP_BC_NEUMANN && a != GP_BC_PERIODIC) || (b != GP_BC_NEUMANN && b != GP_BC_PERIODIC)) {
      gp_set_error("gp_step_f64_noalloc: boundary types must be Neumann (1) or periodic (3)");
      return GP_E_UNSUPPORTED;
    }
  }
  if (m->nonisothermal) {
    gp_set_error("gp_step_f64_noalloc: a non-isothermal model needs the step count (gp_create/gp_step)");
    return GP_E_UNSUPPORTED;
  }
  if (m->bc_phi[0] != m->bc_phi[1] || m->bc_phi[2] != m->bc_phi[3] || m->bc_mu[0] != m->bc_mu[1] ||
      m->bc_mu[2] != m->bc_mu[3] || (m->mu_solver == GP_MU_TERNARY && m->K1 != 2)) {
    gp_set_error("gp_step_f64_noalloc: inconsistent boundary pairs or solver");
    return GP_E_UNSUPPORTED;
  }
  const int64_t rpitch = gp_round_up(m->mesh_y + 2, 32);
  const int64_t rplane = (m->mesh_x + 2) * rpitch;
  const int64_t need = (int64_t)m->N * rplane * (int64_t)sizeof(double);
  if (need > (int64_t)GP_NOALLOC_SCRATCH_BYTES) {
    gp_set_error("gp_step_f64_noalloc: the grid needs %lld bytes of scratch, more than the fixed %lld "
                 "(N * (mesh_x+2) * round_up(mesh_y+2, 32) doubles); use gp_create/gp_step",
                 (long long)need, (long long)GP_NOALLOC_SCRATCH_BYTES);
    return GP_E_SIZE;
  }
  // The step reads neighbours of the old state while it writes the new one, so no byte of an
  // output may lie inside an input (or the other output): compare the byte ranges the call touches.
  {
    const int64_t plane = m->mesh_x * pitch, row_end = (m->mesh_x - 1) * pitch + m->mesh_y;
    const uintptr_t lo[4] = {(uintptr_t)phi, (uintptr_t)mu, (uintptr_t)phi_out, (uintptr_t)mu_out};
    const int64_t n[4] = {(m->N - 1) * plane + row_end, (m->K1 - 1) * plane + row_end,
                          (m->N - 1) * plane + row_end, (m->K1 - 1) * plane + row_end};
    for (int o = 2; o < 4; o++)
      for (int i = 0; i < o; i++) {
        const uintptr_t a0 = lo[i], a1 = lo[i] + (uintptr_t)n[i] * sizeof(double);
        const uintptr_t b0 = lo[o], b1 = lo[o] + (uintptr_t)n[o] * sizeof(double);
        if (a0 < b1 && b0 < a1) {
          gp_set_error("gp_step_f64_noalloc: output %s overlaps %s (the step reads neighbours of the old state "
                       "while it writes the new one)", o == 2 ? "phi_out" : "mu_out",
                       i == 0 ? "phi" : i == 1 ? "mu" : "phi_out");
          return GP_E_ARG;
        }
      }
  }
  // This library carries its own CUDA runtime: its current device is the one gp_set_device chose
  // (device 0 by default), not the host program's.  The buffers and the stream must live there,
  // or the kernels would run on another GPU's scratch array and stream.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    gp_set_error("gp_step_f64_noalloc: no usable current device (%s)", cudaGetErrorString(e));
    return GP_E_CUDA;
  }
  {
    const void* bufs[4] = {phi, mu, phi_out, mu_out};
    const char* names[4] = {"phi", "mu", "phi_out", "mu_out"};
    for (int i = 0; i < 4; i++) {
      cudaPointerAttributes at;
      e = cudaPointerGetAttributes(&at, bufs[i]);
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        gp_set_error("gp_step_f64_noalloc: %s is not a pointer CUDA knows (%s)", names[i], cudaGetErrorString(e));
        return GP_E_ARG;
      }
      if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != dev) {
        gp_set_error("gp_step_f64_noalloc: %s is not device memory of the library's current device %d "
                     "(select the buffers' GPU with gp_set_device)", names[i], dev);
        return GP_E_ARG;
      }
    }
    if (stream) {
      int sdev = -1;
      e = cudaStreamGetDevice((cudaStream_t)stream, &sdev);
      if (e != cudaSuccess || sdev != dev) {
        (void)cudaGetLastError();
        gp_set_error("gp_step_f64_noalloc: the stream belongs to device %d, not the library's current device %d "
                     "(select it with gp_set_device)", sdev, dev);
        return GP_E_ARG;
      }
    }
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_scratch[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_dphi);
      if (e != cudaSuccess || !p) {
        gp_set_error("gp_step_f64_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                     cudaGetErrorString(e));
        return GP_E_CUDA;
      }
      g_scratch[dev] = (double*)p;
    }
    scratch = g_scratch[dev];
  }
  e = gp_f64_step(*m, (int)pitch, m->mesh_x * pitch, (int)rpitch, rplane, phi, mu, scratch, phi_out, mu_out,
                  (cudaStream_t)stream);
  if (e != cudaSuccess) {
    gp_set_error("gp_step_f64_noalloc: launch failed: %s", cudaGetErrorString(e));
    return GP_E_CUDA;
  }
  return GP_OK;
}
