// gp_f32.cu -- placeholder until the FP32 chosen form lands.
#include "gp_common.cuh"

int gp_f32_supported(const gp_model& m) {
  (void)m;
  return 0;
}

cudaError_t gp_f32_step(const gp_model& m, int pitch, int64_t plane, const float* phi, const float* mu,
                        float* phi_out, float* mu_out, cudaStream_t s, int* launches) {
  (void)m; (void)pitch; (void)plane; (void)phi; (void)mu; (void)phi_out; (void)mu_out; (void)s;
  *launches = 0;
  return cudaErrorNotSupported;
}
