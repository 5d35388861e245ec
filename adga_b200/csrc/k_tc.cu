// Tensor-core (tcgen05) trailing update of the mixed-precision LU.
// Placeholder until the BF16x3 kernel lands: reports "not available" so the
// mixed path uses the CUDA-core FP32 update.
#include "lu.cuh"

int tc_available() { return 0; }
cudaError_t tc_trail_setup(void **ctx, z32 *, const LUBatch &, cudaStream_t) {
  *ctx = nullptr;
  return cudaErrorNotSupported;
}
cudaError_t tc_trail_run(void *, int, int, cudaStream_t) { return cudaErrorNotSupported; }
void tc_trail_free(void *) {}
