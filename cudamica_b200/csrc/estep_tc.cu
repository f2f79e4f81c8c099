// tcgen05 (TF32 tensor-core) form of the fused AMICA E-step: placeholder
// until the tensor-core kernel lands; reports every shape as unsupported so
// contexts fall back to the plain FP32 kernel.
#include "common.cuh"

namespace amica {

int tc_supported(int, int, int) { return 0; }
int tc_max_clusters(int, int, int) { return -1; }
int tc_tile_samples() { return 128; }
cudaError_t launch_estep_tc(const EStepArgs&, int, int, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace amica
