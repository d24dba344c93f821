// gen_f32.cu -- FP32 instantiations of the generator passes (all variants).
#include "gen_launch.cuh"

namespace scarl {
cudaError_t run_pass_f32(int pass, int v, const GenArgs& a, cudaStream_t s) {
  return run_pass<float>(pass, v, a, s);
}
}  // namespace scarl
