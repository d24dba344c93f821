// gen_f64.cu -- FP64 instantiations of the generator passes (all variants).
#include "gen_launch.cuh"

namespace scarl {
cudaError_t run_pass_f64(int pass, int v, const GenArgs& a, cudaStream_t s) {
  return run_pass<double>(pass, v, a, s);
}
}  // namespace scarl
