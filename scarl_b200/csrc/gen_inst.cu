// gen_inst.cu -- explicit instantiations of the generator passes (every
// launch variant, single-tile and batched kernels) for one precision and one
// group of line lengths, chosen at compile time so that the instantiations
// build in parallel:
//   SCARL_INST_DT = 4 (FP32) or 8 (FP64)
//   SCARL_INST_N  = 0 (lines of 4..128 points), -1 (mixed lengths 24..112),
//                   -2 (mixed lengths 160..224) or one length 256..2048
#include "gen_launch.cuh"

#ifndef SCARL_INST_DT
#define SCARL_INST_DT 4
#endif
#ifndef SCARL_INST_N
#define SCARL_INST_N 0
#endif

namespace scarl {

template <typename T, int N>
cudaError_t run_pass_len(int pass, int v, const GenArgs& a, const BatchMap* bm, int* nb,
                         cudaStream_t s) {
  return run_pass_n<T, N>(pass, v, a, bm, nb, s);
}

#if SCARL_INST_DT == 8
using InstT = double;
#else
using InstT = float;
#endif

#define SCARL_INST(N)                                                                    \
  template cudaError_t run_pass_len<InstT, N>(int, int, const GenArgs&, const BatchMap*, \
                                              int*, cudaStream_t);
#if SCARL_INST_N == 0
SCARL_INST(4)
SCARL_INST(8)
SCARL_INST(16)
SCARL_INST(32)
SCARL_INST(64)
SCARL_INST(128)
#elif SCARL_INST_N == -1
SCARL_INST(24)
SCARL_INST(40)
SCARL_INST(48)
SCARL_INST(56)
SCARL_INST(80)
SCARL_INST(96)
SCARL_INST(112)
#elif SCARL_INST_N == -2
SCARL_INST(160)
SCARL_INST(192)
SCARL_INST(224)
#else
SCARL_INST(SCARL_INST_N)
#endif

}  // namespace scarl
