// gen_padded.cu -- dispatch of the padded periodic-grid generator passes
// (kernels in gen_kernels.cuh, variants in gen_launch.cuh, instantiated in
// gen_f32.cu / gen_f64.cu) and the FP64 spectral normalisation sum.
#include "gen_launch.cuh"

namespace scarl {

cudaError_t run_pass_f32(int pass, int v, const GenArgs& a, cudaStream_t s);
cudaError_t run_pass_f64(int pass, int v, const GenArgs& a, cudaStream_t s);

cudaError_t launch_gen_pass(int dt, int pass, const GenArgs& a, cudaStream_t s) {
  if (pass < 1 || pass > 3) return cudaErrorInvalidValue;
  const int v = a.var[pass - 1];
  return dt == 8 ? run_pass_f64(pass, v, a, s) : run_pass_f32(pass, v, a, s);
}

int gen_variant_count(int dt, int pass) {
  if (pass == 3) return dt == 8 ? RowVars<double>::n : RowVars<float>::n;
  return dt == 8 ? ColVars<double>::n : ColVars<float>::n;
}

// ---------------------------------------------------------------------------
// FP64 spectral variance-normalisation sum over the full periodic grid.
// ---------------------------------------------------------------------------
constexpr int kSumThreads = 256;
int spectrum_sum_blocks() { return 148 * 8; }

__global__ void __launch_bounds__(kSumThreads) k_spec_sum(const GenArgs a, const double* rx,
                                                          const double* ry, const double* rz,
                                                          double craw2, double* partial) {
  const double* qx = static_cast<const double*>(a.qx);
  const double* qy = static_cast<const double*>(a.qy);
  const double* qz = static_cast<const double*>(a.qz);
  const int64_t total = (int64_t)a.Hx * a.P[1] * a.P[2];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(i % a.Hx);
    const int64_t r = i / a.Hx;
    const int ky = (int)(r % a.P[1]);
    const int kz = (int)(r / a.P[1]);
    const double c = (kx == 0 || 2 * kx == a.P[0]) ? 1.0 : 2.0;
    double v;
    if (a.amp == AMP_SEPARABLE) {
      const double A = rx[kx] * ry[ky] * rz[kz];
      v = A * A;
    } else {
      v = craw2 * pow(1.0 + qx[kx] + qy[ky] + qz[kz], 2.0 * a.expo);
    }
    acc += c * v;
  }
  __shared__ double red[kSumThreads / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kSumThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

cudaError_t launch_spectrum_sum(const GenArgs& a, const double* rx, const double* ry,
                                const double* rz, double craw2, double* partial, int nblocks,
                                cudaStream_t s) {
  k_spec_sum<<<nblocks, kSumThreads, 0, s>>>(a, rx, ry, rz, craw2, partial);
  return cudaGetLastError();
}

}  // namespace scarl
