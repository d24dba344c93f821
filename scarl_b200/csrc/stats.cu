// stats.cu -- directional covariance estimator of Stat_ScaRL
// (SRC_F/Stat_ScaRL/statistics_RF.f90:258-462, rebuild_Sk_FFT) as a direct
// FP64 lag sum.  The reference forms |FFT(t)/n|^2 per line, averages over
// the other two axes and inverts: that is the circular autocorrelation
//   Sk[m] = 1/(n * nlines) * sum_lines sum_i t_i t_{(i+m) mod n},
//   t = ((x - avg) / std) * w (Tukey window along the line),
// which is what this kernel accumulates for the kept lags m < nkeep.
#include <algorithm>

#include "scarl_internal.h"

namespace scarl {

constexpr int kLagT = 256;
constexpr int kLagLines = 8;  // lines staged per block iteration

int lag_cov_parts(const int L[3], int dir) {
  const int64_t n = L[dir];
  const int64_t nl = (int64_t)L[0] * L[1] * L[2] / n;
  const int64_t groups = (nl + kLagLines - 1) / kLagLines;
  return (int)std::max<int64_t>(1, std::min<int64_t>(groups, 148 * 4));
}

// Each block walks line groups g = blockIdx.x, +gridDim.x, ...; a group is
// kLagLines consecutive lines (consecutive in the fastest of the other axes).
template <typename T>
__global__ void __launch_bounds__(kLagT) k_lag_cov(const T* __restrict__ f, int L0, int L1, int L2,
                                                   int dir, double avg, double sd,
                                                   const double* __restrict__ win, int nkeep,
                                                   double* __restrict__ partial) {
  extern __shared__ double tl[];  // [kLagLines][n]
  const int n = dir == 0 ? L0 : (dir == 1 ? L1 : L2);
  // line index l -> (a, b) over the two other axes, a fastest
  const int na = dir == 0 ? L1 : L0;
  const int nbx = dir == 2 ? L1 : L2;
  const int64_t nl = (int64_t)na * nbx;
  const int64_t sa = dir == 0 ? L0 : 1;
  const int64_t sb = dir == 2 ? L0 : (int64_t)L0 * L1;
  const int64_t st = dir == 0 ? 1 : (dir == 1 ? L0 : (int64_t)L0 * L1);
  const int64_t ngroups = (nl + kLagLines - 1) / kLagLines;
  // lag ownership: thread handles lags m = threadIdx.x + kLagT * q
  constexpr int QMAX = 8;  // up to 2048 kept lags
  double acc[QMAX];
#pragma unroll
  for (int q = 0; q < QMAX; ++q) acc[q] = 0.0;
  for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    __syncthreads();
    for (int e = threadIdx.x; e < kLagLines * n; e += kLagT) {
      int bl, i;
      if (dir == 0) { bl = e / n; i = e - bl * n; }
      else { bl = e % kLagLines; i = e / kLagLines; }
      const int64_t l = g * kLagLines + bl;
      double v = 0.0;
      if (l < nl) {
        const int64_t a = l % na, b = l / na;
        v = (((double)f[a * sa + b * sb + (int64_t)i * st] - avg) / sd) * win[i];
      }
      tl[bl * n + i] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < QMAX; ++q) {
      const int m = threadIdx.x + kLagT * q;
      if (m >= nkeep) break;
      double s = 0.0;
      for (int bl = 0; bl < kLagLines; ++bl) {
        const double* t = tl + bl * n;
        int j = m;
        for (int i = 0; i < n; ++i) {
          s = fma(t[i], t[j], s);
          if (++j == n) j = 0;
        }
      }
      acc[q] += s;
    }
  }
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int m = threadIdx.x + kLagT * q;
    if (m < nkeep) partial[(int64_t)blockIdx.x * nkeep + m] = acc[q];
  }
}

cudaError_t launch_lag_cov(int dt, const void* f, const int L[3], int dir, double avg,
                           double sd, const double* win, int nkeep, double* partial, int nparts,
                           cudaStream_t s) {
  if (nkeep > kLagT * 8) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * kLagLines * (size_t)L[dir];
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (dt == 8) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_lag_cov<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lag_cov<double><<<nparts, kLagT, smem, s>>>((const double*)f, L[0], L[1], L[2], dir, avg, sd,
                                                   win, nkeep, partial);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_lag_cov<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lag_cov<float><<<nparts, kLagT, smem, s>>>((const float*)f, L[0], L[1], L[2], dir, avg, sd,
                                                  win, nkeep, partial);
  }
  return cudaGetLastError();
}

// Sum of n FP64 pairs (x, y) into out[0], out[1] in a fixed order: block b
// sums the pairs b, b + gridDim.x, ... (each thread a fixed stride, then a
// fixed tree) into part[b]; one block then sums the gridDim.x parts.
constexpr int kPairBlocks = 148;
__device__ __forceinline__ void pair_tree(double a, double b, double* out) {
  __shared__ double r0[256], r1[256];
  r0[threadIdx.x] = a;
  r1[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      r0[threadIdx.x] += r0[threadIdx.x + w];
      r1[threadIdx.x] += r1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = r0[0];
    out[1] = r1[0];
  }
}
__global__ void __launch_bounds__(256) k_pair_part(const double* __restrict__ p, int64_t n,
                                                   double* __restrict__ part) {
  double a = 0.0, b = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
    a += p[2 * i];
    b += p[2 * i + 1];
  }
  pair_tree(a, b, part + 2 * blockIdx.x);
}
__global__ void __launch_bounds__(256) k_pair_final(const double* __restrict__ part, int nparts,
                                                    double* __restrict__ out) {
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nparts; i += 256) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  pair_tree(a, b, out);
}

// part: 2 kPairBlocks doubles of scratch.
cudaError_t launch_pair_sum(const double* pairs, int64_t n, double* part, double* out, cudaStream_t s) {
  k_pair_part<<<kPairBlocks, 256, 0, s>>>(pairs, n, part);
  k_pair_final<<<1, 256, 0, s>>>(part, kPairBlocks, out);
  return cudaGetLastError();
}
int pair_sum_parts() { return kPairBlocks; }

}  // namespace scarl
