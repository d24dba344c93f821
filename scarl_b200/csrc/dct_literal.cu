// dct_literal.cu -- the reference's active generator, gen_std_gauss_FFT
// (SRC_F/fftw_ScaRL.f90:261-418), in FP64:
//   k_dct_spec : Sk = gamma * sqrt(prod_d corrL_d exp(-PI k_d^2)) * cos(2 PI phi)
//                on the (Np/2)^3 octant (the rest of the reference's array is
//                uninitialised; it is zero here and never stored).
//   k_dct_axis : unnormalised DCT-III (FFTW REDFT01) along one axis as a
//                direct sum y_n = sum_i c_i x_i cos(pi i (2n+1) / (2N)),
//                c_0 = 1, c_i = 2, with exactly reduced angle indices; only
//                the octant's nonzero inputs are summed.  Three launches (x, y,
//                z) form the 3D transform of fftw_plan_r2r_3d(REDFT01 x3).
#include <algorithm>

#include "scarl_common.cuh"
#include "scarl_internal.h"

namespace scarl {

constexpr double kPiRefD = 3.1415926535898;  // SRC_F/constants_ScaRL.f90:5

__global__ void k_dct_spec(const DctArgs a) {
  const int64_t n = (int64_t)a.K[0] * a.K[1] * a.K[2];
  for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < n;
       o += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(o % a.K[0]);
    const int64_t r = o / a.K[0];
    const int j = (int)(r % a.K[1]);
    const int k = (int)(r / a.K[1]);
    double S = 1.0;
    S = __dmul_rn(__dmul_rn(S, a.corrL[0]), a.cx[i]);
    S = __dmul_rn(__dmul_rn(S, a.corrL[1]), a.cy[j]);
    S = __dmul_rn(__dmul_rn(S, a.corrL[2]), a.cz[k]);
    double phi;
    if (a.phi) {
      phi = a.phi[o];
    } else {
      const u32x4 q = philox4x32_10({(uint32_t)o, (uint32_t)((uint64_t)o >> 32), a.stream, 1u}, a.k0, a.k1);
      phi = u01_d(q.x, q.y);
    }
    const double g = a.gamma ? a.gamma[o] : 1.0;
    const double c = cos(__dmul_rn(__dmul_rn(2.0, kPiRefD), phi));
    a.sk[o] = __dmul_rn(__dmul_rn(g, sqrt(S)), c);
  }
}

// Batched direct DCT-III: out(l, n) = sum_{i<K} in(l, i) C(i, n), n < N.
// Line l = la + na * lb addresses in[la*sa + lb*sb + i*si] and
// out[la*oa + lb*ob + n*so].  Tiles of TL lines x TN outputs, TK inputs.
struct DctAxis {
  const double* in;
  double* out;
  const double* ctab;  // cos(pi m / (2N)), m < 4N
  int K, N, na;
  int64_t nl;
  int64_t sa, sb, si, oa, ob, so;
};

constexpr int TL = 64, TN = 64, TK = 16;

template <bool LINES_CONTIG>
__global__ void __launch_bounds__(256) k_dct_axis(const DctAxis d) {
  __shared__ double xs[TK][TL + 1];
  __shared__ double cs[TK][TN + 1];
  const int tid = threadIdx.x;
  const int64_t l0 = (int64_t)blockIdx.x * TL;
  const int n0 = blockIdx.y * TN;
  const int tl = tid % 16, tn = tid / 16;  // 4x4 outputs per thread
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  const int64_t fourN = 4 * (int64_t)d.N;
  for (int i0 = 0; i0 < d.K; i0 += TK) {
    for (int e = tid; e < TK * TL; e += 256) {
      int ii, ll;
      if (LINES_CONTIG) { ll = e % TL; ii = e / TL; }
      else { ii = e % TK; ll = e / TK; }
      const int64_t l = l0 + ll;
      const int i = i0 + ii;
      double v = 0.0;
      if (l < d.nl && i < d.K) {
        const int64_t la = l % d.na, lb = l / d.na;
        v = d.in[la * d.sa + lb * d.sb + (int64_t)i * d.si];
      }
      xs[ii][ll] = v;
    }
    for (int e = tid; e < TK * TN; e += 256) {
      const int nn = e % TN, ii = e / TN;
      const int i = i0 + ii, n = n0 + nn;
      double c = 0.0;
      if (i < d.K && n < d.N) {
        const int64_t m = ((int64_t)i * (2 * (int64_t)n + 1)) % fourN;
        c = (i == 0) ? 1.0 : 2.0 * d.ctab[m];
      }
      cs[ii][nn] = c;
    }
    __syncthreads();
#pragma unroll
    for (int ii = 0; ii < TK; ++ii) {
      double xv[4], cv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) xv[a] = xs[ii][tl + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) cv[b] = cs[ii][tn + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(xv[a], cv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t l = l0 + tl + 16 * a;
    if (l >= d.nl) continue;
    const int64_t la = l % d.na, lb = l / d.na;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int n = n0 + tn + 16 * b;
      if (n < d.N) d.out[la * d.oa + lb * d.ob + (int64_t)n * d.so] = acc[a][b];
    }
  }
}

static cudaError_t run_axis(const DctAxis& d, bool lines_contig, cudaStream_t s) {
  if (d.nl == 0 || d.N == 0) return cudaSuccess;
  dim3 grid((unsigned)((d.nl + TL - 1) / TL), (d.N + TN - 1) / TN);
  if (lines_contig) k_dct_axis<true><<<grid, 256, 0, s>>>(d);
  else k_dct_axis<false><<<grid, 256, 0, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_dct_literal(const DctArgs& a, cudaStream_t s) {
  const int N0 = a.Np[0], N1 = a.Np[1], N2 = a.Np[2];
  const int K0 = a.K[0], K1 = a.K[1], K2 = a.K[2];
  const int64_t nk = (int64_t)K0 * K1 * K2;
  if (nk == 0) {
    return cudaMemsetAsync(a.out, 0, sizeof(double) * (size_t)N0 * N1 * N2, s);
  }
  k_dct_spec<<<(unsigned)std::min<int64_t>((nk + 255) / 256, 148 * 16), 256, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // x: lines (j,k) of the octant, inputs i < K0, outputs n < N0
  DctAxis dx{a.sk, a.t1, a.ctab[0], K0, N0, K1, (int64_t)K1 * K2,
             (int64_t)K0, (int64_t)K0 * K1, 1, (int64_t)N0, (int64_t)N0 * K1, 1};
  if ((e = run_axis(dx, false, s)) != cudaSuccess) return e;
  // y: lines (i < N0, k < K2), inputs j < K1, outputs n < N1
  DctAxis dy{a.t1, a.t2, a.ctab[1], K1, N1, N0, (int64_t)N0 * K2,
             1, (int64_t)N0 * K1, (int64_t)N0, 1, (int64_t)N0 * N1, (int64_t)N0};
  if ((e = run_axis(dy, true, s)) != cudaSuccess) return e;
  // z: lines (i, j) < N0*N1, inputs k < K2, outputs n < N2
  DctAxis dz{a.t2, a.out, a.ctab[2], K2, N2, N0 * N1, (int64_t)N0 * N1,
             1, 0, (int64_t)N0 * N1, 1, 0, (int64_t)N0 * N1};
  return run_axis(dz, true, s);
}

}  // namespace scarl
