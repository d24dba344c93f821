// post.cu -- standalone post steps of the localization method, each a
// memory-bound elementwise or gather pass over HBM:
//   k_blend_tile   : one tile into the global field (PoU, overlap sum,
//                    assembly, marginal) -- the DCT path's epilogue;
//   k_apply_pou    : apply_UnityPartition_mtx (SRC_F/main_ScaRL.f90:1216-1301);
//   k_add_overlap  : add_overlap over all tiles held in HBM (:984-1210);
//   k_marginal     : multiVariateTransformation (:1355-1395);
//   k_affine       : (x - a) / b, the standardisation of normalize_field (:903-953);
//   k_sums         : FP64 sums of x and x^2 per realisation (moments, normalisation).
#include <algorithm>

#include "epilogue.cuh"
#include "scarl_internal.h"

namespace scarl {

static inline unsigned grid_for(int64_t n, int threads, int cap = 148 * 32) {
  int64_t g = (n + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

template <typename T>
__global__ void k_blend_tile(const T* __restrict__ tile, int Nx, int Ny, int Nz, const Epilogue e) {
  const int64_t n = (int64_t)Nx * Ny * Nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % Nx);
    const int64_t r = i / Nx;
    const int y = (int)(r % Ny), z = (int)(r / Ny);
    epilogue_point<T>(e, x, y, z, Nx, Ny, tile[i]);
  }
}

cudaError_t launch_blend_tile(int dt, const void* tile, const int Np[3], const Epilogue& e,
                              cudaStream_t s) {
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  if (dt == 8) k_blend_tile<double><<<grid_for(n, 256), 256, 0, s>>>((const double*)tile, Np[0], Np[1], Np[2], e);
  else k_blend_tile<float><<<grid_for(n, 256), 256, 0, s>>>((const float*)tile, Np[0], Np[1], Np[2], e);
  return cudaGetLastError();
}

struct PouAxes { BlendAxis ax[3]; };

template <typename T>
__global__ void k_apply_pou(T* __restrict__ f, int Nx, int Ny, int Nz, const PouAxes p) {
  const int64_t n = (int64_t)Nx * Ny * Nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % Nx);
    const int64_t r = i / Nx;
    const int y = (int)(r % Ny), z = (int)(r / Ny);
    double w = p.ax[0].lo[x];
    w = __dmul_rn(w, p.ax[1].lo[y]);
    w = __dmul_rn(w, p.ax[2].lo[z]);
    w = __dmul_rn(w, p.ax[0].hi[x]);
    w = __dmul_rn(w, p.ax[1].hi[y]);
    w = __dmul_rn(w, p.ax[2].hi[z]);
    f[i] = (T)((double)f[i] * sqrt(w));
  }
}

cudaError_t launch_apply_pou(int dt, void* field, const int Np[3], const BlendAxis ax[3],
                             cudaStream_t s) {
  PouAxes p{{ax[0], ax[1], ax[2]}};
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  if (dt == 8) k_apply_pou<double><<<grid_for(n, 256), 256, 0, s>>>((double*)field, Np[0], Np[1], Np[2], p);
  else k_apply_pou<float><<<grid_for(n, 256), 256, 0, s>>>((float*)field, Np[0], Np[1], Np[2], p);
  return cudaGetLastError();
}

// out[r] = in[r] + sum over the 26 directions s (reference order, x fastest)
// of in[r - s] on the receiver's region(-s), read at the sender's region(s).
struct OvlArgs { int Np[3], No[3], T[3]; };

__global__ void k_add_overlap(const double* __restrict__ in, double* __restrict__ out,
                              const OvlArgs a) {
  const int64_t nt = (int64_t)a.Np[0] * a.Np[1] * a.Np[2];
  const int nb = a.T[0] * a.T[1] * a.T[2];
  const int64_t n = nt * nb;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(g / nt);
    const int64_t i = g - (int64_t)r * nt;
    int c[3];
    c[0] = (int)(i % a.Np[0]);
    const int64_t q = i / a.Np[0];
    c[1] = (int)(q % a.Np[1]);
    c[2] = (int)(q / a.Np[1]);
    int pos[3];
    {
      int rest = r;
      pos[2] = rest / (a.T[0] * a.T[1]);
      rest -= pos[2] * a.T[0] * a.T[1];
      pos[1] = rest / a.T[0];
      pos[0] = rest - pos[1] * a.T[0];
    }
    double acc = 0.0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          if (ii == 0 && jj == 0 && kk == 0) continue;
          const int s[3] = {ii, jj, kk};
          int src[3], sc[3];
          bool ok = true;
          for (int d = 0; d < 3 && ok; ++d) {
            src[d] = pos[d] - s[d];
            if (src[d] < 0 || src[d] > a.T[d] - 1) ok = false;
            // receiver region(-s): s=+1 -> low side x < No, s=-1 -> high side
            const int lo = (s[d] == 1) ? 0 : (s[d] == -1 ? a.Np[d] - a.No[d] : 0);
            const int hi = (s[d] == 1) ? a.No[d] - 1 : a.Np[d] - 1;
            if (hi <= lo) ok = false;  // degenerate (maxP <= minP)
            if (c[d] < lo || c[d] > hi) ok = false;
            sc[d] = (s[d] == 1) ? c[d] + a.Np[d] - a.No[d] : (s[d] == -1 ? c[d] - (a.Np[d] - a.No[d]) : c[d]);
          }
          if (!ok) continue;
          const int rs = a.T[0] * a.T[1] * src[2] + a.T[0] * src[1] + src[0];
          acc = acc + in[(int64_t)rs * nt + sc[0] + (int64_t)a.Np[0] * (sc[1] + (int64_t)a.Np[1] * sc[2])];
        }
    out[g] = in[g] + acc;
  }
}

cudaError_t launch_add_overlap(const double* in, double* out, const int Np[3],
                               const int Np_ovlp[3], const int topo[3], cudaStream_t s) {
  OvlArgs a;
  for (int d = 0; d < 3; ++d) { a.Np[d] = Np[d]; a.No[d] = Np_ovlp[d]; a.T[d] = topo[d]; }
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2] * topo[0] * topo[1] * topo[2];
  k_add_overlap<<<grid_for(n, 256), 256, 0, s>>>(in, out, a);
  return cudaGetLastError();
}

template <typename T>
__global__ void k_marginal(T* __restrict__ f, int64_t n, int kind, T sc, T mu) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v = f[i] * sc + mu;
    f[i] = (kind == 2) ? exp(v) : v;
  }
}

cudaError_t launch_marginal(int dt, void* f, int64_t n, int kind, double sc, double mu,
                            cudaStream_t s) {
  if (dt == 8) k_marginal<double><<<grid_for(n, 256), 256, 0, s>>>((double*)f, n, kind, sc, mu);
  else k_marginal<float><<<grid_for(n, 256), 256, 0, s>>>((float*)f, n, kind, (float)sc, (float)mu);
  return cudaGetLastError();
}

template <typename T>
__global__ void k_affine(T* __restrict__ f, int64_t n, T sub, T div) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    f[i] = (f[i] - sub) / div;
}

cudaError_t launch_affine(int dt, void* f, int64_t n, double sub, double div, cudaStream_t s) {
  if (dt == 8) k_affine<double><<<grid_for(n, 256), 256, 0, s>>>((double*)f, n, sub, div);
  else k_affine<float><<<grid_for(n, 256), 256, 0, s>>>((float*)f, n, (float)sub, (float)div);
  return cudaGetLastError();
}

// Deterministic FP64 partial sums: block (b, e) covers a fixed slice of
// realisation e; partial[(e*nb + b)*2 + {0,1}] = {sum x, sum x^2}.
constexpr int kSumT = 256;
int sums_blocks(int64_t xN) { return (int)std::max<int64_t>(1, std::min<int64_t>((xN + 4095) / 4096, 148 * 4)); }

template <typename T>
__global__ void __launch_bounds__(kSumT) k_sums(const T* __restrict__ f, int64_t xN, double* partial) {
  const int e = blockIdx.y, nb = gridDim.x;
  const T* p = f + (int64_t)e * xN;
  const int64_t chunk = (xN + nb - 1) / nb;
  const int64_t lo = (int64_t)blockIdx.x * chunk, hi = (lo + chunk < xN) ? lo + chunk : xN;
  double s = 0.0, s2 = 0.0;
  constexpr int U = 8;  // independent loads in flight per thread
  int64_t i = lo + threadIdx.x;
  for (; i + (U - 1) * kSumT < hi; i += U * kSumT) {
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = __ldg(p + i + u * kSumT);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const double d = (double)v[u];
      s += d;
      s2 += d * d;
    }
  }
  for (; i < hi; i += kSumT) {
    const double v = (double)p[i];
    s += v;
    s2 += v * v;
  }
  __shared__ double r1[kSumT / 32], r2[kSumT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) { r1[threadIdx.x >> 5] = s; r2[threadIdx.x >> 5] = s2; }
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < kSumT / 32 ? r1[threadIdx.x] : 0.0;
    s2 = threadIdx.x < kSumT / 32 ? r2[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_down_sync(0xffffffffu, s, o);
      s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if (threadIdx.x == 0) {
      partial[((int64_t)e * nb + blockIdx.x) * 2] = s;
      partial[((int64_t)e * nb + blockIdx.x) * 2 + 1] = s2;
    }
  }
}

cudaError_t launch_sums(int dt, const void* f, int64_t xN, int nmc, double* partial, int nb,
                        cudaStream_t s) {
  dim3 grid(nb, nmc);
  if (dt == 8) k_sums<double><<<grid, kSumT, 0, s>>>((const double*)f, xN, partial);
  else k_sums<float><<<grid, kSumT, 0, s>>>((const float*)f, xN, partial);
  return cudaGetLastError();
}

}  // namespace scarl
