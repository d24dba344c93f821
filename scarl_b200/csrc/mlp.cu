// mlp.cu -- the learned padding / overlap predictor (no counterpart in the
// reference): label generation from the method's own expected covariance, and
// a 3-layer, 64-wide MLP stored in BF16 with FP32 accumulation, trained by
// the forward/backward kernels below.
//
// Labels (k_pad_labels, FP64).  The expected covariance of the padded
// periodic method along an axis of N points at padded length P is the
// normalised 1-D spectral sum of the model's axis spectrum s(f) on the
// frequencies k / P:
//   C_P(h) = [s(0) + 2 sum_{0<k<P/2} s(k/P) cos(2 pi k h / P) (+ s(1/2) cos(pi h))]
//            / [same with h = 0],
// s(f) = exp(-pi l^2 f^2) (Gaussian) or (1 + 4 pi^2 a^2 f^2)^-(nu + 1/2) (Matern,
// a = l Gamma(nu) / (2 sqrt(pi) Gamma(nu + 1/2))).  The padding error is
// e(P) = max_{h<N} |C_P(h) - C_ref(h)| against Pref = 32 N (the infinitely
// padded method); the label is the smallest integer P with e(P) <= tol
// (bisection).  Blending two tiles whose overlap holds W points scales the
// covariance of a pair at lag h by cos(pi min(h/(W-1), 1) / 2) at worst (the
// square-root weights are cos and sin of the same ramp), so the overlap label
// is the smallest W with (1 - cos(pi min(h/(W-1), 1) / 2)) |C_ref(h)| <= tol
// for every h < N.
#include <cuda_bf16.h>

#include "scarl_internal.h"

namespace scarl {

namespace {

constexpr int kLabT = 256;
constexpr int kMaxHalf = 4097;  // Pref / 2 + 1 for N <= 256

__device__ __forceinline__ double axis_spec(const PadLabelIn& c, double f) {
  if (c.kind == 1) return exp(-3.14159265358979323846 * c.ell * c.ell * f * f);
  return pow(1.0 + c.q * f * f, -(c.nu + 0.5));
}

// C_P(h) for every lag h < N (one per thread, strided), spectrum in sm.
__device__ void cov_line(const PadLabelIn& c, int P, double* sm, double* cov, int N) {
  const int half = P / 2;
  for (int k = threadIdx.x; k <= half; k += blockDim.x) sm[k] = axis_spec(c, (double)k / (double)P);
  __syncthreads();
  for (int h = threadIdx.x; h < N; h += blockDim.x) {
    double s, co;
    sincospi(2.0 * (double)h / (double)P, &s, &co);
    double cr = 1.0, ci = 0.0;  // cos / sin of 2 pi k h / P by rotation
    double num = sm[0], den = sm[0];
    const int top = (P % 2 == 0) ? half : half + 1;  // k < P/2 pairs with -k
    for (int k = 1; k < top; ++k) {
      const double nr = cr * co - ci * s;
      ci = cr * s + ci * co;
      cr = nr;
      num += 2.0 * sm[k] * cr;
      den += 2.0 * sm[k];
    }
    if (P % 2 == 0) {
      num += sm[half] * ((h & 1) ? -1.0 : 1.0);
      den += sm[half];
    }
    cov[h] = num / den;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kLabT) k_pad_labels(const PadLabelIn* in, PadLabelOut* out,
                                                      int n, double tol) {
  __shared__ double sm[kMaxHalf];
  __shared__ double cref[256], cp[256];
  __shared__ double red[kLabT / 32];
  const int i = blockIdx.x;
  if (i >= n) return;
  const PadLabelIn c = in[i];
  const int N = c.N;
  auto block_max = [&](double v) -> double {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    __syncthreads();
    return m;
  };
  cov_line(c, 32 * N, sm, cref, N);
  auto err_at = [&](int P) -> double {
    cov_line(c, P, sm, cp, N);
    double e = 0.0;
    for (int h = threadIdx.x; h < N; h += blockDim.x) e = fmax(e, fabs(cp[h] - cref[h]));
    return block_max(e);
  };
  // padding: smallest integer P in [N, 16 N] with e(P) <= tol
  int lo = N, hi = 16 * N;
  const double ehi = err_at(hi);
  PadLabelOut o;
  o.saturated = ehi > tol ? 1 : 0;
  if (err_at(lo) <= tol) hi = lo;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (err_at(mid) <= tol) hi = mid;
    else lo = mid;
  }
  o.P = hi;
  // overlap: smallest W in [2, N] with max_h (1 - cos(pi min(h/(W-1),1)/2)) C_ref(h) <= tol
  auto oerr = [&](int W) -> double {
    double e = 0.0;
    for (int h = threadIdx.x; h < N; h += blockDim.x) {
      const double t = fmin((double)h / (double)(W - 1), 1.0);
      e = fmax(e, (1.0 - cospi(0.5 * t)) * fabs(cref[h]));
    }
    return block_max(e);
  };
  int wl = 2, wh = N;
  if (oerr(wl) <= tol) wh = wl;
  while (wh - wl > 1) {
    const int mid = (wl + wh) / 2;
    if (oerr(mid) <= tol) wh = mid;
    else wl = mid;
  }
  o.W = wh;
  if (threadIdx.x == 0) out[i] = o;
}

// e(P) of given paddings (the check of a prediction).
__global__ void __launch_bounds__(kLabT) k_pad_error(const PadLabelIn* in, const int* P, double* err,
                                                     int n) {
  __shared__ double sm[kMaxHalf];
  __shared__ double cref[256], cp[256];
  __shared__ double red[kLabT / 32];
  const int i = blockIdx.x;
  if (i >= n) return;
  const PadLabelIn c = in[i];
  cov_line(c, 32 * c.N, sm, cref, c.N);
  cov_line(c, P[i], sm, cp, c.N);
  double e = 0.0;
  for (int h = threadIdx.x; h < c.N; h += blockDim.x) e = fmax(e, fabs(cp[h] - cref[h]));
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_down_sync(0xffffffffu, e, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    err[i] = m;
  }
}

// ---------------------------------------------------------------------------
// MLP: x (16) -> 64 -> 64 -> 2, ReLU, weights BF16, FP32 accumulation.
// Master parameters (FP32) in one array: W1[64][16] b1[64] W2[64][64] b2[64]
// W3[2][64] b3[2].
// ---------------------------------------------------------------------------
constexpr int IN = kMlpIn, HID = kMlpHidden, OUT = kMlpOut;
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID,
              OW3 = OB2 + HID, OB3 = OW3 + OUT * HID;
static_assert(OB3 + OUT == kMlpParams, "parameter layout");
constexpr int TS = 64;    // samples per block
constexpr int MT = 256;   // threads per block

struct MlpSmem {
  __nv_bfloat16 w1[HID * IN], w2[HID * HID], w3[OUT * HID];
  float b1[HID], b2[HID], b3[OUT];
  __nv_bfloat16 x[TS * IN], h1[TS * HID], h2[TS * HID];
  float y[TS * OUT], dy[TS * OUT];
  float d2[TS * HID], d1[TS * HID];
};

__device__ void load_weights(MlpSmem& s, const __nv_bfloat16* wb, const float* p) {
  for (int i = threadIdx.x; i < HID * IN; i += blockDim.x) s.w1[i] = wb[OW1 + i];
  for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) s.w2[i] = wb[OW2 + i];
  for (int i = threadIdx.x; i < OUT * HID; i += blockDim.x) s.w3[i] = wb[OW3 + i];
  for (int i = threadIdx.x; i < HID; i += blockDim.x) {
    s.b1[i] = p[OB1 + i];
    s.b2[i] = p[OB2 + i];
  }
  if (threadIdx.x < OUT) s.b3[threadIdx.x] = p[OB3 + threadIdx.x];
}

// Forward pass of the block's samples; rows past n are zero inputs.
__device__ void forward(MlpSmem& s, const __nv_bfloat16* X, int s0, int n) {
  for (int i = threadIdx.x; i < TS * IN; i += blockDim.x) {
    const int r = i / IN;
    s.x[i] = (s0 + r < n) ? X[(size_t)(s0 + r) * IN + i % IN] : __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
    const int r = i / HID, j = i % HID;
    float a = s.b1[j];
    for (int k = 0; k < IN; ++k) a = fmaf(__bfloat162float(s.x[r * IN + k]), __bfloat162float(s.w1[j * IN + k]), a);
    s.h1[i] = __float2bfloat16(fmaxf(a, 0.f));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
    const int r = i / HID, j = i % HID;
    float a = s.b2[j];
    for (int k = 0; k < HID; ++k) a = fmaf(__bfloat162float(s.h1[r * HID + k]), __bfloat162float(s.w2[j * HID + k]), a);
    s.h2[i] = __float2bfloat16(fmaxf(a, 0.f));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < TS * OUT; i += blockDim.x) {
    const int r = i / OUT, o = i % OUT;
    float a = s.b3[o];
    for (int k = 0; k < HID; ++k) a = fmaf(__bfloat162float(s.h2[r * HID + k]), __bfloat162float(s.w3[o * HID + k]), a);
    s.y[i] = a;
  }
  __syncthreads();
}

// Loss (1/n) sum (y - t)^2 over the n samples and its gradient; weight
// gradients summed over the block in FP32, then added to grad.
__global__ void __launch_bounds__(MT) k_mlp_train(const __nv_bfloat16* X, const float* T, int n,
                                                  const __nv_bfloat16* wb, const float* p,
                                                  float* grad, double* loss) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  const int s0 = blockIdx.x * TS;
  load_weights(s, wb, p);
  __syncthreads();
  forward(s, X, s0, n);
  const float inv = 1.f / (float)n;
  float lsum = 0.f;
  for (int i = threadIdx.x; i < TS * OUT; i += blockDim.x) {
    const int r = i / OUT;
    float d = 0.f;
    if (s0 + r < n) {
      const float e = s.y[i] - T[(size_t)(s0 + r) * OUT + i % OUT];
      lsum += e * e;
      d = 2.f * e * inv;
    }
    s.dy[i] = d;
  }
  __syncthreads();
  // dH2 = (dY W3) * relu'
  for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
    const int r = i / HID, j = i % HID;
    float a = 0.f;
    for (int o = 0; o < OUT; ++o) a = fmaf(s.dy[r * OUT + o], __bfloat162float(s.w3[o * HID + j]), a);
    s.d2[i] = __bfloat162float(s.h2[i]) > 0.f ? a : 0.f;
  }
  __syncthreads();
  // dH1 = (dH2 W2) * relu'
  for (int i = threadIdx.x; i < TS * HID; i += blockDim.x) {
    const int r = i / HID, k = i % HID;
    float a = 0.f;
    for (int j = 0; j < HID; ++j) a = fmaf(s.d2[r * HID + j], __bfloat162float(s.w2[j * HID + k]), a);
    s.d1[i] = __bfloat162float(s.h1[i]) > 0.f ? a : 0.f;
  }
  __syncthreads();
  // weight and bias gradients, summed over the block's samples
  for (int i = threadIdx.x; i < OUT * HID; i += blockDim.x) {
    const int o = i / HID, j = i % HID;
    float a = 0.f;
    for (int r = 0; r < TS; ++r) a = fmaf(s.dy[r * OUT + o], __bfloat162float(s.h2[r * HID + j]), a);
    atomicAdd(grad + OW3 + i, a);
  }
  if (threadIdx.x < OUT) {
    float a = 0.f;
    for (int r = 0; r < TS; ++r) a += s.dy[r * OUT + threadIdx.x];
    atomicAdd(grad + OB3 + threadIdx.x, a);
  }
  for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) {
    const int j = i / HID, k = i % HID;
    float a = 0.f;
    for (int r = 0; r < TS; ++r) a = fmaf(s.d2[r * HID + j], __bfloat162float(s.h1[r * HID + k]), a);
    atomicAdd(grad + OW2 + i, a);
  }
  for (int i = threadIdx.x; i < HID * IN; i += blockDim.x) {
    const int j = i / IN, k = i % IN;
    float a = 0.f;
    for (int r = 0; r < TS; ++r) a = fmaf(s.d1[r * HID + j], __bfloat162float(s.x[r * IN + k]), a);
    atomicAdd(grad + OW1 + i, a);
  }
  for (int j = threadIdx.x; j < HID; j += blockDim.x) {
    float a2 = 0.f, a1 = 0.f;
    for (int r = 0; r < TS; ++r) {
      a2 += s.d2[r * HID + j];
      a1 += s.d1[r * HID + j];
    }
    atomicAdd(grad + OB2 + j, a2);
    atomicAdd(grad + OB1 + j, a1);
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0 && lsum != 0.f) atomicAdd(loss, (double)lsum / (double)n);
}

__global__ void __launch_bounds__(MT) k_mlp_infer(const __nv_bfloat16* X, int n,
                                                  const __nv_bfloat16* wb, const float* p, float* Y) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  const int s0 = blockIdx.x * TS;
  load_weights(s, wb, p);
  __syncthreads();
  forward(s, X, s0, n);
  for (int i = threadIdx.x; i < TS * OUT; i += blockDim.x)
    if (s0 + i / OUT < n) Y[(size_t)s0 * OUT + i] = s.y[i];
}

// Adam on the FP32 master parameters; refreshes the BF16 copies and clears
// the gradient.
__global__ void k_mlp_adam(float* p, float* g, float* m, float* v, __nv_bfloat16* wb, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  wb[i] = __float2bfloat16(pi);
  g[i] = 0.f;
}

__global__ void k_to_bf16(const float* a, __nv_bfloat16* b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16(a[i]);
}

}  // namespace

cudaError_t launch_pad_labels(const PadLabelIn* in, PadLabelOut* out, int n, double tol,
                              cudaStream_t s) {
  k_pad_labels<<<n, kLabT, 0, s>>>(in, out, n, tol);
  return cudaGetLastError();
}

cudaError_t launch_pad_error(const PadLabelIn* in, const int* P, double* err, int n,
                             cudaStream_t s) {
  k_pad_error<<<n, kLabT, 0, s>>>(in, P, err, n);
  return cudaGetLastError();
}

static cudaError_t mlp_smem_attr(const void* k) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
}

cudaError_t launch_mlp_train(const void* X, const float* T, int n, const void* wb, const float* p,
                             float* grad, double* loss, cudaStream_t s) {
  cudaError_t e = mlp_smem_attr((const void*)k_mlp_train);
  if (e != cudaSuccess) return e;
  k_mlp_train<<<(n + TS - 1) / TS, MT, sizeof(MlpSmem), s>>>(
      (const __nv_bfloat16*)X, T, n, (const __nv_bfloat16*)wb, p, grad, loss);
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const void* X, int n, const void* wb, const float* p, float* Y,
                             cudaStream_t s) {
  cudaError_t e = mlp_smem_attr((const void*)k_mlp_infer);
  if (e != cudaSuccess) return e;
  k_mlp_infer<<<(n + TS - 1) / TS, MT, sizeof(MlpSmem), s>>>((const __nv_bfloat16*)X, n,
                                                            (const __nv_bfloat16*)wb, p, Y);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* p, float* g, float* m, float* v, void* wb, float lr, int t,
                            cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(p, g, m, v, (__nv_bfloat16*)wb, lr, b1, b2,
                                                     1e-8f, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* a, void* b, int n, cudaStream_t s) {
  k_to_bf16<<<(n + 255) / 256, 256, 0, s>>>(a, (__nv_bfloat16*)b, n);
  return cudaGetLastError();
}

}  // namespace scarl
