// gen_kernels.cuh -- kernels of the padded periodic-grid generator (the spectral method of
// SRC_F/fftw_ScaRL.f90:157-255 with SRC_F/spectra_ScaRL.f90:10-142, made
// Hermitian/C2R), as three HBM passes over a complex half spectrum
// H[kx in 0..P0/2][ky][kz] of the tile's padded grid P:
//
//   pass 1  k_gen_z : synthesise H line by line along kz (amplitude x random
//                     normals, no read from memory), inverse DFT along z,
//                     keep z < Nz.  Output kx-fastest rows of pitch Hpad.
//   pass 2  k_mid_y : inverse DFT along y for every (kx, z < Nz), keep
//                     y < Ny, in place.
//   pass 3  k_c2r_x : Hermitian C2R along x for every (y, z) line (one
//                     half-length complex DFT plus the even/odd split), keep
//                     x < Nx, then the fused epilogue: plain crop, or the
//                     partition-of-unity blend into the global field with the
//                     marginal transform applied by the tile that finishes a
//                     point (SRC_F/main_ScaRL.f90:1216-1301, 984-1210,
//                     1355-1395).
#pragma once

#include "epilogue.cuh"
#include "fft_engine.cuh"
#include "scarl_internal.h"

namespace scarl {

constexpr double kPiRefG = 3.1415926535898;  // SRC_F/constants_ScaRL.f90:5

// ---------------------------------------------------------------------------
// Literal build_Sk_mtx value at padded coordinate (kx, ky, kz), halved for
// the C2R form (Re of the c2c = C2R with H = Sk/2 on kx >= 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int shino_index(int c, int P, int sz) {
  if (c < sz) return c;
  if (c >= P - sz) return c - (P - 2 * sz);
  return -1;
}

template <typename T>
__device__ __forceinline__ cplx_t<T> shino_mode(const GenArgs& a, int kx, int ky, int kz) {
  const int n1 = a.sz[0], n2 = 2 * a.sz[1], n3 = 2 * a.sz[2];
  const int i0 = kx;
  const int j0 = shino_index(ky, a.P[1], a.sz[1]);
  const int k0 = shino_index(kz, a.P[2], a.sz[2]);
  if (i0 < 1 || i0 >= n1 || j0 <= 0 || k0 <= 0 || j0 >= n2 - 1 || k0 >= n3 - 1) return mk(T(0), T(0));
  const uint64_t e = (uint64_t)i0 + (uint64_t)n1 * ((uint64_t)j0 + (uint64_t)n2 * (uint64_t)k0);
  const uint32_t s = pm_jump(a.pm_s1, e, a.pm_pw);
  const double u = (double)(int32_t)s * 4.656612875E-10;
  const double ph = __dmul_rn(__dmul_rn(2.0, kPiRefG), u);
  const double c = (double)(float)cos(ph);
  const double sn = (double)(float)sin(ph);
  const double bi = (double)i0;
  const double bj = (double)(j0 < a.sz[1] ? j0 : n2 - 1 - j0);
  const double bk = (double)(k0 < a.sz[2] ? k0 : n3 - 1 - k0);
  const double arg = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(bi, bi), a.de[0]),
                                         __dmul_rn(__dmul_rn(bj, bj), a.de[1])),
                               __dmul_rn(__dmul_rn(bk, bk), a.de[2]));
  const double sv = sqrt(exp(-arg));
  const double re = __dmul_rn(__dmul_rn(__dmul_rn(c, sv), a.shino_scale), a.shino_f);
  const double im = __dmul_rn(__dmul_rn(__dmul_rn(sn, sv), a.shino_scale), a.shino_f);
  return mk((T)(0.5 * re), (T)(0.5 * im));
}

template <typename T> __device__ __forceinline__ T fast_div(T a, T b);
template <> __device__ __forceinline__ float fast_div<float>(float a, float b) { return __fdividef(a, b); }
template <> __device__ __forceinline__ double fast_div<double>(double a, double b) { return a / b; }

template <typename T> __device__ __forceinline__ T powT(T s, T e);
template <> __device__ __forceinline__ float powT<float>(float s, float e) { return powf(s, e); }
template <> __device__ __forceinline__ double powT<double>(double s, double e) { return pow(s, e); }

// ---------------------------------------------------------------------------
// Pass 1: synthesise + inverse DFT along z.
// ---------------------------------------------------------------------------
template <typename T, int N, int E, int B, int SPEC>
__device__ __forceinline__ void gen_z_body(const GenArgs& a, int bx, int ky) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int kx = bx * B + b;
  const bool valid = kx < a.Hx;
  C* work = static_cast<C*>(a.work);
  const T* ax = static_cast<const T*>(a.ax);
  const T* ay = static_cast<const T*>(a.ay);
  const T* az = static_cast<const T*>(a.az);
  const T* qx = static_cast<const T*>(a.qx);
  const T* qy = static_cast<const T*>(a.qy);
  const T* qz = static_cast<const T*>(a.qz);
  T fx = T(0), fy = T(0);
  if constexpr (SPEC != SPEC_SHINO) {
    if (valid) {
      if (a.amp == AMP_SEPARABLE) { fx = ax[kx]; fy = ay[ky]; }
      else { fx = ax[kx]; fy = T(1) + qx[kx] + qy[ky]; }
    }
  }
  const uint64_t mrow = (uint64_t)kx + (uint64_t)a.Hx * (uint64_t)ky;
  const uint64_t mz = (uint64_t)a.Hx * (uint64_t)a.P[1];
  auto amp = [&](int kz) -> T {
    if (a.amp == AMP_SEPARABLE) return fx * fy * az[kz];
    if (a.amp == AMP_RECIP) return fast_div(fx, fy + qz[kz]);
    return fx * powT<T>(fy + qz[kz], (T)a.expo);
  };
  // First-stage inputs kz = j + r N/R1; r and r + R1/2 are kz and kz + N/2,
  // the two modes of one Philox draw.
  auto load = [&](int j, C* v) {
    constexpr int R1 = StagePlan<N, E>::radix(0);
    constexpr int H = R1 / 2;
#pragma unroll
    for (int r = 0; r < H; ++r) {
      const int kz0 = j + r * (N / R1), kz1 = kz0 + N / 2;
      if (!valid) {
        v[r] = mk(T(0), T(0));
        v[r + H] = mk(T(0), T(0));
        continue;
      }
      if constexpr (SPEC == SPEC_SHINO) {
        v[r] = shino_mode<T>(a, kx, ky, kz0);
        v[r + H] = shino_mode<T>(a, kx, ky, kz1);
      } else {
        C x0, x1;
        if constexpr (SPEC == SPEC_INJECT) {
          x0 = static_cast<const C*>(a.xi)[mrow + mz * (uint64_t)kz0];
          x1 = static_cast<const C*>(a.xi)[mrow + mz * (uint64_t)kz1];
        } else {
          const uint64_t c = mrow + mz * (uint64_t)kz0;
          const u32x4 o = philox4x32_10_ks({(uint32_t)c, (uint32_t)(c >> 32), a.stream, 0u}, a.ks);
          x0 = Normals<T>::from(o.x, o.y);
          x1 = Normals<T>::from(o.z, o.w);
        }
        const T A0 = amp(kz0), A1 = amp(kz1);
        v[r] = mk(A0 * x0.x, A0 * x0.y);
        v[r + H] = mk(A1 * x1.x, A1 * x1.y);
      }
    }
  };
  const int Nz = a.Nout[2];
  constexpr int RL = last_radix<N, E>();
  const size_t zstride = (size_t)a.P[1] * a.Hpad;
  C* wcol = work + (size_t)ky * a.Hpad + kx;
  auto store = [&](int j, const C* o) {
    C* wj = wcol + (size_t)j * zstride;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int z = j + r * (N / RL);
      if (valid && z < Nz) wj[(size_t)(r * (N / RL)) * zstride] = o[r];
    }
  };
  line_ifft<C, N, E, SmemOrder::BatchFast, B, 0, false, 1>(sm, b, t, static_cast<const C*>(a.tw_z),
                                                          load, store);
}

// ---------------------------------------------------------------------------
// Pass 2: inverse DFT along y, in place, keep y < Ny.
// ---------------------------------------------------------------------------
// DIRECT: the first stage reads its inputs straight from global memory (no
// staged copy of the column block); every input is read before the line's
// last stage stores, which the plan's block barriers order (two or more
// stages).
template <typename T, int N, int E, int B, bool DIRECT = false>
__device__ __forceinline__ void mid_y_body(const GenArgs& a, int bx, int z) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int kx0 = bx * B;
  const int kx = kx0 + b;
  const bool valid = kx < a.Hx;
  C* colblk = static_cast<C*>(a.work) + (size_t)z * a.P[1] * a.Hpad + kx0;
  const size_t pitch = (size_t)a.Hpad;
  const int Ny = a.Nout[1];
  constexpr int RL = last_radix<N, E>();
  C* col = colblk + b;
  auto store = [&](int j, const C* o) {
    C* cj = col + (size_t)j * pitch;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int y = j + r * (N / RL);
      if (valid && y < Ny) cj[(size_t)(r * (N / RL)) * pitch] = o[r];
    }
  };
  if constexpr (DIRECT) {
    static_assert(StagePlan<N, E>::S >= 2, "direct loads need a barrier before the stores");
    const C* src = col;
    auto load = each_load<C, N, E>([&](int ky) -> C {
      return valid ? src[(size_t)ky * pitch] : mk(T(0), T(0));
    });
    line_ifft<C, N, E, SmemOrder::BatchFast, B, 0, false, 1>(sm, b, t, static_cast<const C*>(a.tw_y),
                                                            load, store);
  } else {
    {  // stage the N x B column block: raw[n * B + b], 16-byte async copies
      constexpr int CPR = B * (int)sizeof(C) / 16;  // chunks per row
      for (int c = threadIdx.x; c < N * CPR; c += blockDim.x) {
        const int n = c / CPR, q = c - n * CPR;
        cp_async16(reinterpret_cast<char*>(sm + n * B) + q * 16,
                   reinterpret_cast<const char*>(colblk + (size_t)n * pitch) + q * 16);
      }
      cp_async_wait_all();
      __syncthreads();
    }
    auto load = each_load<C, N, E>([&](int ky) -> C { return sm[ky * B + b]; });
    line_ifft<C, N, E, SmemOrder::BatchFast, B, 0, false, 1>(sm, b, t, static_cast<const C*>(a.tw_y),
                                                            load, store);
  }
}

// ---------------------------------------------------------------------------
// Pass 3: Hermitian C2R along x (complex length N = P0/2), crop, epilogue.
// ---------------------------------------------------------------------------
template <int N, int E> __host__ __device__ constexpr int c2r_line_stride() {
  return line_slots<N, E>() > N + 2 ? line_slots<N, E>() : N + 2;
}
// Shared memory of a pass-3 block: B staged lines, the twiddles
// e^{2 pi i m / P0} (m < P0 = 2N) and the x tables of the blend (s_x and the
// flags, Nx <= 2N entries each).
template <typename T, int N, int E, int B> __host__ __device__ constexpr size_t c2r_smem() {
  return (size_t)B * c2r_line_stride<N, E>() * sizeof(cplx_t<T>) + (size_t)2 * N * sizeof(cplx_t<T>) +
         (size_t)2 * N * sizeof(T) + (size_t)2 * N;
}

template <typename T, int N, int E, int B>
__device__ __forceinline__ void c2r_x_body(const GenArgs& a, int bx) {
  using C = cplx_t<T>;
  constexpr int TPL = N / E;
  constexpr int LS = c2r_line_stride<N, E>();
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  C* tws = sm + B * LS;                                   // 2N twiddles
  T* sxs = reinterpret_cast<T*>(tws + 2 * N);             // s_x, x < Nx
  uint8_t* fxs = reinterpret_cast<uint8_t*>(sxs + 2 * N);  // flags, x < Nx
  const int Nx = a.Nout[0], Ny = a.Nout[1], Nz = a.Nout[2];
  const int64_t nlines = (int64_t)Ny * Nz;
  const C* work = static_cast<const C*>(a.work);
  const int b = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const int l = bx * B + b;  // lines of a tile: Ny Nz <= 2048^2
  const bool valid = l < (int)nlines;
  const int y = valid ? l % Ny : 0, z = valid ? l / Ny : 0;
  const bool blend = a.epi.mode != 0;
  {  // the block's tables, then the raw half-spectrum line (N + 1 values, padded to 16 bytes)
    const C* twx = static_cast<const C*>(a.tw_x);
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) tws[i] = __ldg(twx + i);
    if (blend) {
      const T* sx = sw_of<T>(a.epi.ax[0]);
      const uint8_t* fx = a.epi.ax[0].flags;
      for (int i = threadIdx.x; i < Nx; i += blockDim.x) {
        sxs[i] = a.epi.apply_pou ? __ldg(sx + i) : T(1);
        fxs[i] = __ldg(fx + i);
      }
    }
    constexpr int CH = (N + 2) * (int)sizeof(C) / 16;
    const C* src = work + ((size_t)z * a.P[1] + (size_t)y) * a.Hpad;
    if (valid)
      for (int c = t; c < CH; c += TPL)
        cp_async16(reinterpret_cast<char*>(sm + b * LS) + c * 16, reinterpret_cast<const char*>(src) + c * 16);
    cp_async_wait_all();
    __syncthreads();
  }
  const C* line = sm + b * LS;
  auto load = each_load<C, N, E>([&](int k) -> C {
    const C xk = line[k], xn = line[N - k];
    if (k == 0) return mk(xk.x + xn.x, xk.x - xn.x);
    const C xc = cconj(xn);
    const C e = cadd(xk, xc);
    const C o = cmul(csub(xk, xc), tws[k]);
    return mk(e.x - o.y, e.y + o.x);
  });
  LineEpilogue<T> ep(a.epi, y, z, Nx, Ny);
  if (blend) {  // the x tables from shared memory
    ep.fx = fxs;
    ep.sx = sxs;
  }
  constexpr int RL = last_radix<N, E>();
  const bool mom = a.epi.mom != nullptr;
  double s1 = 0.0, s2 = 0.0;
  auto store = [&](int j, const C* o) {
    if (!valid) return;
    T v[2 * RL];
    int xs[2 * RL];
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int n = j + r * (N / RL);
      v[2 * r] = o[r].x;
      v[2 * r + 1] = o[r].y;
      xs[2 * r] = 2 * n;
      xs[2 * r + 1] = 2 * n + 1;
    }
    if (mom) ep.template put_group<2 * RL, true>(xs, v, Nx, &s1, &s2);
    else ep.template put_group<2 * RL>(xs, v, Nx);
  };
  line_ifft<C, N, E, SmemOrder::LineFast, B, LS, false, 2>(sm, b, t, tws, load, store);
  if (mom) {  // the block's FP64 partial sums of the final values, at mom[2 bx]
    __shared__ double red[2][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    const int w = (int)threadIdx.x >> 5, nw = ((int)blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) {
      red[0][w] = s1;
      red[1][w] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t1 = 0.0, t2 = 0.0;
      for (int i = 0; i < nw; ++i) {
        t1 += red[0][i];
        t2 += red[1][i];
      }
      a.epi.mom[2 * (int64_t)bx] = t1;
      a.epi.mom[2 * (int64_t)bx + 1] = t2;
    }
  }
}

// ---------------------------------------------------------------------------
// Kernels.  Single-tile launches take the argument block by value and use the
// grid coordinates directly; batched launches cover the blocks of several
// realisations of one line length with a flat grid, each block finding its
// realisation in the group's block-offset table.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int batch_item(const BatchMap& m, int* local) {
  const int blk = (int)blockIdx.x;
  int lo = 0, hi = m.n;  // start[lo] <= blk < start[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(m.start + mid) <= blk) lo = mid;
    else hi = mid;
  }
  *local = blk - __ldg(m.start + lo);
  return __ldg(m.items + lo);
}

template <typename T, int N, int E, int B, int SPEC>
__global__ void __launch_bounds__(B*(N / E)) k_gen_z(const GenArgs a) {
  gen_z_body<T, N, E, B, SPEC>(a, blockIdx.x, blockIdx.y);
}
template <typename T, int N, int E, int B, int SPEC>
__global__ void __launch_bounds__(B*(N / E)) k_gen_z_batch(const BatchMap m) {
  int loc;
  const GenArgs a = m.args[batch_item(m, &loc)];
  const int gx = (a.Hx + B - 1) / B;
  gen_z_body<T, N, E, B, SPEC>(a, loc % gx, loc / gx);
}

template <typename T, int N, int E, int B, bool DIRECT = false>
__global__ void __launch_bounds__(B*(N / E)) k_mid_y(const GenArgs a) {
  mid_y_body<T, N, E, B, DIRECT>(a, blockIdx.x, blockIdx.y);
}
template <typename T, int N, int E, int B, bool DIRECT = false>
__global__ void __launch_bounds__(B*(N / E)) k_mid_y_batch(const BatchMap m) {
  int loc;
  const GenArgs a = m.args[batch_item(m, &loc)];
  const int gx = (a.Hx + B - 1) / B;
  mid_y_body<T, N, E, B, DIRECT>(a, loc % gx, loc / gx);
}

template <typename T, int N, int E, int B>
__global__ void __launch_bounds__(B*(N / E)) k_c2r_x(const GenArgs a) {
  c2r_x_body<T, N, E, B>(a, blockIdx.x);
}
template <typename T, int N, int E, int B>
__global__ void __launch_bounds__(B*(N / E)) k_c2r_x_batch(const BatchMap m) {
  int loc;
  const GenArgs a = m.args[batch_item(m, &loc)];
  c2r_x_body<T, N, E, B>(a, loc);
}

}  // namespace scarl
