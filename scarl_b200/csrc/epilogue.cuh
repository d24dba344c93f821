// epilogue.cuh -- per-point output stage shared by the C2R pass and the
// tile-blend kernel: plain crop, or partition-of-unity blend into the global
// field (SRC_F/main_ScaRL.f90:1216-1301 weights, 984-1210 overlap sum,
// write_output.f90:373-431 assembly) with the marginal transform
// (SRC_F/main_ScaRL.f90:1355-1395) applied by the tile that finishes a point.
#pragma once

#include "scarl_common.cuh"
#include "scarl_internal.h"

namespace scarl {

// ---------------------------------------------------------------------------
// Epilogue of one output point of a tile.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T marginal_apply(const Epilogue& e, T v) {
  if (e.marginal == 1) return v * (T)e.ms + (T)e.mmu;
  if (e.marginal == 2) return exp(v * (T)e.ms + (T)e.mmu);
  return v;
}

template <typename T> __device__ __forceinline__ const T* sw_of(const BlendAxis& a);
template <> __device__ __forceinline__ const float* sw_of<float>(const BlendAxis& a) { return a.sw32; }
template <> __device__ __forceinline__ const double* sw_of<double>(const BlendAxis& a) { return a.sw64; }

// Output stage of one tile line (fixed y, z; x varies).  In blend mode the
// partition-of-unity factor is the product of the per-axis sqrt factors,
// sqrt(w) = s_x s_y s_z, with s_d = sqrt(lo_d hi_d) computed in FP64 on the
// host (equal to sqrt of the reference's product up to rounding).
template <typename T>
struct LineEpilogue {
  T* out;
  size_t base;        // output index of x = 0
  uint8_t fyz;        // flags of y and z, AND-ed
  T syz;              // s_y s_z
  const uint8_t* fx;  // flags along x (blend)
  const T* sx;        // s_x (blend)
  int mode, marginal, pou;
  T ms, mu;

  __device__ __forceinline__ LineEpilogue(const Epilogue& e, int y, int z, int Nx, int Ny) {
    out = static_cast<T*>(e.out);
    mode = e.mode;
    marginal = e.marginal;
    ms = (T)e.ms;
    mu = (T)e.mmu;
    pou = e.apply_pou;
    if (mode == 0) {
      base = (size_t)Nx * ((size_t)y + (size_t)Ny * z);
      fyz = 7;
      syz = T(1);
      fx = nullptr;
      sx = nullptr;
    } else {
      base = (size_t)e.off[0] + (size_t)e.L[0] * ((size_t)(e.off[1] + y) + (size_t)e.L[1] * (size_t)(e.off[2] + z));
      fyz = e.ax[1].flags[y] & e.ax[2].flags[z];
      syz = pou ? sw_of<T>(e.ax[1])[y] * sw_of<T>(e.ax[2])[z] : T(1);
      fx = e.ax[0].flags;
      sx = sw_of<T>(e.ax[0]);
    }
  }
  // The same epilogue from a line's precomputed base, y-z flags and s_y s_z
  // (the values the constructor above derives) and the x tables fx, sx.
  __device__ __forceinline__ LineEpilogue(const Epilogue& e, size_t base_, uint8_t fyz_, T syz_,
                                          const uint8_t* fx_, const T* sx_) {
    out = static_cast<T*>(e.out);
    mode = e.mode;
    marginal = e.marginal;
    ms = (T)e.ms;
    mu = (T)e.mmu;
    pou = e.apply_pou;
    base = base_;
    fyz = fyz_;
    syz = syz_;
    fx = fx_;
    sx = sx_;
  }
  // lognormal in FP32 with the hardware exponential (relative error a few
  // 2^-23, far inside the FP32 field's 1e-5 tolerance); FP64 keeps exp
  __device__ __forceinline__ T marg(T v) const {
    if (marginal == 1) return v * ms + mu;
    if (marginal == 2) {
      if constexpr (sizeof(T) == 4) return __expf(v * ms + mu);
      else return exp(v * ms + mu);
    }
    return v;
  }
  // K outputs at once: every read of an earlier tile's partial sum is issued
  // before any write.  With MOM, every final value w (a crop point, or a
  // blended point whose last tile this is) is added to *s1 and w^2 to *s2 in
  // FP64.
  template <int K, bool MOM = false>
  __device__ __forceinline__ void put_group(const int* xs, const T* v, int Nx, double* s1 = nullptr,
                                            double* s2 = nullptr) const {
    if (mode == 0) {
#pragma unroll
      for (int i = 0; i < K; ++i)
        if (xs[i] < Nx) {
          const T w = marg(v[i]);
          out[base + xs[i]] = w;
          if constexpr (MOM) {
            *s1 += (double)w;
            *s2 = fma((double)w, (double)w, *s2);
          }
        }
      return;
    }
    uint8_t f[K];
    T old[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      f[i] = xs[i] < Nx ? (uint8_t)(fyz & fx[xs[i]]) : (uint8_t)0;
      old[i] = ((f[i] & 3) == 1) ? out[base + xs[i]] : T(0);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!(f[i] & 1)) continue;
      T w = pou ? v[i] * (syz * sx[xs[i]]) : v[i];
      if (!(f[i] & 2)) w = old[i] + w;
      if (f[i] & 4) {
        w = marg(w);
        if constexpr (MOM) {
          *s1 += (double)w;
          *s2 = fma((double)w, (double)w, *s2);
        }
      }
      out[base + xs[i]] = w;
    }
  }
  // put_group through one line pointer (out + base), each access a 32-bit
  // offset from it.
  template <int K, bool MOM = false>
  __device__ __forceinline__ void put_group_line(const int* xs, const T* v, int Nx, double* s1 = nullptr,
                                                 double* s2 = nullptr) const {
    T* o = out + base;
    if (mode == 0) {
#pragma unroll
      for (int i = 0; i < K; ++i)
        if (xs[i] < Nx) {
          const T w = marg(v[i]);
          o[xs[i]] = w;
          if constexpr (MOM) {
            *s1 += (double)w;
            *s2 = fma((double)w, (double)w, *s2);
          }
        }
      return;
    }
    uint8_t f[K];
    T old[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      f[i] = xs[i] < Nx ? (uint8_t)(fyz & fx[xs[i]]) : (uint8_t)0;
      old[i] = ((f[i] & 3) == 1) ? o[xs[i]] : T(0);
    }
#pragma unroll
    for (int i = 0; i < K; ++i) {
      if (!(f[i] & 1)) continue;
      T w = pou ? v[i] * (syz * sx[xs[i]]) : v[i];
      if (!(f[i] & 2)) w = old[i] + w;
      if (f[i] & 4) {
        w = marg(w);
        if constexpr (MOM) {
          *s1 += (double)w;
          *s2 = fma((double)w, (double)w, *s2);
        }
      }
      o[xs[i]] = w;
    }
  }
  __device__ __forceinline__ void put(int x, T v) const {
    if (mode == 0) {
      out[base + x] = marg(v);
      return;
    }
    const uint8_t f = fyz & fx[x];
    if (!(f & 1)) return;
    if (pou) v = v * (syz * sx[x]);
    if (!(f & 2)) v = out[base + x] + v;
    if (f & 4) v = marg(v);
    out[base + x] = v;
  }
};

template <typename T>
__device__ __forceinline__ void epilogue_point(const Epilogue& e, int x, int y, int z, int Nx,
                                               int Ny, T v) {
  LineEpilogue<T>(e, y, z, Nx, Ny).put(x, v);
}

}  // namespace scarl
