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

template <typename T>
__device__ __forceinline__ void epilogue_point(const Epilogue& e, int x, int y, int z, int Nx,
                                               int Ny, T v) {
  if (e.mode == 0) {
    static_cast<T*>(e.out)[(size_t)x + (size_t)Nx * ((size_t)y + (size_t)Ny * z)] = marginal_apply(e, v);
    return;
  }
  const uint8_t f = e.ax[0].flags[x] & e.ax[1].flags[y] & e.ax[2].flags[z];
  if (!(f & 1)) return;
  if (e.apply_pou) {
    double w = e.ax[0].lo[x];
    w = __dmul_rn(w, e.ax[1].lo[y]);
    w = __dmul_rn(w, e.ax[2].lo[z]);
    w = __dmul_rn(w, e.ax[0].hi[x]);
    w = __dmul_rn(w, e.ax[1].hi[y]);
    w = __dmul_rn(w, e.ax[2].hi[z]);
    if (w != 1.0) v = (T)((double)v * sqrt(w));
  }
  const size_t g = (size_t)(e.off[0] + x) +
                   (size_t)e.L[0] * ((size_t)(e.off[1] + y) + (size_t)e.L[1] * (size_t)(e.off[2] + z));
  T* o = static_cast<T*>(e.out);
  if (!(f & 2)) v = o[g] + v;
  if (f & 4) v = marginal_apply(e, v);
  o[g] = v;
}

}  // namespace scarl
