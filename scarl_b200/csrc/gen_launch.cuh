// gen_launch.cuh -- launch variants of the three generator passes.  Each
// variant fixes E (values per thread, hence the radix plan) and B (lines per
// block); the autotuner in api.cpp times the valid variants on the caller's
// grid and keeps the fastest per (precision, pass, line length).
#pragma once

#include <type_traits>

#include "c2r_shfl.cuh"
#include "gen_kernels.cuh"

namespace scarl {

struct VarEB {
  int E, B;
};

// passes 1 and 2 (lines strided in memory, lanes span lines)
template <typename T> struct ColVars;
template <> struct ColVars<float> {
  static constexpr int n = 6;
  static constexpr VarEB v[n] = {{16, 8}, {16, 4}, {16, 16}, {32, 4}, {32, 8}, {8, 16}};
};
template <> struct ColVars<double> {
  static constexpr int n = 4;
  static constexpr VarEB v[n] = {{16, 4}, {8, 8}, {8, 4}, {16, 8}};
};
// pass 2 with the first stage read straight from global memory (FP32)
struct ColDirectVars {
  static constexpr int n = 3;
  static constexpr VarEB v[n] = {{32, 8}, {16, 8}, {16, 16}};
};
template <typename T> constexpr int kDirectVars = std::is_same<T, float>::value ? ColDirectVars::n : 0;
// pass 3 (contiguous lines, lanes span a line)
template <typename T> struct RowVars;
template <> struct RowVars<float> {
  static constexpr int n = 5;
  static constexpr VarEB v[n] = {{16, 8}, {16, 4}, {32, 4}, {8, 8}, {32, 2}};
};
template <> struct RowVars<double> {
  static constexpr int n = 3;
  static constexpr VarEB v[n] = {{16, 4}, {8, 8}, {8, 4}};
};

// Every radix of the plan within the in-register DFTs (powers of two up to
// 32, or 3, 5, 7).
template <int N, int E> __host__ __device__ constexpr bool radices_ok() {
  for (int s = 0; s < StagePlan<N, E>::S; ++s)
    if (StagePlan<N, E>::radix(s) > 32) return false;
  return true;
}

// E: the effective values per thread (eff_E of the variant).
template <typename T, int N, int Ee, int B, bool ROW>
__host__ __device__ constexpr bool variant_ok() {
  if (!StagePlan<N, Ee>::valid() || !radices_ok<N, Ee>()) return false;
  constexpr int threads = B * (N / Ee);
  constexpr size_t smem = ROW ? c2r_smem<T, N, Ee, B>() : (size_t)B * line_slots<N, Ee>() * sizeof(cplx_t<T>);
  return threads >= 1 && threads <= 1024 && smem <= 220 * 1024 && (N % Ee) == 0;
}

template <typename K, typename A>
inline cudaError_t launch_k(K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            const A& a) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kernel<<<grid, block, smem, s>>>(a);
  return cudaGetLastError();
}

// Each run_*_v launches one variant: with bm == nullptr a single tile (grid
// from a), else the batched kernel over bm->total blocks.  With blocks != 0
// nothing is launched and *blocks receives the tile's block count.
template <typename T, int N, int E0, int B, int SPEC>
inline cudaError_t run_gen_z_v(const GenArgs& a, const BatchMap* bm, int* blocks, cudaStream_t s) {
  constexpr int E = eff_E<N, E0>();
  if constexpr (!variant_ok<T, N, E, B, false>()) {
    return cudaErrorInvalidConfiguration;
  } else {
    dim3 grid((a.Hx + B - 1) / B, a.P[1], 1);
    if (blocks) {
      *blocks = (int)(grid.x * grid.y);
      return cudaSuccess;
    }
    dim3 block(B * (N / E));
    size_t smem = (size_t)B * line_slots<N, E>() * sizeof(cplx_t<T>);
    if (bm) {
      if constexpr (SPEC == SPEC_PHILOX)
        return launch_k(k_gen_z_batch<T, N, E, B, SPEC>, dim3(bm->total), block, smem, s, *bm);
      return cudaErrorInvalidConfiguration;
    }
    return launch_k(k_gen_z<T, N, E, B, SPEC>, grid, block, smem, s, a);
  }
}

template <typename T, int N, int E0, int B, bool DIRECT = false>
inline cudaError_t run_mid_y_v(const GenArgs& a, const BatchMap* bm, int* blocks, cudaStream_t s) {
  constexpr int E = eff_E<N, E0>();
  if constexpr (!variant_ok<T, N, E, B, false>() || (DIRECT && StagePlan<N, E>::S < 2)) {
    return cudaErrorInvalidConfiguration;
  } else {
    dim3 grid((a.Hx + B - 1) / B, a.Nout[2], 1);
    if (blocks) {
      *blocks = (int)(grid.x * grid.y);
      return cudaSuccess;
    }
    dim3 block(B * (N / E));
    size_t smem = (size_t)B * line_slots<N, E>() * sizeof(cplx_t<T>);
    if (bm) return launch_k(k_mid_y_batch<T, N, E, B, DIRECT>, dim3(bm->total), block, smem, s, *bm);
    return launch_k(k_mid_y<T, N, E, B, DIRECT>, grid, block, smem, s, a);
  }
}

template <typename T, int N, int E0, int B>
inline cudaError_t run_c2r_x_v(const GenArgs& a, const BatchMap* bm, int* blocks, cudaStream_t s) {
  constexpr int E = eff_E<N, E0>();
  if constexpr (!variant_ok<T, N, E, B, true>()) {
    return cudaErrorInvalidConfiguration;
  } else {
    const int64_t nlines = (int64_t)a.Nout[1] * a.Nout[2];
    dim3 grid((unsigned)((nlines + B - 1) / B), 1, 1);
    if (blocks) {
      *blocks = (int)grid.x;
      return cudaSuccess;
    }
    dim3 block(B * (N / E));
    size_t smem = c2r_smem<T, N, E, B>();
    if (bm) return launch_k(k_c2r_x_batch<T, N, E, B>, dim3(bm->total), block, smem, s, *bm);
    return launch_k(k_c2r_x<T, N, E, B>, grid, block, smem, s, a);
  }
}

// Pass 3 with the line transform in registers and warp shuffles
// (c2r_shfl.cuh), L lanes a line, one group of lines a warp: FP32 only,
// needs the status word.  With blocks != nullptr nothing is launched and
// *blocks receives the block count (the FP64 moment pairs a single-tile
// launch writes: one a block).
template <typename T, int N, int L>
inline cudaError_t run_c2r_shfl(const GenArgs& a, const BatchMap* bm, int* blocks, cudaStream_t s) {
  using Cfg = ShflCfg<N, L>;
  if constexpr (!std::is_same<T, float>::value || !Cfg::valid()) {
    return cudaErrorInvalidConfiguration;
  } else {
    const int64_t nlines = (int64_t)a.Nout[1] * a.Nout[2];
    const int64_t per_block = (int64_t)Cfg::WPB * Cfg::G;
    dim3 grid((unsigned)((nlines + per_block - 1) / per_block), 1, 1);
    if (blocks) {
      *blocks = (int)grid.x;
      return cudaSuccess;
    }
    if (!a.status) return cudaErrorInvalidValue;
    if (bm)
      return launch_k(k_c2r_x_shfl_batch<N, L>, dim3(bm->total), dim3(Cfg::THREADS), Cfg::SMEM, s, *bm);
    return launch_k(k_c2r_x_shfl<N, L>, grid, dim3(Cfg::THREADS), Cfg::SMEM, s, a);
  }
}
// Pass-3 variants after the engine's (RowVars) ones: the register transform
// with 8, 16 and 32 lanes a line (FP32).
template <typename T> constexpr int kShflVars = std::is_same<T, float>::value ? 3 : 0;

// Variant v of pass `pass` for line length N (pass 3: N = P0/2).  Lengths
// below 128 (64 for pass 3) have only variant 0; SPEC_INJECT / SPEC_SHINO
// pass-1 kernels only variant 0.
template <typename T, int N>
inline cudaError_t run_pass_n(int pass, int v, const GenArgs& a, const BatchMap* bm, int* nb,
                              cudaStream_t s) {
  using CV = ColVars<T>;
  using RV = RowVars<T>;
  constexpr bool tuned_col = N >= 128;
  constexpr bool tuned_row = N >= 64;
#define SCARL_COLV(I)                                                                     \
  case I:                                                                                 \
    if constexpr (I < CV::n && tuned_col) {                                               \
      if (pass == 1)                                                                      \
        return run_gen_z_v<T, N, CV::v[I].E, CV::v[I].B, SPEC_PHILOX>(a, bm, nb, s);      \
      return run_mid_y_v<T, N, CV::v[I].E, CV::v[I].B>(a, bm, nb, s);                     \
    }                                                                                     \
    return cudaErrorInvalidConfiguration;
#define SCARL_ROWV(I)                                                                     \
  case I:                                                                                 \
    if constexpr (I < RV::n && tuned_row)                                                 \
      return run_c2r_x_v<T, N, RV::v[I].E, RV::v[I].B>(a, bm, nb, s);                     \
    return cudaErrorInvalidConfiguration;
  if (pass == 1 && a.spec != SPEC_PHILOX) {
    if (v != 0) return cudaErrorInvalidConfiguration;
    if (a.spec == SPEC_INJECT)
      return run_gen_z_v<T, N, CV::v[0].E, CV::v[0].B, SPEC_INJECT>(a, bm, nb, s);
    return run_gen_z_v<T, N, CV::v[0].E, CV::v[0].B, SPEC_SHINO>(a, bm, nb, s);
  }
  if (pass == 2 && v >= CV::n && v < CV::n + kDirectVars<T>) {
    if constexpr (tuned_col && kDirectVars<T> > 0) {
      using DV = ColDirectVars;
      if (v == CV::n) return run_mid_y_v<T, N, DV::v[0].E, DV::v[0].B, true>(a, bm, nb, s);
      if (v == CV::n + 1) return run_mid_y_v<T, N, DV::v[1].E, DV::v[1].B, true>(a, bm, nb, s);
      return run_mid_y_v<T, N, DV::v[2].E, DV::v[2].B, true>(a, bm, nb, s);
    }
    return cudaErrorInvalidConfiguration;
  }
  if (pass == 1 || pass == 2) {
    if (v == 0) {
      if (pass == 1) return run_gen_z_v<T, N, CV::v[0].E, CV::v[0].B, SPEC_PHILOX>(a, bm, nb, s);
      return run_mid_y_v<T, N, CV::v[0].E, CV::v[0].B>(a, bm, nb, s);
    }
    switch (v) {
      SCARL_COLV(1)
      SCARL_COLV(2)
      SCARL_COLV(3)
      SCARL_COLV(4)
      SCARL_COLV(5)
      default: return cudaErrorInvalidConfiguration;
    }
  }
  if (pass == 3) {
    if (v >= RV::n && v < RV::n + kShflVars<T>) {
      if (v == RV::n) return run_c2r_shfl<T, N, 8>(a, bm, nb, s);
      if (v == RV::n + 1) return run_c2r_shfl<T, N, 16>(a, bm, nb, s);
      return run_c2r_shfl<T, N, 32>(a, bm, nb, s);
    }
    if (v == 0) return run_c2r_x_v<T, N, RV::v[0].E, RV::v[0].B>(a, bm, nb, s);
    switch (v) {
      SCARL_ROWV(1)
      SCARL_ROWV(2)
      SCARL_ROWV(3)
      SCARL_ROWV(4)
      default: return cudaErrorInvalidConfiguration;
    }
  }
#undef SCARL_COLV
#undef SCARL_ROWV
  return cudaErrorInvalidValue;
}

}  // namespace scarl
