// fft_engine.cuh -- batched 1D inverse DFTs (sign +, unnormalised) of
// power-of-two length N inside one thread block.
//
// A block owns B lines of length N.  Each line is served by TPL = N/E
// threads holding E complex values in registers.  The transform is the
// Stockham autosort formulation (Govindaraju, Lloyd, Dotsenko, Smith,
// Manferdelli, "High performance discrete Fourier transforms on graphics
// processors", SC08): stage s with radix R reads x[j + r N/R], applies the
// twiddle w_{Ns R}^{r (j mod Ns)}, runs an R-point DFT in registers and
// writes x[(j/Ns) Ns R + (j mod Ns) + r Ns]; Ns grows by R every stage.
// The first stage reads straight from the caller's loader (global memory or
// an in-register generator) and the last stage hands each output to the
// caller's storer, so only the middle hand-offs touch shared memory.
#pragma once

#include "scarl_common.cuh"

namespace scarl {

// ---------------------------------------------------------------------------
// R-point inverse DFT in registers, R = 2..32: radix-2 decimation in
// frequency, result left in bit-reversed order (read it through brev<R>).
// ---------------------------------------------------------------------------
template <int R> __host__ __device__ constexpr int ilog2c() { return R <= 1 ? 0 : 1 + ilog2c<R / 2>(); }

template <int R> __host__ __device__ __forceinline__ constexpr int brev(int i) {
  int r = 0;
  for (int b = 0; b < ilog2c<R>(); ++b)
    if (i & (1 << b)) r |= 1 << (ilog2c<R>() - 1 - b);
  return r;
}

// d * e^{+2 pi i m / 32}, m < 16, m known after unrolling.
template <typename C> __device__ __forceinline__ C tw32(C d, int m) {
  using T = decltype(d.x);
  if (m == 0) return d;
  if (m == 8) return cmul_i(d);
  if (m == 4 || m == 12) {
    const T h = (T)0.70710678118654752440;
    // (1+i)/sqrt2 or (-1+i)/sqrt2
    return (m == 4) ? mk((d.x - d.y) * h, (d.x + d.y) * h) : mk((-d.x - d.y) * h, (d.x - d.y) * h);
  }
  const T c = (T)kCos32[m], s = (T)kSin32[m];
  return mk(d.x * c - d.y * s, d.x * s + d.y * c);
}

template <int R, typename C> __device__ __forceinline__ void dft_reg(C* v) {
#pragma unroll
  for (int len = R; len >= 2; len >>= 1) {
    const int half = len >> 1;
#pragma unroll
    for (int s = 0; s < R; s += len) {
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const C a = v[s + k], b = v[s + k + half];
        v[s + k] = cadd(a, b);
        v[s + k + half] = tw32(csub(a, b), k * (32 / len));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Stage plan for N = 2^n with at most E values per thread.
// ---------------------------------------------------------------------------
template <int N, int E> struct StagePlan {
  __host__ __device__ static constexpr int radix(int s) {
    int rem = N;
    for (int i = 0; i < s; ++i) rem /= (rem > E ? E : rem);
    return rem > E ? E : rem;
  }
  __host__ __device__ static constexpr int count() {
    int rem = N, c = 0;
    while (rem > 1) { rem /= (rem > E ? E : rem); ++c; }
    return c;
  }
  static constexpr int S = count();
};

// Shared-memory addressing of line element n of line b, skewed by one slot
// per SK elements (SK = first radix) so the first stage's stride-SK writes
// fall in distinct banks:
//   BatchFast: element (n, b) at p(n)*B + b  (lanes of a warp span lines)
//   LineFast : element (n, b) at b*LS + p(n) (lanes of a warp span a line)
// with p(n) = n + n / SK.  A line occupies N + N/SK slots.
enum class SmemOrder { BatchFast, LineFast };

template <int N, int SK> __host__ __device__ constexpr int skewed_len() { return N + N / SK; }

template <SmemOrder O, int B, int LS, int SK> __device__ __forceinline__ int sidx(int n, int b) {
  const int p = n + n / SK;
  return O == SmemOrder::BatchFast ? p * B + b : b * LS + p;
}

// One Stockham stage reading/writing shared memory (middle stages).
// tw: e^{+2 pi i m / (N * twmul)} table, so w_{Ns R}^{q} = tw[q * (N / (Ns R)) * twmul].
template <typename C, int N, int E, int R, int Ns, SmemOrder O, int B, int LS, int SK>
__device__ __forceinline__ void stockham_smem_stage(C* __restrict__ sm, int b, int t,
                                                    const C* __restrict__ tw, int twmul) {
  constexpr int TPL = N / E;
  constexpr int NB = E / R;  // butterflies per thread
  C v[E];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = t + TPL * q;
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = sm[sidx<O, B, LS, SK>(j + r * (N / R), b)];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = t + TPL * q;
    const int k = j % Ns;
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const C w = __ldg(reinterpret_cast<const C*>(tw) + (size_t)(r * k) * (N / (Ns * R)) * twmul);
      v[q * R + r] = cmul(v[q * R + r], w);
    }
    dft_reg<R>(v + q * R);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) sm[sidx<O, B, LS, SK>(base + r * Ns, b)] = v[q * R + brev<R>(r)];
  }
  __syncthreads();
}

// Full line transform.  load(j, v) fills the first stage's R1 inputs
// v[r] = x[j + r N/R1] (r < R1, R1 = StagePlan<N,E>::radix(0)); store(j, v)
// takes the last stage's RL outputs v[r] = y[j + r N/RL] together, so a
// caller can issue all its memory reads for them before its writes.  sm holds
// B lines laid out by O with skew SK = R1 (line stride LS for LineFast).  All
// threads of the block must call.  With SYNC_STORE every thread has finished
// its shared-memory reads before the first store, so store may write sm.
template <typename C, int N, int E, SmemOrder O, int B, int LS, bool SYNC_STORE = false,
          class Load, class Store>
__device__ __forceinline__ void line_ifft(C* __restrict__ sm, int b, int t, const C* __restrict__ tw,
                                          int twmul, Load&& load, Store&& store) {
  using P = StagePlan<N, E>;
  constexpr int TPL = N / E;
  constexpr int R1 = P::radix(0);
  constexpr int SK = R1;
  constexpr int NB1 = E / R1;
  C v[E];
#pragma unroll
  for (int q = 0; q < NB1; ++q) load(t + TPL * q, v + q * R1);
  if constexpr (P::S == 1) {
#pragma unroll
    for (int q = 0; q < NB1; ++q) {
      const int j = t + TPL * q;
      dft_reg<R1>(v + q * R1);
      C o[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) o[r] = v[q * R1 + brev<R1>(r)];
      store(j, o);
    }
    __syncthreads();  // keep the barrier count uniform with the multi-stage path
  } else {
    // first stage: Ns = 1, no twiddles; output index j*R1 + r
#pragma unroll
    for (int q = 0; q < NB1; ++q) dft_reg<R1>(v + q * R1);
    __syncthreads();  // the loader may have read shared memory
#pragma unroll
    for (int q = 0; q < NB1; ++q) {
      const int j = t + TPL * q;
#pragma unroll
      for (int r = 0; r < R1; ++r) sm[sidx<O, B, LS, SK>(j * R1 + r, b)] = v[q * R1 + brev<R1>(r)];
    }
    __syncthreads();
    if constexpr (P::S >= 3)
      stockham_smem_stage<C, N, E, P::radix(1), R1, O, B, LS, SK>(sm, b, t, tw, twmul);
    if constexpr (P::S >= 4)
      stockham_smem_stage<C, N, E, P::radix(2), R1 * P::radix(1), O, B, LS, SK>(sm, b, t, tw, twmul);
    static_assert(P::S <= 4, "line length too long for the register budget");
    // last stage
    constexpr int RL = P::radix(P::S - 1);
    constexpr int NsL = N / RL;
    constexpr int NBL = E / RL;
#pragma unroll
    for (int q = 0; q < NBL; ++q) {
      const int j = t + TPL * q;
#pragma unroll
      for (int r = 0; r < RL; ++r) v[q * RL + r] = sm[sidx<O, B, LS, SK>(j + r * (N / RL), b)];
    }
    if constexpr (SYNC_STORE) __syncthreads();
#pragma unroll
    for (int q = 0; q < NBL; ++q) {
      const int j = t + TPL * q;
      const int k = j % NsL;
#pragma unroll
      for (int r = 1; r < RL; ++r) {
        const C w = __ldg(reinterpret_cast<const C*>(tw) + (size_t)(r * k) * twmul);
        v[q * RL + r] = cmul(v[q * RL + r], w);
      }
      dft_reg<RL>(v + q * RL);
      // last stage: (j / NsL) == 0, output index j + r * NsL
      C o[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) o[r] = v[q * RL + brev<RL>(r)];
      store(j, o);
    }
  }
}

// Shared-memory slots of one line for a block using line_ifft<.., N, E, ..>.
template <int N, int E> __host__ __device__ constexpr int line_slots() {
  return skewed_len<N, StagePlan<N, E>::radix(0)>();
}

// Radix of the last stage (outputs per store group).
template <int N, int E> __host__ __device__ constexpr int last_radix() {
  return StagePlan<N, E>::radix(StagePlan<N, E>::S - 1);
}

// Asynchronous 16-byte global -> shared copy (cp.async, L2 only).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Adapts a per-element loader f(n) -> C to the group interface of line_ifft.
template <typename C, int N, int E, class F>
struct EachLoad {
  F f;
  __device__ __forceinline__ void operator()(int j, C* v) const {
    constexpr int R1 = StagePlan<N, E>::radix(0);
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = f(j + r * (N / R1));
  }
};
template <typename C, int N, int E, class F>
__device__ __forceinline__ EachLoad<C, N, E, F> each_load(F f) {
  return EachLoad<C, N, E, F>{f};
}

}  // namespace scarl
