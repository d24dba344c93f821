// fft_engine.cuh -- batched 1D inverse DFTs (sign +, unnormalised) of
// length N = m 2^a (m = 1, 3, 5 or 7) inside one thread block.
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
// caller's storer, so only the middle hand-offs touch shared memory.  The
// power-of-two radices come first (the first radix is even, so a first-stage
// group holds the modes k and k + N/2 together); an odd factor m is the last
// stage, a direct DFT in registers.
#pragma once

#include "scarl_common.cuh"

namespace scarl {

// ---------------------------------------------------------------------------
// R-point inverse DFT in registers.  R = 2..32 (power of two): radix-2
// decimation in frequency, result left in bit-reversed order; R = 3, 5, 7:
// direct sums over the conjugate-symmetric pairs, result in natural order.
// operm<R>(r) is the register holding output r.
// ---------------------------------------------------------------------------
template <int R> __host__ __device__ constexpr int ilog2c() { return R <= 1 ? 0 : 1 + ilog2c<R / 2>(); }
__host__ __device__ constexpr bool is_pow2c(int n) { return n >= 1 && (n & (n - 1)) == 0; }
__host__ __device__ constexpr int odd_part(int n) { return (n > 0 && n % 2 == 0) ? odd_part(n / 2) : n; }

template <int R> __host__ __device__ __forceinline__ constexpr int brev(int i) {
  int r = 0;
  for (int b = 0; b < ilog2c<R>(); ++b)
    if (i & (1 << b)) r |= 1 << (ilog2c<R>() - 1 - b);
  return r;
}
template <int R> __host__ __device__ __forceinline__ constexpr int operm(int i) {
  if constexpr (is_pow2c(R)) return brev<R>(i);
  else return i;
}

// cos and sin of 2 pi j / p, j = 1 .. (p - 1) / 2, for p = 3, 5, 7.
__device__ constexpr double kOddCos[3][3] = {
    {-0.5000000000000000000000, 0.0, 0.0},
    {0.3090169943749474241023, -0.8090169943749474241023, 0.0},
    {0.6234898018587335305250, -0.2225209339563144042889, -0.9009688679024191262361}};
__device__ constexpr double kOddSin[3][3] = {
    {0.8660254037844386467637, 0.0, 0.0},
    {0.9510565162951535721164, 0.5877852522924731291687, 0.0},
    {0.7818314824680298087084, 0.9749279121818236070181, 0.4338837391175581204758}};

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

// X_k = sum_n v_n e^{+2 pi i n k / P}, P odd: with s_n = v_n + v_{P-n},
// d_n = v_n - v_{P-n}, X_0 = v_0 + sum s_n and, for k = 1 .. (P-1)/2,
// X_k = A_k + i B_k, X_{P-k} = A_k - i B_k, A_k = v_0 + sum_n s_n cos(2 pi n k / P),
// B_k = sum_n d_n sin(2 pi n k / P).
template <int P, typename C> __device__ __forceinline__ void dft_odd(C* v) {
  using T = decltype(v[0].x);
  constexpr int H = (P - 1) / 2, row = P / 2 - 1;  // table row of P = 3, 5, 7
  C sp[H], dm[H];
#pragma unroll
  for (int n = 1; n <= H; ++n) {
    sp[n - 1] = cadd(v[n], v[P - n]);
    dm[n - 1] = csub(v[n], v[P - n]);
  }
  C x0 = v[0];
#pragma unroll
  for (int n = 0; n < H; ++n) x0 = cadd(x0, sp[n]);
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    C a = v[0], b = mk(T(0), T(0));
#pragma unroll
    for (int n = 1; n <= H; ++n) {
      const int j = (n * k) % P;  // angle index, folded into 1 .. H with the sine's sign
      const int jj = j <= H ? j : P - j;
      const T c = (T)kOddCos[row][jj - 1];
      const T sn = (j <= H) ? (T)kOddSin[row][jj - 1] : -(T)kOddSin[row][jj - 1];
      a = mk(a.x + sp[n - 1].x * c, a.y + sp[n - 1].y * c);
      b = mk(b.x + dm[n - 1].x * sn, b.y + dm[n - 1].y * sn);
    }
    v[k] = mk(a.x - b.y, a.y + b.x);
    v[P - k] = mk(a.x + b.y, a.y - b.x);
  }
  v[0] = x0;
}

template <int R, typename C> __device__ __forceinline__ void dft_reg(C* v) {
  if constexpr (!is_pow2c(R)) {
    static_assert(R == 3 || R == 5 || R == 7, "odd radix 3, 5 or 7");
    dft_odd<R>(v);
  } else {
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
}

// ---------------------------------------------------------------------------
// Stage plan for N = m 2^a with E values per thread: power-of-two radices of
// at most the largest power of two dividing E, then the odd factor m as the
// last stage (m must divide E).  At most 5 stages.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int pow2_of(int e) { return (e % 2 == 0) ? 2 * pow2_of(e / 2) : 1; }

template <int N, int E> struct StagePlan {
  static constexpr int M = odd_part(N), P2 = N / M, E2 = pow2_of(E);
  __host__ __device__ static constexpr int p2_count() {
    int rem = P2, c = 0;
    while (rem > 1) { rem /= (rem > E2 ? E2 : rem); ++c; }
    return c;
  }
  __host__ __device__ static constexpr int radix(int s) {
    if (M > 1 && s == p2_count()) return M;
    int rem = P2;
    for (int i = 0; i < s; ++i) rem /= (rem > E2 ? E2 : rem);
    return rem > E2 ? E2 : rem;
  }
  __host__ __device__ static constexpr int count() { return p2_count() + (M > 1 ? 1 : 0); }
  // a plan the engine can run: every radix divides E, 2 <= stages <= 5 (or
  // one power-of-two stage), first radix even
  __host__ __device__ static constexpr bool valid() {
    return (M == 1 || M == 3 || M == 5 || M == 7) && E % M == 0 && N % E == 0 && count() <= 5 &&
           (M == 1 || P2 >= 2) && (count() >= 2 || M == 1);
  }
  static constexpr int S = count();
};

// Power-of-two stages of a 2^a length with radices of at most e2.
__host__ __device__ constexpr int p2_stages(int p2, int e2) {
  return p2 > 1 ? 1 + p2_stages(p2 / (p2 > e2 ? e2 : p2), e2) : 0;
}
__host__ __device__ constexpr int grow_e2(int p2, int e2) {
  return (e2 < p2 && p2_stages(p2, e2) + 1 > 5) ? grow_e2(p2, 2 * e2) : e2;
}
// Values per thread of a launch variant: E itself for power-of-two lengths;
// for N = m 2^a (m odd) m e2 with e2 >= E / 4 the smallest power of two whose
// plan (power-of-two stages, then the radix-m stage) has at most 5 stages.
template <int N, int E> __host__ __device__ constexpr int eff_E() {
  constexpr int m = odd_part(N);
  if constexpr (m == 1) {
    return E < N ? E : N;
  } else {
    constexpr int p2 = N / m;
    constexpr int e0 = (E / 4 < 2 ? 2 : E / 4) > p2 ? p2 : (E / 4 < 2 ? 2 : E / 4);
    return m * grow_e2(p2, e0);
  }
}

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
// Slot distance of one step of p along the layout (B lines apart in
// BatchFast order, adjacent in LineFast order).
template <SmemOrder O, int B> __host__ __device__ constexpr int sstep() {
  return O == SmemOrder::BatchFast ? B : 1;
}
// Where m is a multiple of SK, p(n + m) = p(n) + m + m / SK: a thread's
// accesses at n0 + c (c a compile-time multiple of SK) are one base address
// plus compile-time offsets (immediate offsets of the shared-memory loads).
template <int SK> __host__ __device__ constexpr int skew_span(int m) { return m + m / SK; }

// One Stockham stage reading/writing shared memory (middle stages).
// tw: e^{+2 pi i m / (N * TWMUL)} table, so w_{Ns R}^{q} = tw[q * (N / (Ns R)) * TWMUL];
// it may live in global or shared memory (plain loads, no read-only-cache path).
template <typename C, int N, int E, int R, int Ns, SmemOrder O, int B, int LS, int SK, int TWMUL>
__device__ __forceinline__ void stockham_smem_stage(C* __restrict__ sm, int b, int t,
                                                    const C* __restrict__ tw) {
  constexpr int TPL = N / E;
  constexpr int NB = E / R;  // butterflies per thread
  constexpr int ST = sstep<O, B>();
  C v[E];
  if constexpr ((N / R) % SK == 0 && TPL % SK == 0) {
    // reads at j + r N/R, j = t + TPL q: base of t plus constant offsets
    const int a0 = sidx<O, B, LS, SK>(t, b);
#pragma unroll
    for (int q = 0; q < NB; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r)
        v[q * R + r] = sm[a0 + (skew_span<SK>(TPL * q) + skew_span<SK>(r * (N / R))) * ST];
  } else {
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int j = t + TPL * q;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = sm[sidx<O, B, LS, SK>(j + r * (N / R), b)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int j = t + TPL * q;
    const int k = j % Ns;
    const int tk = k * ((N / (Ns * R)) * TWMUL);
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const C w = tw[r * tk];  // global or shared table
      v[q * R + r] = cmul(v[q * R + r], w);
    }
    dft_reg<R>(v + q * R);
    const int base = (j / Ns) * Ns * R + k;
    if constexpr (Ns % SK == 0) {
      // writes at base + r Ns
      const int a0 = sidx<O, B, LS, SK>(base, b);
#pragma unroll
      for (int r = 0; r < R; ++r) sm[a0 + skew_span<SK>(r * Ns) * ST] = v[q * R + operm<R>(r)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) sm[sidx<O, B, LS, SK>(base + r * Ns, b)] = v[q * R + operm<R>(r)];
    }
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
          int TWMUL = 1, class Load, class Store>
__device__ __forceinline__ void line_ifft(C* __restrict__ sm, int b, int t, const C* __restrict__ tw,
                                          Load&& load, Store&& store) {
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
      for (int r = 0; r < R1; ++r) o[r] = v[q * R1 + operm<R1>(r)];
      store(j, o);
    }
    __syncthreads();  // keep the barrier count uniform with the multi-stage path
  } else {
    // first stage: Ns = 1, no twiddles; output index j*R1 + r
#pragma unroll
    for (int q = 0; q < NB1; ++q) dft_reg<R1>(v + q * R1);
    __syncthreads();  // the loader may have read shared memory
    constexpr int ST = sstep<O, B>();
    {
      // output j R1 + r of the first stage (r < R1 = SK) sits at slot p = j (R1 + 1) + r
      const int a0 = sidx<O, B, LS, SK>(t * R1, b);
#pragma unroll
      for (int q = 0; q < NB1; ++q)
#pragma unroll
        for (int r = 0; r < R1; ++r)
          sm[a0 + (TPL * q * (R1 + 1) + r) * ST] = v[q * R1 + operm<R1>(r)];
    }
    __syncthreads();
    if constexpr (P::S >= 3)
      stockham_smem_stage<C, N, E, P::radix(1), R1, O, B, LS, SK, TWMUL>(sm, b, t, tw);
    if constexpr (P::S >= 4)
      stockham_smem_stage<C, N, E, P::radix(2), R1 * P::radix(1), O, B, LS, SK, TWMUL>(sm, b, t, tw);
    if constexpr (P::S >= 5)
      stockham_smem_stage<C, N, E, P::radix(3), R1 * P::radix(1) * P::radix(2), O, B, LS, SK, TWMUL>(
          sm, b, t, tw);
    static_assert(P::S <= 5, "line length too long for the register budget");
    // last stage
    constexpr int RL = P::radix(P::S - 1);
    constexpr int NsL = N / RL;
    constexpr int NBL = E / RL;
    if constexpr ((N / RL) % SK == 0 && TPL % SK == 0) {
      const int a0 = sidx<O, B, LS, SK>(t, b);
#pragma unroll
      for (int q = 0; q < NBL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r)
          v[q * RL + r] = sm[a0 + (skew_span<SK>(TPL * q) + skew_span<SK>(r * (N / RL))) * ST];
    } else {
#pragma unroll
      for (int q = 0; q < NBL; ++q) {
        const int j = t + TPL * q;
#pragma unroll
        for (int r = 0; r < RL; ++r) v[q * RL + r] = sm[sidx<O, B, LS, SK>(j + r * (N / RL), b)];
      }
    }
    if constexpr (SYNC_STORE) __syncthreads();
#pragma unroll
    for (int q = 0; q < NBL; ++q) {
      const int j = t + TPL * q;
      const int k = j % NsL;
      const int tk = k * TWMUL;
#pragma unroll
      for (int r = 1; r < RL; ++r) {
        const C w = tw[r * tk];
        v[q * RL + r] = cmul(v[q * RL + r], w);
      }
      dft_reg<RL>(v + q * RL);
      // last stage: (j / NsL) == 0, output index j + r * NsL
      C o[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) o[r] = v[q * RL + operm<RL>(r)];
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
