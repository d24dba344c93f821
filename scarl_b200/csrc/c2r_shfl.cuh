// c2r_shfl.cuh -- pass 3 of the padded generator (Hermitian C2R along x, crop,
// blend epilogue) with each line's transform held in registers.
//
// A line of N = N2 * L complex half-spectrum values is served by L lanes of
// one warp (G = 32 / L lines per warp).  With k = k1 + L k2 (lane k1 < L,
// register k2 < N2) and n = n2 + N2 n1:
//   stage A  Y[k1][n2] = sum_k2 z[k1 + L k2] e^{+2 pi i n2 k2 / N2}   (registers)
//   twiddle  Y'       = Y e^{+2 pi i n2 k1 / N}
//   stage B  y[n2 + N2 n1] = sum_k1 Y'[k1][n2] e^{+2 pi i n1 k1 / L}  (across lanes)
// Stage B is a radix-2 decimation-in-frequency transform over the L lanes of
// the line, one butterfly level per __shfl_xor_sync span (L/2, ..., 1); lane
// k1 ends with outputs n1 = bitrev(k1).  No shared-memory hand-off and no
// block barrier sits inside the transform.
//
// The raw line (N + 1 values, rows of the pass-2 output) is staged in shared
// memory by bulk asynchronous copies (cp.async.bulk, one per line, completion
// on a per-warp mbarrier) issued by lane 0 of the warp; z = the C2R
// pre-combination of X[k] and conj X[N - k] (the same arithmetic as the
// engine's pass 3).  The outputs go back to the line's shared slot and the
// epilogue runs with consecutive lanes on consecutive x (coalesced stores,
// read-modify-writes and table reads).
#pragma once

#include "gen_kernels.cuh"
#include "tc_sm100.cuh"

namespace scarl {

// ---------------------------------------------------------------------------
// Compile-time unit roots: cos and sin of 2 pi j / n in double, from Taylor
// series on |x| <= pi/4 after an exact integer reduction to the first octant.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr double cx_sin_oct(double x) {
  double term = x, sum = x;
  for (int i = 1; i < 14; ++i) {
    term *= -x * x / (double)((2 * i) * (2 * i + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double cx_cos_oct(double x) {
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 14; ++i) {
    term *= -x * x / (double)((2 * i - 1) * (2 * i));
    sum += term;
  }
  return sum;
}
// (cos, sin)(2 pi j / n): quadrant q = floor(4 j / n), remainder angle
// r = 2 pi num / (4 n) with num = 4 j - q n in [0, n); r > pi / 4 uses the
// complement 2 pi (n - num) / (4 n).
__host__ __device__ constexpr void cx_root(long long j, long long n, double& c, double& s) {
  constexpr double kTwoPi = 6.283185307179586476925286766559;
  j %= n;
  if (j < 0) j += n;
  const long long q = (4 * j) / n, num = 4 * j - q * n;
  double c0 = 0.0, s0 = 0.0;
  if (2 * num <= n) {
    const double x = kTwoPi * (double)num / (double)(4 * n);
    c0 = cx_cos_oct(x);
    s0 = cx_sin_oct(x);
  } else {
    const double x = kTwoPi * (double)(n - num) / (double)(4 * n);
    c0 = cx_sin_oct(x);
    s0 = cx_cos_oct(x);
  }
  if (q == 0) { c = c0; s = s0; }
  else if (q == 1) { c = -s0; s = c0; }
  else if (q == 2) { c = -c0; s = -s0; }
  else { c = s0; s = -c0; }
}

template <int N> struct RootTable {
  float c[N], s[N];
  constexpr RootTable() : c(), s() {
    for (int j = 0; j < N; ++j) {
      double cc = 0.0, ss = 0.0;
      cx_root(j, N, cc, ss);
      c[j] = (float)cc;
      s[j] = (float)ss;
    }
  }
};
template <int N> __device__ constexpr RootTable<N> kRootTable = RootTable<N>();

// ---------------------------------------------------------------------------
// In-register inverse DFT of N2 = P Q points (P a power of two <= 32, Q = 1,
// 3, 5 or 7), natural order in and out: with k = q + Q p and n = np + P nq,
// DFT-P over p for each q, twiddle e^{+2 pi i np q / N2}, DFT-Q over q.
// ---------------------------------------------------------------------------
template <int N2, typename C> __device__ __forceinline__ void dft_natural(C* v) {
  constexpr int Q = odd_part(N2), P = N2 / Q;
  static_assert(P <= 32 && (Q == 1 || Q == 3 || Q == 5 || Q == 7), "in-register length");
  if constexpr (Q == 1) {
    dft_reg<P>(v);
    C t[P];
#pragma unroll
    for (int i = 0; i < P; ++i) t[i] = v[operm<P>(i)];
#pragma unroll
    for (int i = 0; i < P; ++i) v[i] = t[i];
  } else if constexpr (P == 1) {
    dft_odd<Q>(v);
  } else {
    C y[N2];  // y[q P + np]
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      C t[P];
#pragma unroll
      for (int p = 0; p < P; ++p) t[p] = v[q + Q * p];
      dft_reg<P>(t);
#pragma unroll
      for (int np = 0; np < P; ++np) y[q * P + np] = t[operm<P>(np)];
    }
#pragma unroll
    for (int q = 1; q < Q; ++q)
#pragma unroll
      for (int np = 1; np < P; ++np) {
        const int j = (np * q) % N2;
        const float c = kRootTable<N2>.c[j], s = kRootTable<N2>.s[j];
        const C d = y[q * P + np];
        y[q * P + np] = mk(d.x * c - d.y * s, d.x * s + d.y * c);
      }
#pragma unroll
    for (int np = 0; np < P; ++np) {
      C t[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) t[q] = y[q * P + np];
      dft_odd<Q>(t);
#pragma unroll
      for (int nq = 0; nq < Q; ++nq) v[np + P * nq] = t[nq];
    }
  }
}

// ---------------------------------------------------------------------------
// Bulk asynchronous global -> shared copy with mbarrier completion.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
               : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(mbar)
      : "memory");
}

// ---------------------------------------------------------------------------
// Configuration of a line length N served by L lanes.
// ---------------------------------------------------------------------------
template <int N, int L> struct ShflCfg {
  static constexpr int N2 = N / L, G = 32 / L, WPB = 4, THREADS = 32 * WPB;
  // bytes copied per line: N + 1 complex FP32 values rounded up to 16 bytes
  static constexpr int LINE_BYTES = ((N + 1) * 8 + 15) / 16 * 16;
  // line slot: 64 bytes past a multiple of 128, so that two lines read by one
  // half-warp (L = 8) fall on disjoint banks
  static constexpr int SLOT = LINE_BYTES + ((64 - LINE_BYTES % 128) + 128) % 128;
  static constexpr int OFF_TW = WPB * G * SLOT;           // 2N twiddles e^{2 pi i m / 2N}
  static constexpr int OFF_SX = OFF_TW + 2 * N * 8;      // s_x, x < 2N
  static constexpr int OFF_FX = OFF_SX + 2 * N * 4;      // flags, x < 2N
  static constexpr int OFF_BAR = OFF_FX + (2 * N + 15) / 16 * 16;
  static constexpr int OFF_RED = OFF_BAR + WPB * 8;      // the warps' FP64 moment pairs
  static constexpr int SMEM = OFF_RED + WPB * 16;
  static constexpr int K = (2 * N + 31) / 32;            // epilogue outputs a lane, a line
  static constexpr int ODD = odd_part(N2 > 0 ? N2 : 1);  // N2 = (N2 / ODD) ODD
  // resident blocks asked of the compiler: 9 (56 registers a thread) for
  // per-lane lines of at most 8 values, 8 (64 registers) up to 16, else what
  // the registers allow
  static constexpr int MINB = N2 <= 8 ? 9 : (N2 <= 16 ? 8 : 1);
  __host__ __device__ static constexpr bool valid() {
    return (L == 8 || L == 16 || L == 32) && N % L == 0 && N2 >= 2 && N2 <= 32 &&
           (ODD == 1 || ODD == 3 || ODD == 5 || ODD == 7) && SMEM <= 200 * 1024;
  }
};

constexpr uint64_t kBulkWaitNs = 1000000000ull;  // 1 s per line-copy wait

// Epilogue of the KC x values x0 + lane + 32 j (j < KC) of one line whose
// C2R outputs sit at ob (x < Nx <= 2N read).
template <int KC, bool MOM>
__device__ __forceinline__ void epi_chunk(const LineEpilogue<float>& ep, const float* ob, int x0, int lane,
                                          int Nx, double* s1, double* s2) {
  int xs[KC];
  float vv[KC];
#pragma unroll
  for (int j = 0; j < KC; ++j) {
    xs[j] = x0 + lane + 32 * j;
    vv[j] = xs[j] < Nx ? ob[xs[j]] : 0.f;
  }
  ep.template put_group_line<KC, MOM>(xs, vv, Nx, s1, s2);
}

// Block bx of a launch: warp w takes the G lines of group bx WPB + w.  With
// a.epi.mom set, every final value f of the block's points (and f^2) is added
// in FP64 and the block's pair stored at mom[2 bx].
template <int N, int L>
__device__ __forceinline__ void c2r_shfl_body(const GenArgs& a, int64_t bx) {
  using Cfg = ShflCfg<N, L>;
  using C = float2;
  constexpr int N2 = Cfg::N2, G = Cfg::G;
  extern __shared__ __align__(128) unsigned char shfl_sm[];
  unsigned char* smraw = shfl_sm;
  const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
  const int li = lane / L, t = lane % L;
  unsigned char* wreg = smraw + warp * G * Cfg::SLOT;
  C* tws = reinterpret_cast<C*>(smraw + Cfg::OFF_TW);
  float* sxs = reinterpret_cast<float*>(smraw + Cfg::OFF_SX);
  uint8_t* fxs = smraw + Cfg::OFF_FX;
  const uint32_t bar = tc::smem_u32(smraw + Cfg::OFF_BAR + warp * 8);
  const int Nx = a.Nout[0], Ny = a.Nout[1];
  const int64_t nlines = (int64_t)Ny * a.Nout[2];
  const int64_t l0 = (bx * Cfg::WPB + warp) * G;  // the warp's first line
  const bool blend = a.epi.mode != 0;
  // ---- lane 0: the group's line copies, first of all ----
  if (lane == 0) {
    tc::mbar_init(bar, 1);
    const int nv = (int)(nlines - l0 < G ? (nlines - l0 > 0 ? nlines - l0 : 0) : G);
    if (nv > 0) {
      mbar_expect_tx(bar, (uint32_t)(nv * Cfg::LINE_BYTES));
      const C* work = static_cast<const C*>(a.work);
      for (int i = 0; i < nv; ++i) {
        const int64_t l = l0 + i;
        const int y = (int)(l % Ny), z = (int)(l / Ny);
        bulk_g2s(tc::smem_u32(wreg + i * Cfg::SLOT), work + ((size_t)z * a.P[1] + (size_t)y) * a.Hpad,
                 Cfg::LINE_BYTES, bar);
      }
    }
  }
  // ---- the block's tables ----
  {
    const C* twx = static_cast<const C*>(a.tw_x);
    for (int i = (int)threadIdx.x; i < 2 * N; i += Cfg::THREADS) tws[i] = __ldg(twx + i);
    if (blend) {
      const float* sx = sw_of<float>(a.epi.ax[0]);
      const uint8_t* fx = a.epi.ax[0].flags;
      for (int i = (int)threadIdx.x; i < Nx; i += Cfg::THREADS) {
        sxs[i] = a.epi.apply_pou ? __ldg(sx + i) : 1.f;
        fxs[i] = __ldg(fx + i);
      }
    }
  }
  __syncthreads();  // tables and the warps' barrier initialisation
  double s1 = 0.0, s2 = 0.0;
  const bool mom = a.epi.mom != nullptr;
  bool work_here = l0 < nlines;
  if (work_here && !tc::mbar_wait(bar, 0, kBulkWaitNs)) {
    // a copy did not land in time: report, give it one more bounded wait
    // (the copies write this block's shared memory), skip the group
    if (lane == 0) {
      atomicOr(a.status, 1);
      tc::mbar_wait(bar, 0, kBulkWaitNs);
    }
    __syncwarp();
    work_here = false;
  }
  if (work_here) {
    // ---- pre-combination and stage A ----
    C v[N2];
    {
      const C* line = reinterpret_cast<const C*>(wreg + li * Cfg::SLOT);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int k = t + L * k2;
        const C xk = line[k], xn = line[N - k];
        const C xc = cconj(xn);
        const C e = cadd(xk, xc);
        const C o = cmul(csub(xk, xc), tws[k]);
        C z = mk(e.x - o.y, e.y + o.x);
        if (k2 == 0 && t == 0) z = mk(xk.x + xn.x, xk.x - xn.x);
        v[k2] = z;
      }
    }
    dft_natural<N2>(v);
    // ---- twiddle e^{2 pi i n2 k1 / N} = tws[2 n2 k1] ----
    {
      const C* tw = tws + 2 * t;
#pragma unroll
      for (int n2 = 1; n2 < N2; ++n2) v[n2] = cmul(v[n2], tw[(2 * t) * (n2 - 1)]);
    }
    // ---- stage B across the line's lanes ----
#pragma unroll
    for (int s = L / 2; s >= 1; s >>= 1) {
      const bool hi = (t & s) != 0;
      const float sg = hi ? -1.f : 1.f;
      // hi lanes: (partner - own) e^{2 pi i (t mod s) / 2s} = tws[(t mod s) N / s]
      const C w = hi ? tws[(t & (s - 1)) * (N / s)] : mk(1.f, 0.f);
#pragma unroll
      for (int i = 0; i < N2; ++i) {
        const float pr = __shfl_xor_sync(0xffffffffu, v[i].x, s);
        const float pi = __shfl_xor_sync(0xffffffffu, v[i].y, s);
        const float ar = fmaf(sg, v[i].x, pr), ai = fmaf(sg, v[i].y, pi);
        v[i] = (s > 1) ? mk(ar * w.x - ai * w.y, ar * w.y + ai * w.x) : mk(ar, ai);
      }
    }
    // ---- outputs y[n2 + N2 n1], n1 = bitrev(t): reals 2n, 2n + 1 ----
    __syncwarp();  // every lane has read its raw line
    {
      C* ob = reinterpret_cast<C*>(wreg + li * Cfg::SLOT) + N2 * brev<L>(t);
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) ob[n2] = v[n2];
    }
    __syncwarp();
    // ---- epilogue: one line at a time, lanes along x ----
#pragma unroll 1
    for (int i = 0; i < G; ++i) {
      const int64_t l = l0 + i;
      if (l >= nlines) break;
      const int y = (int)(l % Ny), z = (int)(l / Ny);
      LineEpilogue<float> ep(a.epi, y, z, Nx, Ny);
      if (blend) {
        ep.fx = fxs;
        ep.sx = sxs;
      }
      const float* ob = reinterpret_cast<const float*>(wreg + i * Cfg::SLOT);
      // x < 32 KA in one group (its reads of earlier tiles' partial sums all
      // issued before its writes), then steps of 64 points up to Nx
      constexpr int KA = Cfg::K < 8 ? Cfg::K : 8;
      if (mom) epi_chunk<KA, true>(ep, ob, 0, lane, Nx, &s1, &s2);
      else epi_chunk<KA, false>(ep, ob, 0, lane, Nx, &s1, &s2);
#pragma unroll
      for (int j0 = KA; j0 < Cfg::K; j0 += 2) {
        if (32 * j0 >= Nx) break;
        if (mom) epi_chunk<2, true>(ep, ob, 32 * j0, lane, Nx, &s1, &s2);
        else epi_chunk<2, false>(ep, ob, 32 * j0, lane, Nx, &s1, &s2);
      }
    }
  }
  if (mom) {  // the block's pair: warps in shared memory, then warp 0
    double* red = reinterpret_cast<double*>(smraw + Cfg::OFF_RED);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      red[2 * warp] = s1;
      red[2 * warp + 1] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t1 = 0.0, t2 = 0.0;
#pragma unroll
      for (int w = 0; w < Cfg::WPB; ++w) {
        t1 += red[2 * w];
        t2 += red[2 * w + 1];
      }
      a.epi.mom[2 * bx] = t1;
      a.epi.mom[2 * bx + 1] = t2;
    }
  }
}

template <int N, int L>
__global__ void __launch_bounds__(ShflCfg<N, L>::THREADS, ShflCfg<N, L>::MINB) k_c2r_x_shfl(const GenArgs a) {
  c2r_shfl_body<N, L>(a, blockIdx.x);
}
template <int N, int L>
__global__ void __launch_bounds__(ShflCfg<N, L>::THREADS, ShflCfg<N, L>::MINB) k_c2r_x_shfl_batch(const BatchMap m) {
  int loc;
  const GenArgs a = m.args[batch_item(m, &loc)];
  c2r_shfl_body<N, L>(a, loc);
}

}  // namespace scarl
