// c2r_tc.cu -- pass 3 of the padded generator (Hermitian C2R along x, crop,
// blend epilogue) with the x DFT on the tensor cores in split BF16: the FP32
// output of scarl_gen_padded / scarl_generate_sample when the caller asks for
// SCARL_F32 | SCARL_SPLIT_BF16_X and the half length N = P0 / 2 factors as
// N1 x N2 with N2 = 32 or 16 and N1 <= 8 (single-tile launches).
//
// A line of N + 1 half-spectrum values X[k] (a row of the pass-2 output) is
// pre-combined into the complex sequence
//   z[k] = (X[k] + conj X[N - k]) + i e^{2 pi i k / 2N} (X[k] - conj X[N - k]),
//   z[0] = (Re X[0] + Re X[N], Re X[0] - Re X[N]),
// whose inverse DFT y[n] gives the real outputs x[2n] = Re y[n], x[2n + 1] =
// Im y[n] (the same arithmetic as the CUDA-core pass 3).  The DFT runs in two
// matrix stages (k = k1 + N1 k2, n = n2 + N2 n1):
//   stage 1  Y[k1][n2] = sum_k2 z[k1 + N1 k2] e^{+2 pi i n2 k2 / N2}
//   twiddle  Y'[k1][n2] = Y[k1][n2] e^{+2 pi i n2 k1 / N}          (FP32)
//   stage 2  y[n2 + N2 n1] = sum_k1 Y'[k1][n2] e^{+2 pi i n1 k1 / N1}
// each a real GEMM D = A B^T on interleaved re/im columns with every operand
// split into a BF16 head and tail and D = Ah Bh + Ah Bt + At Bh accumulated
// in FP32 in tensor memory (2^-17 relative per stage, like pass 1).  Stage-1
// rows are (line, k1) with k1 < 8 (rows k1 >= N1 are zero), so that an item
// of 16 lines is one 128-row tile; stage 2 has 16 N2 rows (line, n2) with
// K = 16 (re and im of k1 < 8) and 16 outputs (re and im of n1 < 8).
//
// Persistent CTAs of 128 threads, four per SM (each CTA's phases wait on
// the tensor core, on global loads and on its block barriers; four
// independent CTAs keep the SM issuing), walk items of 16 consecutive lines
// of the tile.  Each thread builds one stage-1 row from the line in global
// memory through the read-only path (every value is read twice, as X[k] by
// one row and as X[N - k] by another; the second read hits the cache).  The epilogue's per-line tables (output base, y-z flags,
// s_y s_z) are read into shared memory while the operand is built.  The
// epilogue (crop, or partition-of-unity blend into the global field with the
// marginal transform, and the FP64 moment sums; the same arithmetic as the
// CUDA-core pass 3) runs straight from the stage-2 accumulators: the thread
// holding row (line, n2) writes x = 2 (n2 + N2 n1) and x + 1, so consecutive
// lanes write consecutive pairs of x, all of a row's values in one group (one
// round trip for the earlier tiles' partial sums).  Every wait
// on the tensor core is bounded; on timeout the kernel raises the status
// word and returns after its products have had one more bounded wait and
// its tensor memory is freed.
#include <algorithm>

#include "c2r_shfl.cuh"
#include "tc_sm100.cuh"

namespace scarl {

namespace {

template <int N1_, int N2_>
struct C2rTcCfg {
  static constexpr int N1 = N1_, N2 = N2_, N = N1 * N2;
  static constexpr int LB = 16;  // lines per item
  static constexpr int THREADS = 128, CTAS_PER_SM = 4;
  static constexpr int ROWS2 = LB * N2;  // stage-2 rows (line, n2)
  static constexpr int T2 = ROWS2 / 128;
  static constexpr int K1 = 2 * N2;  // stage-1 K = N: re k2 < N2, im k2 < N2
  // stage-1 A (one 128-row tile), K-major: 16-byte K chunks 128 B apart,
  // 8-row groups SBO1 apart
  static constexpr int SBO1 = 128 * (K1 / 8), A1B = 16 * SBO1;
  // stage-2 A, MN-major: the two 8-row K groups (re k1, im k1) 128 B apart,
  // 8-element M groups SBO2 apart, 128-row tiles contiguous
  static constexpr int SBO2 = 256, TILE2 = 16 * SBO2, A2B = T2 * TILE2;
  static constexpr int AB = A1B > A2B ? A1B : A2B;
  static constexpr int REGION = 2 * AB;  // head and tail operands
  static constexpr int B1B = (K1 / 8) * SBO1;               // 2 N2 rows x K1
  static constexpr int SBOB2 = 256, B2B = 2 * SBOB2;         // 16 rows x K = 16
  static constexpr int OFF_AH = 0, OFF_AL = AB;
  static constexpr int OFF_B1H = REGION, OFF_B1L = OFF_B1H + B1B;
  static constexpr int OFF_B2H = OFF_B1L + B1B, OFF_B2L = OFF_B2H + B2B;
  static constexpr int OFF_TW = OFF_B2L + B2B;          // 2N twiddles e^{2 pi i m / 2N}
  static constexpr int OFF_SX = OFF_TW + 2 * N * 8;     // s_x, x < 2N
  static constexpr int OFF_LB = OFF_SX + 2 * N * 4;     // per line: output base (8 B)
  static constexpr int OFF_LS = OFF_LB + LB * 8;        // per line: s_y s_z (4 B)
  static constexpr int OFF_LF = OFF_LS + LB * 4;        // per line: y-z flags (1 B)
  static constexpr int OFF_FX = OFF_LF + LB;            // flags, x < 2N
  static constexpr int OFF_BAR = (OFF_FX + 2 * N + 15) / 16 * 16;  // mbarrier, tensor-memory slot
  static constexpr int OFF_RED = OFF_BAR + 16;          // the warps' FP64 moment pairs
  static constexpr int SMEM = OFF_RED + (THREADS / 32) * 16;
  static constexpr int TMEM_COLS = 64;  // stage 1: K1 <= 64 columns; stage 2: T2 x 16 <= 64
  static_assert(N2 == 16 || N2 == 32, "stage-1 length");
  static_assert(N1 >= 2 && N1 <= 8, "stage-2 length");
  static_assert(K1 <= TMEM_COLS && T2 * 16 <= TMEM_COLS, "tensor memory");
  static_assert(CTAS_PER_SM * (SMEM + 1024) <= 228 * 1024, "shared memory");
  static_assert(TMEM_COLS * CTAS_PER_SM <= 512, "tensor memory per SM");
};

constexpr uint64_t kTcWaitNs = 1000000000ull;  // 1 s per wait

// The split inverse DFT of length L (<= LP) as a (2 LP x 2 LP) K-major B
// operand: row n = output (re n < LP, im n >= LP), column k = input (re k <
// LP, im k >= LP); entries of outputs or inputs >= L are zero.
template <int LP, int L, int SBO>
__device__ void fill_dft_pad(unsigned char* hi, unsigned char* lo) {
  for (int idx = threadIdx.x; idx < 4 * LP * LP; idx += blockDim.x) {
    const int n = idx / (2 * LP), k = idx % (2 * LP);
    const int no = n % LP, ki = k % LP;
    double v = 0.0;
    if (no < L && ki < L) {
      const int m = (no * ki) % L;
      double s, c;
      sincospi(2.0 * (double)m / (double)L, &s, &c);
      const bool im_out = n >= LP, im_in = k >= LP;
      v = (im_out == im_in) ? c : (im_out ? s : -s);
    }
    const __nv_bfloat16 h = __double2bfloat16(v);
    const __nv_bfloat16 t = __double2bfloat16(v - (double)__bfloat162float(h));
    const uint32_t off = (uint32_t)((n >> 3) * SBO + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
    *reinterpret_cast<__nv_bfloat16*>(hi + off) = h;
    *reinterpret_cast<__nv_bfloat16*>(lo + off) = t;
  }
}

template <int N1, int N2>
__global__ void __launch_bounds__(128, 4) k_c2r_x_tc(const GenArgs a) {
  using Cfg = C2rTcCfg<N1, N2>;
  using C = float2;
  constexpr int N = Cfg::N, LB = Cfg::LB;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* AH = sm + Cfg::OFF_AH;
  unsigned char* AL = sm + Cfg::OFF_AL;
  const uint32_t sAH = tc::smem_u32(AH), sAL = tc::smem_u32(AL);
  const uint32_t sB1H = tc::smem_u32(sm + Cfg::OFF_B1H), sB1L = tc::smem_u32(sm + Cfg::OFF_B1L);
  const uint32_t sB2H = tc::smem_u32(sm + Cfg::OFF_B2H), sB2L = tc::smem_u32(sm + Cfg::OFF_B2L);
  const uint32_t mbar = tc::smem_u32(sm + Cfg::OFF_BAR);  // matrix products
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + Cfg::OFF_BAR + 8);
  C* tws = reinterpret_cast<C*>(sm + Cfg::OFF_TW);
  float* sxs = reinterpret_cast<float*>(sm + Cfg::OFF_SX);
  uint8_t* fxs = sm + Cfg::OFF_FX;
  uint64_t* lbase = reinterpret_cast<uint64_t*>(sm + Cfg::OFF_LB);
  float* lsyz = reinterpret_cast<float*>(sm + Cfg::OFF_LS);
  uint8_t* lfyz = sm + Cfg::OFF_LF;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Nx = a.Nout[0], Ny = a.Nout[1];
  const int nlines = a.Nout[1] * a.Nout[2];  // <= 2048^2
  const int nitems = (nlines + LB - 1) / LB;
  const bool blend = a.epi.mode != 0;
  const bool mom = a.epi.mom != nullptr;
  const C* work = static_cast<const C*>(a.work);

  if (tid == 0) tc::mbar_init(mbar, 1);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), Cfg::TMEM_COLS);
  fill_dft_pad<N2, N2, Cfg::SBO1>(sm + Cfg::OFF_B1H, sm + Cfg::OFF_B1L);
  fill_dft_pad<8, N1, Cfg::SBOB2>(sm + Cfg::OFF_B2H, sm + Cfg::OFF_B2L);
  {
    const C* twx = static_cast<const C*>(a.tw_x);
    for (int i = tid; i < 2 * N; i += Cfg::THREADS) tws[i] = __ldg(twx + i);
    if (blend) {
      const float* sx = sw_of<float>(a.epi.ax[0]);
      const uint8_t* fx = a.epi.ax[0].flags;
      for (int i = tid; i < Nx; i += Cfg::THREADS) {
        sxs[i] = a.epi.apply_pou ? __ldg(sx + i) : 1.f;
        fxs[i] = __ldg(fx + i);
      }
    }
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  constexpr uint32_t ID1 = tc::idesc_bf16(128, Cfg::K1, false);
  constexpr uint32_t ID2 = tc::idesc_bf16(128, 16, true);  // A MN-major

  // this thread's stage-1 row (line, k1)
  const int r_line = tid >> 3, r_k1 = tid & 7;
  const uint32_t rowoff = (uint32_t)((tid >> 3) * Cfg::SBO1 + (tid & 7) * 16);
  uint32_t mphase = 0;
  bool ok = true;
  double s1 = 0.0, s2 = 0.0;

  for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
    const int l0 = it * LB;
    const int nv = min(LB, nlines - l0);
    // ---- the epilogue's line tables (threads 0..nv-1) ----
    if (tid < nv) {
      const int l = l0 + tid;
      const LineEpilogue<float> ep(a.epi, l % Ny, l / Ny, Nx, Ny);
      lbase[tid] = (uint64_t)ep.base;
      lsyz[tid] = ep.syz;
      lfyz[tid] = ep.fyz;
    }
    // ---- stage-1 operand: row (line, k1), K = re k2 | im k2, from the
    //      line in global memory ----
    {
      const bool live = r_line < nv && r_k1 < N1;
      const int l = l0 + (live ? r_line : 0);
      const C* X = work + ((size_t)(l / Ny) * a.P[1] + (size_t)(l % Ny)) * a.Hpad;
#pragma unroll 2
      for (int c = 0; c < N2 / 8; ++c) {  // chunks of 8 k2
        float re[8], im[8];
        C xk[8], xn[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = live ? r_k1 + N1 * (8 * c + e) : 0;  // < N
          xk[e] = live ? __ldg(X + k) : mk(0.f, 0.f);
          xn[e] = live ? __ldg(X + (N - k)) : mk(0.f, 0.f);
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = r_k1 + N1 * (8 * c + e);
          if (k == 0) {
            re[e] = xk[e].x + xn[e].x;
            im[e] = xk[e].x - xn[e].x;
          } else {
            const C xc = cconj(xn[e]);
            const C ev = cadd(xk[e], xc);
            const C od = cmul(csub(xk[e], xc), tws[live ? k : 0]);
            re[e] = ev.x - od.y;
            im[e] = ev.y + od.x;
          }
        }
        uint4 hr, lr, hi, li;
        tc::split2(re[0], re[1], hr.x, lr.x);
        tc::split2(re[2], re[3], hr.y, lr.y);
        tc::split2(re[4], re[5], hr.z, lr.z);
        tc::split2(re[6], re[7], hr.w, lr.w);
        tc::split2(im[0], im[1], hi.x, li.x);
        tc::split2(im[2], im[3], hi.y, li.y);
        tc::split2(im[4], im[5], hi.z, li.z);
        tc::split2(im[6], im[7], hi.w, li.w);
        const uint32_t ore = rowoff + (uint32_t)c * 128;
        const uint32_t oim = rowoff + (uint32_t)(N2 / 8 + c) * 128;
        *reinterpret_cast<uint4*>(AH + ore) = hr;
        *reinterpret_cast<uint4*>(AL + ore) = lr;
        *reinterpret_cast<uint4*>(AH + oim) = hi;
        *reinterpret_cast<uint4*>(AL + oim) = li;
      }
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- stage 1 ----
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < Cfg::K1 / 16; ++s) {
        const uint32_t o = s * 2 * 128;
        const uint64_t ah = tc::desc(sAH + o, 128, Cfg::SBO1);
        const uint64_t al = tc::desc(sAL + o, 128, Cfg::SBO1);
        const uint64_t bh = tc::desc(sB1H + o, 128, Cfg::SBO1);
        const uint64_t bl = tc::desc(sB1L + o, 128, Cfg::SBO1);
        tc::mma_bf16(tmem, ah, bh, ID1, s > 0 ? 1u : 0u);
        tc::mma_bf16(tmem, ah, bl, ID1, 1u);
        tc::mma_bf16(tmem, al, bh, ID1, 1u);
      }
      tc::commit(mbar);
    }
    ok = warp == 0 ? tc::mbar_wait(mbar, mphase, kTcWaitNs) : true;
    mphase ^= 1;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    tc::fence_after_sync();
    // ---- stage-1 rows back (warp w: rows 32 w .. 32 w + 31), twiddled, into
    //      the MN-major stage-2 operand: element (row line N2 + n2, k = k1
    //      (re) | 8 + k1 (im)) ----
    {
      const int line = tid >> 3, k1 = tid & 7;
      const bool live = k1 < N1;
      const uint32_t base = (uint32_t)(N2 * line / 8) * Cfg::SBO2 + (uint32_t)k1 * 16;
      const uint32_t col = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 2
      for (int g = 0; g < N2 / 8; ++g) {  // 8 n2 = one M group
        float v[16];
        tc::tmem_ld<8>(col + 8 * g, v);           // re of n2 = 8 g ..
        tc::tmem_ld<8>(col + N2 + 8 * g, v + 8);  // im
        tc::tmem_wait_ld();
        uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const int n2 = 8 * g + e;
          C w0 = mk(0.f, 0.f), w1 = mk(0.f, 0.f);
          if (live) {
            w0 = tws[2 * n2 * k1];
            w1 = tws[2 * (n2 + 1) * k1];
          }
          const float yr0 = v[e] * w0.x - v[8 + e] * w0.y, yi0 = v[e] * w0.y + v[8 + e] * w0.x;
          const float yr1 = v[e + 1] * w1.x - v[9 + e] * w1.y, yi1 = v[e + 1] * w1.y + v[9 + e] * w1.x;
          tc::split2(yr0, yr1, rh[e / 2], rl[e / 2]);
          tc::split2(yi0, yi1, ih[e / 2], il[e / 2]);
        }
        const uint32_t off = base + (uint32_t)g * Cfg::SBO2;
        *reinterpret_cast<uint4*>(AH + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(AL + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4*>(AH + off + 128) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4*>(AL + off + 128) = make_uint4(il[0], il[1], il[2], il[3]);
      }
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- stage 2 ----
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int t = 0; t < Cfg::T2; ++t) {
        const uint32_t o = t * Cfg::TILE2;
        const uint64_t ah = tc::desc(sAH + o, 128, Cfg::SBO2);
        const uint64_t al = tc::desc(sAL + o, 128, Cfg::SBO2);
        const uint64_t bh = tc::desc(sB2H, 128, Cfg::SBOB2);
        const uint64_t bl = tc::desc(sB2L, 128, Cfg::SBOB2);
        const uint32_t d = tmem + t * 16;
        tc::mma_bf16(d, ah, bh, ID2, 0u);
        tc::mma_bf16(d, ah, bl, ID2, 1u);
        tc::mma_bf16(d, al, bh, ID2, 1u);
      }
      tc::commit(mbar);
    }
    ok = warp == 0 ? tc::mbar_wait(mbar, mphase, kTcWaitNs) : true;
    mphase ^= 1;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    tc::fence_after_sync();
    // ---- epilogue straight from tensor memory: thread R of tile t holds
    //      row (line, n2) = (R / N2, R % N2) with y[n2 + N2 n1], the reals
    //      x = 2 (n2 + N2 n1) and x + 1 (consecutive lanes on consecutive
    //      pairs of x) ----
#pragma unroll 1
    for (int t = 0; t < Cfg::T2; ++t) {
      const int R = t * 128 + tid;
      const int line = R / N2, n2 = R % N2;
      float v[16];
      tc::tmem_ld<16>(tmem + ((uint32_t)(warp * 32) << 16) + t * 16, v);
      tc::tmem_wait_ld();
      if (line < nv) {
        const LineEpilogue<float> ep(a.epi, (size_t)lbase[line], lfyz[line], lsyz[line],
                                     blend ? fxs : nullptr, blend ? sxs : nullptr);
        int xs[2 * N1];
        float vv[2 * N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
          xs[2 * n1] = 2 * (n2 + N2 * n1);
          xs[2 * n1 + 1] = 2 * (n2 + N2 * n1) + 1;
          vv[2 * n1] = v[n1];
          vv[2 * n1 + 1] = v[8 + n1];
        }
        if (mom) ep.template put_group_line<2 * N1, true>(xs, vv, Nx, &s1, &s2);
        else ep.template put_group_line<2 * N1, false>(xs, vv, Nx);
      }
    }
    tc::fence_before_sync();
    __syncthreads();  // tensor memory and the line tables are the next item's
  }
  if (!ok) {
    // a product did not complete in time: report, then give it one more
    // bounded wait before the tensor memory it writes is released
    if (tid == 0) {
      atomicOr(a.status, 1);
      tc::mbar_wait(mbar, mphase ^ 1, kTcWaitNs);
    }
    __syncthreads();
  }
  if (mom) {  // the CTA's pair: warps in shared memory, then thread 0
    double* red = reinterpret_cast<double*>(sm + Cfg::OFF_RED);
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
    if (tid == 0) {
      double t1 = 0.0, t2 = 0.0;
#pragma unroll
      for (int w = 0; w < Cfg::THREADS / 32; ++w) {
        t1 += red[2 * w];
        t2 += red[2 * w + 1];
      }
      a.epi.mom[2 * (int64_t)blockIdx.x] = t1;
      a.epi.mom[2 * (int64_t)blockIdx.x + 1] = t2;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_free(tmem, Cfg::TMEM_COLS);
}

constexpr int kMaxDev = 64;

// The CTA count of a tile's launch: one per item up to two per SM.
template <int N1, int N2>
cudaError_t grid_of(const GenArgs& a, bool prepare, int* grid) {
  using Cfg = C2rTcCfg<N1, N2>;
  static int sms[kMaxDev] = {};
  static bool ready[kMaxDev] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  if (!sms[dev]) {
    int n = 0;
    if ((e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    sms[dev] = n;
  }
  if (prepare && !ready[dev]) {
    auto kern = k_c2r_x_tc<N1, N2>;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM)) !=
        cudaSuccess)
      return e;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
      return e;
    ready[dev] = true;
  }
  const int nlines = a.Nout[1] * a.Nout[2];
  const int nitems = (nlines + Cfg::LB - 1) / Cfg::LB;
  *grid = std::max(1, std::min(nitems, sms[dev] * Cfg::CTAS_PER_SM));
  return cudaSuccess;
}

template <int N1, int N2>
cudaError_t run_tc(const GenArgs& a, int* blocks, cudaStream_t s) {
  using Cfg = C2rTcCfg<N1, N2>;
  int grid = 0;
  cudaError_t e = grid_of<N1, N2>(a, blocks == nullptr, &grid);
  if (e != cudaSuccess) return e;
  if (blocks) {
    *blocks = grid;
    return cudaSuccess;
  }
  if (!a.status || a.Nout[0] > 2 * Cfg::N) return cudaErrorInvalidValue;
  k_c2r_x_tc<N1, N2><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(a);
  return cudaGetLastError();
}

cudaError_t run_any(const GenArgs& a, int* blocks, cudaStream_t s) {
  switch (a.P[0] / 2) {
    case 64: return run_tc<2, 32>(a, blocks, s);
    case 96: return run_tc<3, 32>(a, blocks, s);
    case 128: return run_tc<4, 32>(a, blocks, s);
    case 160: return run_tc<5, 32>(a, blocks, s);
    case 192: return run_tc<6, 32>(a, blocks, s);
    case 224: return run_tc<7, 32>(a, blocks, s);
    case 256: return run_tc<8, 32>(a, blocks, s);
    case 32: return run_tc<2, 16>(a, blocks, s);
    case 48: return run_tc<3, 16>(a, blocks, s);
    case 80: return run_tc<5, 16>(a, blocks, s);
    case 112: return run_tc<7, 16>(a, blocks, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

// Half lengths N = P0 / 2 with a tensor-core pass 3: N1 x 32 (N1 = 2..8) and
// N1 x 16 (N1 = 2, 3, 5, 7).
bool c2r_x_tc_supported(int N) {
  switch (N) {
    case 32: case 48: case 64: case 80: case 96: case 112: case 128: case 160: case 192:
    case 224: case 256:
      return true;
    default:
      return false;
  }
}

cudaError_t launch_c2r_x_tc(const GenArgs& a, cudaStream_t s) { return run_any(a, nullptr, s); }

int c2r_x_tc_blocks(const GenArgs& a) {
  int nb = 0;
  if (run_any(a, &nb, nullptr) != cudaSuccess) return -1;
  return nb;
}

}  // namespace scarl
