// gen_tc.cu -- pass 1 of the padded generator (spectrum synthesis + inverse
// DFT along z) with the DFT on the tensor cores in split BF16: the FP32
// output of scarl_gen_padded / scarl_generate_sample when the caller asks for
// SCARL_F32 | SCARL_SPLIT_BF16.
//
// A line of N = N1 * N2 modes along z is transformed in two matrix stages
// (the "four-step" factorisation, k = k1 + N1 k2, n = n2 + N2 n1):
//   stage 1  Y[k1][n2] = sum_k2 x[k1 + N1 k2] e^{+2 pi i n2 k2 / N2}
//   twiddle  Y'[k1][n2] = Y[k1][n2] e^{+2 pi i n2 k1 / N}          (FP32)
//   stage 2  X[n2 + N2 n1] = sum_k1 Y'[k1][n2] e^{+2 pi i n1 k1 / N1}
// Each stage is a real GEMM on interleaved re/im columns, D = A B^T with the
// DFT matrix B = [[C, -S], [S, C]].  Every operand is split into a BF16 head
// and a BF16 tail (h = bf16(v), t = bf16(v - h); v = h + t to 2^-17 |v|),
// and D = Ah Bh + Ah Bt + At Bh accumulates in FP32 in tensor memory (the
// dropped At Bt term is 2^-17 relative).  So each DFT stage carries about
// 2^-17 relative error instead of FP32's 2^-24; the field's relative L2
// error against FP64 stays near 4e-6 (tests bound it by 1e-5).
//
// Persistent CTAs of 256 threads, two per SM, walk work items of LB
// consecutive lines (line l = kx + Hx ky, the Philox counter base of the
// line's modes).  Per item: every thread synthesises one stage-1 row (LB N1
// rows: line, k1) from the canonical Philox normals and amplitude tables and
// stores it split into a K-major operand; one thread issues the stage-1
// MMAs; each row comes back from tensor memory, is twiddled, split and
// written into the stage-2 operand, which is MN-major with rows (line, n2)
// so that a thread's 8 consecutive n2 form one 16-byte store; one thread
// issues stage 2; the results pass through shared memory (z-major, padded
// against bank conflicts) so that z < Nz leaves in 128-byte runs of
// consecutive kx.  Every wait on the tensor core is bounded; on timeout the
// kernel raises a status word and returns after freeing its tensor memory.
#include <algorithm>

#include "gen_kernels.cuh"
#include "tc_sm100.cuh"

namespace scarl {

namespace {

template <int N1_, int N2_, int LB_, int NCH_>
struct TcCfg {
  static constexpr int N1 = N1_, N2 = N2_, LB = LB_, N = N1 * N2, NCH = NCH_;
  static constexpr int THREADS = 256, CTAS_PER_SM = 2;
  static constexpr int ROWS1 = LB * N1;  // stage-1 rows (line, k1)
  static constexpr int ROWS2 = LB * N2;  // stage-2 rows (line, n2)
  static constexpr int T1 = ROWS1 / 128, T2 = ROWS2 / 128;
  static constexpr int K1 = 2 * N2, K2 = 2 * N1;  // real K (= MMA N) of each stage
  // stage 1, K-major: 16-byte K chunks 128 B apart, 8-row groups SBO1 apart
  static constexpr int LBO1 = 128, SBO1 = 128 * (K1 / 8), TILE1 = 16 * SBO1;
  // stage 2 operand, MN-major: 8-row K groups LBO2 apart, 8-element M groups
  // SBO2 apart; B2 K-major like stage 1
  static constexpr int LBO2 = 128, SBO2 = 128 * (K2 / 8), TILE2 = 16 * SBO2;
  static constexpr int A1B = T1 * TILE1, A2B = T2 * TILE2;
  static constexpr int AB = A1B > A2B ? A1B : A2B;
  static constexpr int STAGE_LD = LB + 1;  // output staging row (one z), float2 units
  static constexpr int STAGEB = N / NCH * STAGE_LD * 8;
  static constexpr int REGION = (2 * AB > STAGEB ? 2 * AB : STAGEB);
  static constexpr int B1B = (K1 / 8) * SBO1, B2B = (K2 / 8) * SBO2;
  static constexpr int TMEM_USED = LB * N / 64;  // = T1 K1 = T2 K2
  static constexpr int TMEM_COLS = TMEM_USED <= 32 ? 32 : TMEM_USED <= 64 ? 64 : TMEM_USED <= 128 ? 128 : 256;
  static constexpr int OFF_AH = 0, OFF_AL = AB, OFF_B1H = REGION, OFF_B1L = OFF_B1H + B1B;
  static constexpr int OFF_B2H = OFF_B1L + B1B, OFF_B2L = OFF_B2H + B2B;
  static constexpr int OFF_ZT = OFF_B2L + B2B;   // z factor of the amplitude, N floats
  static constexpr int OFF_TW = OFF_ZT + 4 * N;   // twiddles [n2][k1], N float2
  static constexpr int OFF_BAR = OFF_TW + 8 * N;  // mbarrier (8 B) + tensor-memory slot (4 B)
  static constexpr int SMEM = OFF_BAR + 16;
  static_assert(ROWS1 == THREADS, "one stage-1 row per thread");
  static_assert(N1 / NCH == 4 || N1 / NCH == 8 || N1 / NCH == 16, "output chunk widths");
  static_assert(ROWS2 % 128 == 0 && T1 * K1 == TMEM_USED && T2 * K2 == TMEM_USED, "tiling");
  static_assert((N1 == 8 || N1 == 16 || N1 == 32) && N2 % 8 == 0 && K1 <= 256, "radices");
  static_assert(TMEM_USED <= 256 && TMEM_COLS * CTAS_PER_SM <= 512, "tensor memory");
  static_assert(CTAS_PER_SM * (SMEM + 1024) <= 228 * 1024, "shared memory");
};

constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s per tensor-core wait

// The canonical Box-Muller pair of Normals<float> (u1 = (a + 1/2) 2^-32,
// u2 = (b + 1/2) 2^-32, r (cos 2 pi u2, sin 2 pi u2), r = sqrt(-2 ln u1)) at
// the split path's accuracy: r as t rsqrt(t) (0 at t = 0) and u2 from the top 23 bits of
// b (phase error <= 2 pi 2^-24), both far below the 2^-17 of the BF16 split.
__device__ __forceinline__ float2 split_normals(uint32_t a, uint32_t b) {
  const float u1 = __fmaf_rn((float)a, 0x1p-32f, 0x1p-33f);
  const float u2 = __uint_as_float(0x3F800000u | (b >> 9)) - 1.5f + 0x1p-24f;  // u2 - 1/2
  const float t = -2.0f * __logf(u1);            // 0 when u1 rounds to 1
  const float r = t * rsqrtf(fmaxf(t, 0x1p-100f));
  float s, c;
  __sincosf(6.28318530717958647692f * u2, &s, &c);
  return make_float2(-r * c, -r * s);
}

// b^e for b >= 1 as 2^(e log2 b) on the hardware approximations (lg2.approx,
// ex2.approx): relative error a few 2^-22 for the exponents of the Matern
// amplitude (e = -(nu + 3/2) / 2), far below the 2^-17 of the BF16 split.
__device__ __forceinline__ float pow_split(float b, float e) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(e * __log2f(b)));
  return r;
}

// Byte offset of element (row, k) in a canonical K-major operand with
// 16-byte K chunks 128 B apart and 8-row groups sbo apart (rows < 128).
__device__ __forceinline__ uint32_t kmaj_off(int row, int k, int sbo) {
  return (uint32_t)((row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// The split DFT matrix of length L as a (2L x 2L) K-major B operand:
// row n = output (re n < L, im n >= L); column k = input, in natural order
// (re k < L, im k >= L) or, with DRAW_ORDER, in the stage-1 operand's draw
// order: k = 4 d + part with part 0 / 1 = re / im of input d, 2 / 3 = re / im
// of input d + L / 2 (the two modes of one Philox draw).
template <int L, int SBO, bool DRAW_ORDER>
__device__ void fill_dft_b(unsigned char* hi, unsigned char* lo) {
  for (int idx = threadIdx.x; idx < 4 * L * L; idx += blockDim.x) {
    const int n = idx / (2 * L), k = idx % (2 * L);
    const int no = n % L;
    const int ki = DRAW_ORDER ? k / 4 + ((k & 2) ? L / 2 : 0) : k % L;
    const bool im_in = DRAW_ORDER ? (k & 1) != 0 : k >= L;
    const int m = (no * ki) % L;
    double s, c;
    sincospi(2.0 * (double)m / (double)L, &s, &c);
    const bool im_out = n >= L;
    const double v = (im_out == im_in) ? c : (im_out ? s : -s);
    const __nv_bfloat16 h = __double2bfloat16(v);
    const __nv_bfloat16 t = __double2bfloat16(v - (double)__bfloat162float(h));
    const uint32_t off = kmaj_off(n, k, SBO);
    *reinterpret_cast<__nv_bfloat16*>(hi + off) = h;
    *reinterpret_cast<__nv_bfloat16*>(lo + off) = t;
  }
}

// One CTA's walk over work items.  Single tile: items of a0's grid.  Batch
// (several realisations sharing the z length): the flat item index is mapped
// to (realisation, local item) through the group's offset table, and the
// realisation's argument block and amplitude table are reloaded into shared
// memory when it changes.
template <int N1, int N2, int LB, int NCH, int AMP, bool BATCH>
__device__ __forceinline__ void gen_z_tc_body(const GenArgs& a0, const GenArgs* __restrict__ bargs,
                                              const int* __restrict__ bitems,
                                              const int* __restrict__ bstart, int bn, int btotal) {
  using Cfg = TcCfg<N1, N2, LB, NCH>;
  constexpr int N = Cfg::N;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ GenArgs sa;  // batch: the current realisation's arguments
  unsigned char* AH = sm + Cfg::OFF_AH;
  unsigned char* AL = sm + Cfg::OFF_AL;
  const uint32_t sAH = tc::smem_u32(AH), sAL = tc::smem_u32(AL);
  const uint32_t sB1H = tc::smem_u32(sm + Cfg::OFF_B1H), sB1L = tc::smem_u32(sm + Cfg::OFF_B1L);
  const uint32_t sB2H = tc::smem_u32(sm + Cfg::OFF_B2H), sB2L = tc::smem_u32(sm + Cfg::OFF_B2L);
  const uint32_t bar = tc::smem_u32(sm + Cfg::OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + Cfg::OFF_BAR + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = warp & 3;

  if (tid == 0) tc::mbar_init(bar, 1);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tslot), Cfg::TMEM_COLS);
  fill_dft_b<N2, Cfg::SBO1, true>(sm + Cfg::OFF_B1H, sm + Cfg::OFF_B1L);
  fill_dft_b<N1, Cfg::SBO2, false>(sm + Cfg::OFF_B2H, sm + Cfg::OFF_B2L);
  float* zt = reinterpret_cast<float*>(sm + Cfg::OFF_ZT);
  float2* tw2 = reinterpret_cast<float2*>(sm + Cfg::OFF_TW);
  auto load_zt = [&](const GenArgs& g) {
    const float* zsrc = static_cast<const float*>(AMP == AMP_SEPARABLE ? g.az : g.qz);
    for (int i = tid; i < N; i += Cfg::THREADS) zt[i] = zsrc[i];
  };
  {
    const float2* tw = static_cast<const float2*>(a0.tw_z);  // e^{2 pi i m / N}
    for (int i = tid; i < N; i += Cfg::THREADS) tw2[i] = tw[(i / N1) * (i % N1)];  // [n2][k1]
    if (!BATCH) load_zt(a0);
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  constexpr uint32_t ID1 = tc::idesc_bf16(128, Cfg::K1, false);
  constexpr uint32_t ID2 = tc::idesc_bf16(128, Cfg::K2, true);  // A MN-major

  // this thread's stage-1 row: (line, k1) with k1 = k1lo + 8 k1hi
  const int R1 = tid;
  const int s_line = (R1 >> 3) % LB, s_k1 = (R1 & 7) + 8 * (R1 / (8 * LB));
  uint32_t phase = 0;
  bool ok = true;
  // test hook: no stage-1 MMA is issued, so the first wait runs out (after
  // 20 ms) and the bounded-wait path below reports it
  const bool wait_test = a0.wait_test != 0;
  const uint64_t wait_ns = wait_test ? 20000000ull : kWaitNs;
  const int nitems0 = BATCH ? btotal : (a0.Hx * a0.P[1] + LB - 1) / LB;
  int cur = -1;

  for (int gitem = blockIdx.x; gitem < nitems0 && ok; gitem += gridDim.x) {
    int item = gitem;
    if constexpr (BATCH) {
      int lo = 0, hi = bn;  // bstart[lo] <= gitem < bstart[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(bstart + mid) <= gitem) lo = mid;
        else hi = mid;
      }
      item = gitem - __ldg(bstart + lo);
      const int r = __ldg(bitems + lo);
      if (r != cur) {  // uniform over the CTA: every thread walks the same items
        __syncthreads();
        const uint32_t* src = reinterpret_cast<const uint32_t*>(bargs + r);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
        for (int i = tid; i < (int)(sizeof(GenArgs) / 4); i += Cfg::THREADS) dst[i] = __ldg(src + i);
        __syncthreads();
        load_zt(sa);
        __syncthreads();
        cur = r;
      }
    }
    const GenArgs& a = BATCH ? sa : a0;
    const int nlines = a.Hx * a.P[1];  // <= 1025 * 2048
    const uint64_t mz = (uint64_t)a.Hx * (uint64_t)a.P[1];
    const float* ax = static_cast<const float*>(a.ax);
    const float* ay = static_cast<const float*>(a.ay);
    const float* qx = static_cast<const float*>(a.qx);
    const float* qy = static_cast<const float*>(a.qy);
    float2* work = static_cast<float2*>(a.work);
    const int Nz = a.Nout[2];
    const int l0 = item * LB;
    // ---- synthesis of stage-1 row R1 ----
    {
      const int l = l0 + s_line;
      const bool valid = l < nlines;
      const int ky = valid ? l / a.Hx : 0, kx = valid ? l - ky * a.Hx : 0;
      float fx = 0.f, fy = 0.f;
      if (valid) {
        if (AMP == AMP_SEPARABLE) { fx = ax[kx] * ay[ky]; }
        else { fx = ax[kx]; fy = 1.f + qx[kx] + qy[ky]; }
      }
      const float expo = (float)a.expo;
      auto amp = [&](int kz) -> float {
        if (AMP == AMP_SEPARABLE) return fx * zt[kz];
        if (AMP == AMP_RECIP) return __fdividef(fx, fy + zt[kz]);
        return fx * pow_split(fy + zt[kz], expo);
      };
      // K-major row R1 (tiles of 128 rows are contiguous); K in draw order:
      // draw d (modes k2 = d and d + N2/2) fills K columns 4d .. 4d + 3, so
      // two draws make one 16-byte chunk
      const uint32_t rowoff = (uint32_t)((R1 >> 3) * Cfg::SBO1 + (R1 & 7) * 16);
      // the Philox round keys and stream in registers for the item's draws
      // (a batch's argument block lives in shared memory beside the operands)
      uint32_t kr[20];
#pragma unroll
      for (int r = 0; r < 20; ++r) kr[r] = a.ks[r];
      const uint32_t strm = a.stream;
      auto put = [&](const float* v, int chunk) {
        uint4 h, t;
        tc::split2(v[0], v[1], h.x, t.x);
        tc::split2(v[2], v[3], h.y, t.y);
        tc::split2(v[4], v[5], h.z, t.z);
        tc::split2(v[6], v[7], h.w, t.w);
        const uint32_t off = rowoff + chunk * Cfg::LBO1;
        *reinterpret_cast<uint4*>(AH + off) = h;
        *reinterpret_cast<uint4*>(AL + off) = t;
      };
#pragma unroll 2
      for (int d0 = 0; d0 < N2 / 2; d0 += 4) {  // four draws: two chunks
        float v[16];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int kz0 = s_k1 + N1 * (d0 + e);
          if (valid) {
            const uint64_t c = (uint64_t)l + mz * (uint64_t)kz0;
            const u32x4 o = philox4x32_10_ks({(uint32_t)c, (uint32_t)(c >> 32), strm, 0u}, kr);
            const float2 x0 = split_normals(o.x, o.y);
            const float2 x1 = split_normals(o.z, o.w);
            const float A0 = amp(kz0), A1 = amp(kz0 + N / 2);
            v[4 * e] = A0 * x0.x;
            v[4 * e + 1] = A0 * x0.y;
            v[4 * e + 2] = A1 * x1.x;
            v[4 * e + 3] = A1 * x1.y;
          } else {
            v[4 * e] = v[4 * e + 1] = v[4 * e + 2] = v[4 * e + 3] = 0.f;
          }
        }
        put(v, d0 / 2);
        put(v + 8, d0 / 2 + 1);
      }
    }
    tc::fence_smem_to_async();
    __syncthreads();
    // ---- stage 1 on the tensor cores ----
    if (tid == 0 && !wait_test) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int t = 0; t < Cfg::T1; ++t) {
#pragma unroll
        for (int s = 0; s < Cfg::K1 / 16; ++s) {
          const uint32_t ao = t * Cfg::TILE1 + s * 2 * Cfg::LBO1, bo = s * 2 * Cfg::LBO1;
          const uint64_t ah = tc::desc(sAH + ao, Cfg::LBO1, Cfg::SBO1);
          const uint64_t al = tc::desc(sAL + ao, Cfg::LBO1, Cfg::SBO1);
          const uint64_t bh = tc::desc(sB1H + bo, Cfg::LBO1, Cfg::SBO1);
          const uint64_t bl = tc::desc(sB1L + bo, Cfg::LBO1, Cfg::SBO1);
          const uint32_t d = tmem + t * Cfg::K1;
          tc::mma_bf16(d, ah, bh, ID1, s > 0 ? 1u : 0u);
          tc::mma_bf16(d, ah, bl, ID1, 1u);
          tc::mma_bf16(d, al, bh, ID1, 1u);
        }
      }
      tc::commit(bar);
    }
    ok = warp == 0 ? tc::mbar_wait(bar, phase, wait_ns) : true;  // one warp sleeps in the barrier
    phase ^= 1;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    tc::fence_after_sync();
    // ---- stage-1 rows back, twiddled, split into the MN-major stage-2
    //      operand: element (row n2 + N2 line, k), rows in 8-element M groups
    //      SBO2 apart (128-row tiles contiguous), K groups LBO2 apart,
    //      k = k1 (re) or N1 + k1 (im) ----
#pragma unroll 1
    for (int t = warp >> 2; t < Cfg::T1; t += Cfg::THREADS / 128) {
      const int R = t * 128 + q * 32 + lane;
      const int line = (R >> 3) % LB, k1 = (R & 7) + 8 * (R / (8 * LB));
      const float2* twk = tw2 + k1;  // e^{2 pi i n2 k1 / N} at twk[n2 N1]
      const uint32_t base = (uint32_t)(N2 * line / 8) * Cfg::SBO2 + (k1 >> 3) * Cfg::LBO2 + (k1 & 7) * 16;
      constexpr uint32_t IM = (N1 / 8) * Cfg::LBO2;  // im K groups follow the re ones
      const uint32_t col = tmem + ((uint32_t)(q * 32) << 16) + t * Cfg::K1;
#pragma unroll 2
      for (int g = 0; g < N2 / 8; ++g) {  // 8 n2: one M group, one 16-byte store per part
        float v[16];
        tc::tmem_ld<8>(col + 8 * g, v);           // re of n2 = 8 g ..
        tc::tmem_ld<8>(col + N2 + 8 * g, v + 8);  // im
        tc::tmem_wait_ld();
        uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const int n2 = 8 * g + e;
          const float2 w0 = twk[n2 * N1], w1 = twk[(n2 + 1) * N1];
          const float yr0 = v[e] * w0.x - v[8 + e] * w0.y, yi0 = v[e] * w0.y + v[8 + e] * w0.x;
          const float yr1 = v[e + 1] * w1.x - v[9 + e] * w1.y, yi1 = v[e + 1] * w1.y + v[9 + e] * w1.x;
          tc::split2(yr0, yr1, rh[e / 2], rl[e / 2]);
          tc::split2(yi0, yi1, ih[e / 2], il[e / 2]);
        }
        const uint32_t off = base + (uint32_t)g * Cfg::SBO2;
        *reinterpret_cast<uint4*>(AH + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(AL + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4*>(AH + off + IM) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4*>(AL + off + IM) = make_uint4(il[0], il[1], il[2], il[3]);
      }
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // ---- stage 2 on the tensor cores ----
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int t = 0; t < Cfg::T2; ++t) {
#pragma unroll
        for (int s = 0; s < Cfg::K2 / 16; ++s) {
          const uint32_t ao = t * Cfg::TILE2 + s * 2 * Cfg::LBO2, bo = s * 2 * Cfg::LBO1;
          const uint64_t ah = tc::desc(sAH + ao, Cfg::LBO2, Cfg::SBO2);
          const uint64_t al = tc::desc(sAL + ao, Cfg::LBO2, Cfg::SBO2);
          const uint64_t bh = tc::desc(sB2H + bo, Cfg::LBO1, Cfg::SBO2);
          const uint64_t bl = tc::desc(sB2L + bo, Cfg::LBO1, Cfg::SBO2);
          const uint32_t d = tmem + t * Cfg::K2;
          tc::mma_bf16(d, ah, bh, ID2, s > 0 ? 1u : 0u);
          tc::mma_bf16(d, ah, bl, ID2, 1u);
          tc::mma_bf16(d, al, bh, ID2, 1u);
        }
      }
      tc::commit(bar);
    }
    ok = warp == 0 ? tc::mbar_wait(bar, phase, wait_ns) : true;  // one warp sleeps in the barrier
    phase ^= 1;
    if (!__syncthreads_and(ok)) { ok = false; break; }
    tc::fence_after_sync();
    // ---- results X[n2 + N2 n1] of row (line, n2) into the z-major staging
    //      area (the operand region, free now): stage[z][line], NCH
    //      chunks of N1 / NCH consecutive n1 (z ranges of N / NCH) ----
    float2* stage = reinterpret_cast<float2*>(sm);
    constexpr int CN1 = N1 / Cfg::NCH, CZ = N / Cfg::NCH;
#pragma unroll 1
    for (int ch = 0; ch < Cfg::NCH && ch * CZ < Nz; ++ch) {
#pragma unroll 1
      for (int t = warp >> 2; t < Cfg::T2; t += Cfg::THREADS / 128) {
        const int R = t * 128 + q * 32 + lane;
        const int line = R / N2, n2 = R % N2;
        float v[2 * CN1];
        const uint32_t col = tmem + ((uint32_t)(q * 32) << 16) + t * Cfg::K2 + ch * CN1;
        tc::tmem_ld<CN1>(col, v);            // re of n1 = ch CN1 + ..
        tc::tmem_ld<CN1>(col + N1, v + CN1);  // im
        tc::tmem_wait_ld();
#pragma unroll
        for (int n1 = 0; n1 < CN1; ++n1)
          stage[(n2 + N2 * n1) * Cfg::STAGE_LD + line] = make_float2(v[n1], v[CN1 + n1]);
      }
      tc::fence_before_sync();
      __syncthreads();
      // ---- z < Nz of this chunk to global memory, LB consecutive lines per z
      {
        const int line = tid % LB;
        const int l = l0 + line;
        const bool valid = l < nlines;
        const int ky = valid ? l / a.Hx : 0, kx = valid ? l - ky * a.Hx : 0;
        const size_t zstride = (size_t)a.P[1] * a.Hpad;
        float2* dst = work + (size_t)ky * a.Hpad + kx + (size_t)(ch * CZ) * zstride;
        const int zn = min(CZ, Nz - ch * CZ);
        if (valid)
#pragma unroll 4
          for (int z = tid / LB; z < zn; z += Cfg::THREADS / LB)
            dst[(size_t)z * zstride] = stage[z * Cfg::STAGE_LD + line];
      }
      __syncthreads();  // the staging area: next chunk, or the next item's operands
    }
  }
  if (!ok) {
    // an MMA did not complete in time: report, then give it one more bounded
    // wait before the tensor memory it writes is released
    if (tid == 0) {
      atomicOr(a0.status, 1);  // the context's status word, shared by every member of a batch
      tc::mbar_wait(bar, phase ^ 1, wait_ns);
    }
    __syncthreads();
  }
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_free(tmem, Cfg::TMEM_COLS);
}

template <int N1, int N2, int LB, int NCH, int AMP>
__global__ void __launch_bounds__(256, 2) k_gen_z_tc(const GenArgs a) {
  gen_z_tc_body<N1, N2, LB, NCH, AMP, false>(a, nullptr, nullptr, nullptr, 0, 0);
}
template <int N1, int N2, int LB, int NCH, int AMP>
__global__ void __launch_bounds__(256, 2) k_gen_z_tc_batch(const GenArgs rep, const BatchMap m) {
  gen_z_tc_body<N1, N2, LB, NCH, AMP, true>(rep, m.args, m.items, m.start, m.n, m.total);
}

// One-time per device and kernel: the shared-memory opt-in; returns the SM
// count.  sms is the caller's per-kernel cache (one per instantiation).
constexpr int kMaxDev = 64;
template <class K>
cudaError_t tc_prepare(K kern, int smem, int (&sms)[kMaxDev], int* sms_out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  if (!sms[dev]) {
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
      return e;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
      return e;
    int n = 0;
    if ((e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    sms[dev] = n;
  }
  *sms_out = sms[dev];
  return cudaSuccess;
}

// bm == nullptr: one tile; else the batched kernel over bm->total items.
template <int N1, int N2, int LB, int NCH, int AMP>
cudaError_t launch_tc(const GenArgs& a, const BatchMap* bm, cudaStream_t s) {
  using Cfg = TcCfg<N1, N2, LB, NCH>;
  int sms = 0;
  cudaError_t e;
  // two resident CTAs per SM (registers, shared and tensor memory are sized for it)
  if (bm) {
    static int cache[kMaxDev] = {};
    auto kern = k_gen_z_tc_batch<N1, N2, LB, NCH, AMP>;
    if ((e = tc_prepare(kern, Cfg::SMEM, cache, &sms)) != cudaSuccess) return e;
    kern<<<std::min(bm->total, sms * Cfg::CTAS_PER_SM), Cfg::THREADS, Cfg::SMEM, s>>>(a, *bm);
  } else {
    static int cache[kMaxDev] = {};
    auto kern = k_gen_z_tc<N1, N2, LB, NCH, AMP>;
    if ((e = tc_prepare(kern, Cfg::SMEM, cache, &sms)) != cudaSuccess) return e;
    const int nitems = (a.Hx * a.P[1] + LB - 1) / LB;
    kern<<<std::min(nitems, sms * Cfg::CTAS_PER_SM), Cfg::THREADS, Cfg::SMEM, s>>>(a);
  }
  return cudaGetLastError();
}

template <int N1, int N2, int LB, int NCH>
cudaError_t launch_amp(const GenArgs& a, const BatchMap* bm, cudaStream_t s) {
  if (a.amp == AMP_SEPARABLE) return launch_tc<N1, N2, LB, NCH, AMP_SEPARABLE>(a, bm, s);
  if (a.amp == AMP_RECIP) return launch_tc<N1, N2, LB, NCH, AMP_RECIP>(a, bm, s);
  return launch_tc<N1, N2, LB, NCH, AMP_POW>(a, bm, s);
}

cudaError_t launch_any(const GenArgs& a, const BatchMap* bm, cudaStream_t s) {
  if (!a.status || a.spec != SPEC_PHILOX) return cudaErrorInvalidValue;
  switch (a.P[2]) {
    case 256: return launch_amp<16, 16, 16, 1>(a, bm, s);
    case 320: return launch_amp<8, 40, 32, 2>(a, bm, s);
    case 384: return launch_amp<16, 24, 16, 1>(a, bm, s);
    case 512: return launch_amp<16, 32, 16, 1>(a, bm, s);
    case 1024: return launch_amp<32, 32, 8, 2>(a, bm, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

// Line lengths with a tensor-core pass 1 (FP32 output, Philox spectrum):
// N = N1 x N2 = 16 x 16, 8 x 40, 16 x 24, 16 x 32, 32 x 32 (the others do
// not fit two CTAs per SM).
bool gen_z_tc_supported(int N) { return N == 256 || N == 320 || N == 384 || N == 512 || N == 1024; }

// Work items (256 / N1 lines each) of one realisation.
int gen_z_tc_items(const GenArgs& a) {
  if (!gen_z_tc_supported(a.P[2])) return -1;
  const int lb = a.P[2] == 320 ? 32 : (a.P[2] == 1024 ? 8 : 16);
  return (a.Hx * a.P[1] + lb - 1) / lb;
}

cudaError_t launch_gen_z_tc(const GenArgs& a, cudaStream_t s) { return launch_any(a, nullptr, s); }

cudaError_t launch_gen_z_tc_batch(const GenArgs& rep, const BatchMap& m, cudaStream_t s) {
  if (m.n < 1 || m.total < 1) return cudaErrorInvalidValue;
  return launch_any(rep, &m, s);
}

}  // namespace scarl
