// cov.cu -- streamed axis-covariance estimator for large fields: the sample
// covariance along each axis up to lag H,
//   C_d(h) = sum over point pairs (x, x + h e_d) of (f(x) - mu)(f(x + h e_d) - mu),
// accumulated in FP64.  (Stat_ScaRL's rebuild_Sk_FFT, SRC_F/Stat_ScaRL/
// statistics_RF.f90:258-462, windows each line and wraps it around; this
// estimator keeps the plain linear lag sum that a covariance model is checked
// against.)
//
// Each line of L_d values, centred by the global mean, is zero-padded to
// M = 2N >= L_d + H points (N a power of two or 320, 384, 640, 768, 1280,
// 1536, whichever is smallest) and transformed as one complex DFT of length N
// (even samples real, odd samples imaginary, then the even/odd split).  The
// power |Y_k|^2, k = 0..N, is summed over all lines of the block in the
// working precision and added to per-thread FP64 accumulators; one pass reads
// the field once.  The circular autocorrelation of the padded line,
//   S(h) = (1/M) sum_k |Y_k|^2 e^{-2 pi i k h / M},
// equals the linear lag sum for h <= M - L_d (Wiener-Khinchin); the cosine
// sum over k is formed in FP64 by k_cov_lags.
//
// FP32 fields whose lines and line groups start on 16-byte boundaries (L_0 a
// multiple of 4; column layouts with a group width B that is a multiple of 4
// and divides L_0) take the staged form: each line group's values are copied
// into a shared-memory input buffer by the TMA unit (one cp.async.bulk a line
// of x; for y and z lines one cp.async.bulk.tensor a box of B x up to 256
// rows through a tensor map of the field, issued by one thread and completing
// on an mbarrier with a bounded wait), and the next group's copies are issued
// as soon as the current group's first-stage values are in registers, so
// that the loads' latency overlaps the transform and the power sums; x lines
// are then transformed with lanes across lines, like the column layouts
// (fewer shared-memory bank conflicts than the line-fast layout).  Without a
// status word or a tensor map the same staging uses every thread's 16-byte
// cp.async.  Same values, same order: the staged and the direct form give
// identical sums.
#include <cuda.h>

#include <algorithm>
#include <cstring>

#include "fft_engine.cuh"
#include "scarl_internal.h"
#include "tc_sm100.cuh"

namespace scarl {

namespace {

// values per thread: 16 complex in FP32, 8 in FP64 (mixed lengths m 2^a:
// m times a power of two, eff_E)
template <typename T, int N> __host__ __device__ constexpr int cov_E() {
  return eff_E<N, (sizeof(T) == 4 ? 16 : 8)>();
}
// lines per block, for blocks of at most 256 threads in FP32 (two blocks per
// SM, whose barriers fall at different times) and 512 in FP64: ROW (x lines,
// lanes along a line) up to 32 lines, column layouts (lanes across lines) up
// to 16
template <typename T, int N, bool ROW> __host__ __device__ constexpr int cov_B() {
  constexpr int tpl = N / cov_E<T, N>();
  constexpr int cap = ROW ? 32 : 16;
  constexpr int nt = sizeof(T) == 4 ? 256 : 512;
  return (nt / tpl) < 1 ? 1 : ((nt / tpl) > cap ? cap : nt / tpl);
}
template <typename T, int N, bool ROW> __host__ __device__ constexpr int cov_threads() {
  return cov_B<T, N, ROW>() * (N / cov_E<T, N>());
}
// resident blocks asked of the compiler: 512 threads per SM (128 registers a
// thread: room for the FP32 prefetch of the next lines), at most 32 blocks
template <typename T, int N, bool ROW> __host__ __device__ constexpr int cov_minb() {
  constexpr int per_sm = 512;
  return (per_sm / cov_threads<T, N, ROW>()) > 32 ? 32
         : (per_sm / cov_threads<T, N, ROW>()) < 1 ? 1 : per_sm / cov_threads<T, N, ROW>();
}
// complex slots of a block's line region: the transform's scratch, then the
// power rows (B lines N + 1 apart); FP32 twiddles follow it
template <typename T, int N, bool ROW> __host__ __device__ constexpr int cov_rows() {
  constexpr int fft = cov_B<T, N, ROW>() * line_slots<N, cov_E<T, N>()>();
  constexpr int pw = cov_B<T, N, ROW>() * (N + 1);
  return fft > pw ? fft : pw;
}
struct CovGeom {
  const void* f;
  int n;          // points per line (L_d)
  int64_t na;     // lines along the fastest other axis
  int64_t sa, sb; // element strides of the two other axes
  int64_t st;     // element stride along the line
  int64_t nlines;
  double mu;
  const void* tw;  // e^{2 pi i m / M}, m < M, working precision
  double* partial; // gridDim.x * (N + 1)
  int* status;     // device word, bit 0 set when a bounded copy wait expired (TMA form)
  int box;         // TMA form, column layouts: rows a tensor box (<= 256)
  int dir;         // line axis (0 x, 1 y, 2 z)
};

// Staged form: input buffer floats (B lines of L values 16 bytes more than L
// apart, or L rows of B values, rounded up to whole tensor boxes of `box`
// rows in the TMA form); 16 bytes for the copies' mbarrier follow it.
template <int N, bool ROW> __host__ __device__ constexpr int cov_in_floats(int L, int box = 1) {
  return ROW ? cov_B<float, N, ROW>() * (L + 4) : cov_B<float, N, ROW>() * ((L + box - 1) / box) * box;
}
// Byte offset of the staged form's input buffer (after the transform's rows
// and the twiddles), 128-byte aligned for the tensor copies.
template <typename T, int N, bool ROW> __host__ __device__ constexpr int cov_in_off() {
  return ((cov_rows<T, N, ROW>() + 2 * N) * (int)sizeof(cplx_t<T>) + 127) / 128 * 128;
}

constexpr uint64_t kCopyWaitNs = 1000000000ull;  // 1 s per group's copies (TMA form)

// ASYNC: the staged form.  TMA (with ASYNC): the group's copies are bulk
// copies by the TMA unit issued by thread 0 (one cp.async.bulk a line of x,
// one cp.async.bulk.tensor a box of a column group through tmap) completing
// on an mbarrier, instead of every thread's 16-byte cp.async.
template <typename T, int N, bool ROW, bool ASYNC = false, bool TMA = false>
__global__ void __launch_bounds__(cov_threads<T, N, ROW>(), cov_minb<T, N, ROW>())
    k_axis_power(const CovGeom g, const __grid_constant__ CUtensorMap tmap) {
  using C = cplx_t<T>;
  constexpr int E = cov_E<T, N>();
  constexpr int B = cov_B<T, N, ROW>();
  constexpr int TPL = N / E;
  constexpr int NT = B * TPL;
  constexpr int QB = (N + NT) / NT;  // bins per thread (bins 0..N)
  // lanes along a line (line-fast shared layout) only in the direct form of
  // x lines; the staged form transforms x lines like the column layouts
  // (lanes across lines), reading them from a line-major input buffer
  constexpr bool LROW = ROW && !ASYNC;
  constexpr SmemOrder O = LROW ? SmemOrder::LineFast : SmemOrder::BatchFast;
  constexpr int LS = LROW ? line_slots<N, E>() : 0;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int b = LROW ? (int)threadIdx.x / TPL : (int)threadIdx.x % B;
  const int t = LROW ? (int)threadIdx.x % TPL : (int)threadIdx.x / B;
  const T* f = static_cast<const T*>(g.f);
  // FP32: the 2N twiddles e^{2 pi i m / M} in shared memory (once per block)
  constexpr bool TWS = sizeof(T) == 4;
  const C* tw = static_cast<const C*>(g.tw);
  if constexpr (TWS) {
    C* tws = sm + cov_rows<T, N, ROW>();
    for (int i = (int)threadIdx.x; i < 2 * N; i += (int)blockDim.x) tws[i] = __ldg(tw + i);
    __syncthreads();
    tw = tws;
  }
  double acc[QB];
#pragma unroll
  for (int q = 0; q < QB; ++q) acc[q] = 0.0;
  const int64_t ngroups = (g.nlines + B - 1) / B;
  const T mu = (T)g.mu;
  // First-stage inputs of this thread for the lines of group grp, centred and
  // zero-padded: dst[q R1 + r] = (x[2k], x[2k + 1]), k = t + TPL q + r N / R1.
  // In FP32 the next group's inputs are fetched into registers before the
  // current group's transform, so their global-memory latency overlaps it
  // (FP64, and lines of more than 20 values a thread or one thread a line,
  // have no registers to spare for it).
  constexpr bool PF = sizeof(T) == 4 && E <= 20 && TPL > 1;
  constexpr int R1 = StagePlan<N, E>::radix(0);
  auto fetch = [&](int64_t grp, C* dst) {
    const int64_t l = grp * B + b;
    const bool valid = l < g.nlines;
    const int64_t base = valid ? (l % g.na) * g.sa + (l / g.na) * g.sb : 0;
    auto val = [&](int i) -> T {
      if (!valid || i >= g.n) return T(0);
      return __ldg(f + base + (int64_t)i * g.st) - mu;
    };
#pragma unroll
    for (int q = 0; q < E / R1; ++q)
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        const int k = t + TPL * q + r * (N / R1);
        dst[q * R1 + r] = mk(val(2 * k), val(2 * k + 1));
      }
  };
  // staged form: the group's values in the input buffer after the twiddles
  float* inb = reinterpret_cast<float*>(smraw + cov_in_off<T, N, ROW>());
  // TMA form: the mbarrier after the input buffer (128-byte aligned region)
  const uint32_t cbar = tc::smem_u32(inb + (ROW ? B * (g.n + 4) : ((g.n + g.box - 1) / g.box) * g.box * B));
  auto issue_tma = [&](int64_t grp) {  // thread 0: the group's bulk copies
    const int64_t l0 = grp * B;
    tc::fence_smem_to_async();
    if constexpr (ROW) {
      const int nv = (int)(g.nlines - l0 < B ? g.nlines - l0 : B);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cbar),
                   "r"((uint32_t)(nv * g.n * 4))
                   : "memory");
      for (int bb = 0; bb < nv; ++bb) {
        const int64_t l = l0 + bb;
        const float* src = static_cast<const float*>(g.f) + (l % g.na) * g.sa + (l / g.na) * g.sb;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                tc::smem_u32(inb + bb * (g.n + 4))),
            "l"(src), "r"((uint32_t)(g.n * 4)), "r"(cbar)
            : "memory");
      }
    } else {
      const int nbox = (g.n + g.box - 1) / g.box;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cbar),
                   "r"((uint32_t)(nbox * g.box * B * 4))
                   : "memory");
      // coordinates (x, y, z) of the box: x = first line's x (a multiple of
      // B, so 16-byte aligned), the line axis stepping by box rows
      const int x0 = (int)(l0 % g.na), o = (int)(l0 / g.na);
      const bool ydir = g.dir == 1;  // y lines: the other axis is z; z lines: y
      for (int r = 0; r < nbox; ++r) {
        const int c1 = ydir ? r * g.box : o, c2 = ydir ? o : r * g.box;
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tc::smem_u32(inb + r * g.box * B)),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(x0), "r"(c1), "r"(c2), "r"(cbar)
            : "memory");
      }
    }
  };
  auto issue = [&](int64_t grp) {  // 16-byte copies of group grp (every thread)
    const int64_t l0 = grp * B;
    if constexpr (ROW) {
      const int cpl = g.n / 4;  // chunks a line
      for (int c = (int)threadIdx.x; c < B * cpl; c += (int)blockDim.x) {
        const int bb = c / cpl, qq = c - bb * cpl;
        const int64_t l = l0 + bb;
        if (l >= g.nlines) continue;
        const float* src = static_cast<const float*>(g.f) + (l % g.na) * g.sa + (l / g.na) * g.sb + 4 * qq;
        cp_async16(inb + bb * (g.n + 4) + 4 * qq, src);  // lines 16 bytes more than L apart
      }
    } else {
      constexpr int cpr = B >= 4 ? B / 4 : 1;  // chunks a row (staged_ok: B a multiple of 4)
      const float* base = static_cast<const float*>(g.f) + (l0 % g.na) * g.sa + (l0 / g.na) * g.sb;
      for (int c = (int)threadIdx.x; c < g.n * cpr; c += (int)blockDim.x) {
        const int i = c / cpr, qq = c - i * cpr;
        cp_async16(inb + i * B + 4 * qq, base + (int64_t)i * g.st + 4 * qq);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  auto fetch_staged = [&](int64_t grp, C* dst) {
    const int64_t l = grp * B + b;
    const bool valid = l < g.nlines;
    auto val = [&](int i) -> T {
      if (!valid || i >= g.n) return T(0);
      return (T)(ROW ? inb[b * (g.n + 4) + i] : inb[i * B + b]) - mu;
    };
#pragma unroll
    for (int q = 0; q < E / R1; ++q)
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        const int k = t + TPL * q + r * (N / R1);
        dst[q * R1 + r] = mk(val(2 * k), val(2 * k + 1));
      }
  };
  C nxt[PF && !ASYNC ? E : 1];
  uint32_t cphase = 0;
  bool pending = false;  // thread 0, TMA form: copies issued and not yet waited for
  if constexpr (TMA) {
    if (threadIdx.x == 0) tc::mbar_init(cbar, 1);
    __syncthreads();
    if (threadIdx.x == 0 && (int64_t)blockIdx.x < ngroups) {
      issue_tma(blockIdx.x);
      pending = true;
    }
  } else if constexpr (ASYNC) {
    issue(blockIdx.x);
  } else if constexpr (PF) {
    fetch(blockIdx.x, nxt);
  }
  for (int64_t grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    C cur[E];
    if constexpr (TMA) {
      const bool ok = tc::mbar_wait(cbar, cphase, kCopyWaitNs);
      if (!__syncthreads_and(ok)) break;  // reported after the loop
      cphase ^= 1;
      if (threadIdx.x == 0) pending = false;
      fetch_staged(grp, cur);
      tc::fence_smem_to_async();  // this thread's reads before the next copies' writes
      __syncthreads();            // every thread has read the input buffer
      if (threadIdx.x == 0 && grp + gridDim.x < ngroups) {
        issue_tma(grp + gridDim.x);
        pending = true;
      }
    } else if constexpr (ASYNC) {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      __syncthreads();  // every thread's copies of this group have landed
      fetch_staged(grp, cur);
      __syncthreads();  // every thread has read the input buffer
      if (grp + gridDim.x < ngroups) issue(grp + gridDim.x);
    } else if constexpr (PF) {
#pragma unroll
      for (int i = 0; i < E; ++i) cur[i] = nxt[i];
      if (grp + gridDim.x < ngroups) fetch(grp + gridDim.x, nxt);
    } else {
      fetch(grp, cur);
    }
    auto load = [&](int j, C* v) {
      const int q = (j - t) / TPL;
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = cur[q * R1 + r];
    };
    constexpr int RL = last_radix<N, E>();
    // outputs go straight to shared memory (line b at b (N + 1): the odd
    // stride spreads the lines of a column layout, whose lanes store the same
    // j of different lines, over the banks), after every thread has left the
    // transform's shared-memory reads
    auto store = [&](int j, const C* o) {
#pragma unroll
      for (int r = 0; r < RL; ++r) sm[b * (N + 1) + j + r * (N / RL)] = o[r];
    };
    line_ifft<C, N, E, O, B, LS, true, 2>(sm, b, t, tw, load, store);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int k = (int)threadIdx.x + NT * q;
      if (k > N) break;
      const C w = tw[k];
      T s = T(0);
      for (int bb = 0; bb < B; ++bb) {
        const C zk = sm[bb * (N + 1) + (k == N ? 0 : k)];
        const C zc = cconj(sm[bb * (N + 1) + (k == 0 || k == N ? 0 : N - k)]);
        const C e = mk((zk.x + zc.x) * T(0.5), (zk.y + zc.y) * T(0.5));
        // (zk - zc) / (2i)
        const C od = mk((zk.y - zc.y) * T(0.5), -(zk.x - zc.x) * T(0.5));
        const C y = cadd(e, cmul(w, od));
        s += y.x * y.x + y.y * y.y;
      }
      acc[q] += (double)s;
    }
    __syncthreads();
  }
  if constexpr (TMA) {
    // a group's copies did not land in time: report, and give them one more
    // bounded wait (they write this block's shared memory)
    if (threadIdx.x == 0 && pending) {
      atomicOr(g.status, 1);
      tc::mbar_wait(cbar, cphase, kCopyWaitNs);
    }
  }
#pragma unroll
  for (int q = 0; q < QB; ++q) {
    const int k = (int)threadIdx.x + NT * q;
    if (k <= N) g.partial[(int64_t)blockIdx.x * (N + 1) + k] = acc[q];
  }
}

template <typename T, int N, bool ROW> size_t cov_smem() {
  return ((size_t)cov_rows<T, N, ROW>() + (sizeof(T) == 4 ? 2 * N : 0)) * sizeof(cplx_t<T>);
}
// The staged form's dynamic shared memory: rows, twiddles, the input buffer
// and its mbarrier.
template <typename T, int N, bool ROW> size_t cov_smem_staged(const CovGeom& g) {
  return (size_t)cov_in_off<T, N, ROW>() + (size_t)cov_in_floats<N, ROW>(g.n, g.box) * 4 + 16;
}

// The staged form serves FP32 lines whose copies are 16-byte aligned: L_0 a
// multiple of 4; a column layout's group width B a multiple of 4 dividing
// L_0 (groups never wrap across x); the buffer fitting two blocks an SM.
template <typename T, int N, bool ROW> bool staged_ok(const CovGeom& g, int L0) {
  if (sizeof(T) != 4 || L0 % 4 != 0) return false;
  constexpr int B = cov_B<T, N, ROW>();
  if (!ROW && (B % 4 != 0 || L0 % B != 0)) return false;
  return cov_smem_staged<T, N, ROW>(g) <= 110 * 1024;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  // looked up once (thread-safe static initialisation)
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
    return nullptr;
  }();
  return fn;
}

// The tensor map of a column layout's groups: the field as an L0 x L1 x L2
// FP32 tensor, boxes of B x box rows along the line axis (x offsets of a
// group are multiples of B >= 4 floats: 16-byte aligned).
bool column_tmap(const CovGeom& g, const int L[3], int B, CUtensorMap* tm) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc || g.dir == 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)L[0], (cuuint64_t)L[1], (cuuint64_t)L[2]};
  const cuuint64_t strides[2] = {(cuuint64_t)L[0] * 4, (cuuint64_t)L[0] * L[1] * 4};
  const cuuint32_t box[3] = {(cuuint32_t)B, (cuuint32_t)(g.dir == 1 ? g.box : 1),
                             (cuuint32_t)(g.dir == 2 ? g.box : 1)};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(g.f), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T, int N, bool ROW, bool ASYNC, bool TMA>
cudaError_t run_power_k(CovGeom g, const CUtensorMap& tm, int want_blocks, int* blocks, cudaStream_t s) {
  auto kern = k_axis_power<T, N, ROW, ASYNC, TMA>;
  const size_t smem = ASYNC ? cov_smem_staged<T, N, ROW>(g) : cov_smem<T, N, ROW>();
  const int threads = cov_threads<T, N, ROW>();
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t ngroups = (g.nlines + cov_B<T, N, ROW>() - 1) / cov_B<T, N, ROW>();
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>(ngroups, (int64_t)std::max(per_sm, 1) * sms));
  if (blocks && want_blocks < 0) {  // query only
    *blocks = nb;
    return cudaSuccess;
  }
  const int grid = want_blocks > 0 ? want_blocks : nb;
  kern<<<grid, threads, smem, s>>>(g, tm);
  return cudaGetLastError();
}

// Form of a launch: staged where staged_ok and the field pointer is 16-byte
// aligned, its copies by the TMA unit where the launch has a status word and
// (column layouts) a tensor map; the blocks query (g.f == nullptr) sizes the
// staged form, whose grid every form can run (the grid is only the stride
// of the group loop).
template <typename T, int N, bool ROW>
cudaError_t run_power(CovGeom g, const int* L, int want_blocks, int* blocks, cudaStream_t s) {
  CUtensorMap tm;
  std::memset(&tm, 0, sizeof tm);
  if constexpr (sizeof(T) == 4) {
    const bool aligned = g.f == nullptr || (reinterpret_cast<uintptr_t>(g.f) & 15) == 0;
    if (staged_ok<T, N, ROW>(g, L[0]) && aligned) {
      if (!blocks && g.status && (ROW || column_tmap(g, L, cov_B<T, N, ROW>(), &tm)))
        return run_power_k<T, N, ROW, true, true>(g, tm, want_blocks, blocks, s);
      return run_power_k<T, N, ROW, true, false>(g, tm, want_blocks, blocks, s);
    }
  }
  return run_power_k<T, N, ROW, false, false>(g, tm, want_blocks, blocks, s);
}

template <typename T, bool ROW>
cudaError_t run_power_n(int N, CovGeom g, const int* L, int want_blocks, int* blocks, cudaStream_t s) {
  switch (N) {
    case 4: return run_power<T, 4, ROW>(g, L, want_blocks, blocks, s);
    case 8: return run_power<T, 8, ROW>(g, L, want_blocks, blocks, s);
    case 16: return run_power<T, 16, ROW>(g, L, want_blocks, blocks, s);
    case 32: return run_power<T, 32, ROW>(g, L, want_blocks, blocks, s);
    case 64: return run_power<T, 64, ROW>(g, L, want_blocks, blocks, s);
    case 128: return run_power<T, 128, ROW>(g, L, want_blocks, blocks, s);
    case 256: return run_power<T, 256, ROW>(g, L, want_blocks, blocks, s);
    case 512: return run_power<T, 512, ROW>(g, L, want_blocks, blocks, s);
    case 1024: return run_power<T, 1024, ROW>(g, L, want_blocks, blocks, s);
    case 2048: return run_power<T, 2048, ROW>(g, L, want_blocks, blocks, s);
    case 320: return run_power<T, 320, ROW>(g, L, want_blocks, blocks, s);
    case 384: return run_power<T, 384, ROW>(g, L, want_blocks, blocks, s);
    case 640: return run_power<T, 640, ROW>(g, L, want_blocks, blocks, s);
    case 768: return run_power<T, 768, ROW>(g, L, want_blocks, blocks, s);
    case 1280: return run_power<T, 1280, ROW>(g, L, want_blocks, blocks, s);
    case 1536: return run_power<T, 1536, ROW>(g, L, want_blocks, blocks, s);
    default: return cudaErrorInvalidValue;
  }
}

CovGeom geom(const void* f, const int L[3], int dir, double mu, const void* tw, double* partial) {
  CovGeom g;
  g.f = f;
  g.n = L[dir];
  g.mu = mu;
  g.tw = tw;
  g.partial = partial;
  g.status = nullptr;
  g.dir = dir;
  g.box = L[dir] < 256 ? L[dir] : 256;
  const int64_t L0 = L[0], L1 = L[1], L2 = L[2];
  if (dir == 0) {  // x lines, consecutive in memory
    g.na = L1; g.sa = L0; g.sb = L0 * L1; g.st = 1; g.nlines = L1 * L2;
  } else if (dir == 1) {  // y lines, consecutive x in a group
    g.na = L0; g.sa = 1; g.sb = L0 * L1; g.st = L0; g.nlines = L0 * L2;
  } else {  // z lines
    g.na = L0; g.sa = 1; g.sb = L0; g.st = L0 * L1; g.nlines = L0 * L1;
  }
  return g;
}

cudaError_t dispatch(int dt, int dir, int N, CovGeom g, const int* L, int want, int* blocks, cudaStream_t s) {
  if (dt == 8) return dir == 0 ? run_power_n<double, true>(N, g, L, want, blocks, s)
                               : run_power_n<double, false>(N, g, L, want, blocks, s);
  return dir == 0 ? run_power_n<float, true>(N, g, L, want, blocks, s)
                  : run_power_n<float, false>(N, g, L, want, blocks, s);
}

// P_k = sum over blocks of the partial power (one thread per bin).
__global__ void k_cov_bins(const double* __restrict__ partial, int nblocks, int nbins,
                           double* __restrict__ bins) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nbins) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partial[(int64_t)b * nbins + k];
  bins[k] = s;
}

// S(h) = (1/M) [P_0 + (-1)^h P_N + 2 sum_{k=1}^{N-1} P_k cos(2 pi k h / M)],
// one block per lag, FP64.
__global__ void k_cov_lags(const double* __restrict__ bins, int N, const double2* __restrict__ tw64,
                           double* __restrict__ S) {
  const int h = blockIdx.x;
  const int M = 2 * N;
  double s = 0.0;
  for (int k = 1 + threadIdx.x; k < N; k += blockDim.x)
    s += bins[k] * tw64[(int)(((int64_t)k * h) % M)].x;
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0)
      S[h] = (bins[0] + ((h & 1) ? -bins[N] : bins[N]) + 2.0 * s) / (double)M;
  }
}

}  // namespace

int axis_power_blocks(int dt, const int L[3], int dir, int N) {
  int nb = -1;
  CovGeom g = geom(nullptr, L, dir, 0.0, nullptr, nullptr);
  if (dispatch(dt, dir, N, g, L, -1, &nb, nullptr) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return nb;
}

cudaError_t launch_axis_power(int dt, const void* f, const int L[3], int dir, int N, double mu,
                              const void* tw, double* partial, int nblocks, cudaStream_t s, int* status) {
  CovGeom g = geom(f, L, dir, mu, tw, partial);
  g.status = status;
  return dispatch(dt, dir, N, g, L, nblocks, nullptr, s);
}

cudaError_t launch_cov_lags(const double* partial, int nblocks, int N, int maxlag,
                            const double* tw64, double* bins, double* S, cudaStream_t s) {
  k_cov_bins<<<(N + 1 + 255) / 256, 256, 0, s>>>(partial, nblocks, N + 1, bins);
  k_cov_lags<<<maxlag + 1, 256, 0, s>>>(bins, N, reinterpret_cast<const double2*>(tw64), S);
  return cudaGetLastError();
}

}  // namespace scarl
