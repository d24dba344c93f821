// noalloc.cu -- scarl_gen_padded_noalloc: the padded periodic generator of
// scarl_gen_padded for callers that cannot allocate GPU memory, e.g. a host
// code whose device memory is entirely owned by its own pool allocator, or a
// time-critical loop that must not call cudaMalloc (which can block on or
// synchronise the device) once it is running.
//
// All scratch (the half-spectrum intermediate, twiddle and spectrum tables,
// the partial sums of the spectral normalisation) lives in one file-scope
// device array of kScratchBytes, reserved on every GPU that loads the library
// for the life of the process.  Each call carves it up afresh; nothing in it
// needs to start at zero, since every value a kernel reads is written earlier
// in the same call.  All calls share the array, so calls whose GPU work
// overlaps in time (other host threads, other streams) race: serialise them.
//
// The array's device address is looked up once per device (the first call
// made with that device current), so make that first call before any CUDA
// stream capture.  The call itself allocates nothing: no cudaMalloc,
// cudaFree or allocating library routine.  Each call uploads its spectrum
// and twiddle tables from host memory with cudaMemcpyAsync, and with
// normalise = 1 it also waits on the stream for the FP64 spectral sum (the
// host blocks until the GPU has reached that point).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/scarl.h"
#include "host_maps.h"
#include "scarl_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void* g_dev_addr[kMaxDevices] = {};

int say(char* msg, size_t len, int code, const char* text) {
  if (msg && len) std::snprintf(msg, len, "%s", text);
  return code;
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }

double freq(int k, int P, double dx) {
  const int s = (2 * k <= P) ? k : k - P;
  return (double)s / ((double)P * dx);
}

}  // namespace

extern "C" int scarl_gen_padded_noalloc(void* out, int dtype, const int Np[3], const int pad[3],
                                        const double xStep[3], const double corrL[3],
                                        int corrMod, double nu, int normalise, uint64_t seed,
                                        uint32_t stream, void* cuda_stream, char* msg,
                                        size_t msg_len) {
  using namespace scarl;
  if (!out || !Np || !xStep || !corrL) return say(msg, msg_len, SCARL_EINVAL, "null argument");
  if (dtype != SCARL_F32 && dtype != SCARL_F64)
    return say(msg, msg_len, SCARL_EINVAL, "dtype must be SCARL_F32 or SCARL_F64");
  if (corrMod < 1 || corrMod > 3 || (corrMod == SCARL_CM_VON_KARMAN && !(nu > 0.0)))
    return say(msg, msg_len, SCARL_EINVAL, "corrMod must be 1, 2 (with nu > 0) or 3");
  int P[3];
  for (int d = 0; d < 3; ++d) {
    if (Np[d] < 1 || !(xStep[d] > 0.0) || !(corrL[d] > 0.0))
      return say(msg, msg_len, SCARL_EINVAL, "Np >= 1, xStep > 0 and corrL > 0 required");
    int p = 1;  // default: 2^ceil(log2(2 Np)), as scarl_gen_padded
    while (p < 2 * Np[d]) p <<= 1;
    P[d] = (pad && pad[d] > 0) ? pad[d] : p;
    if (!fft_length_supported(P[d]))
      return say(msg, msg_len, SCARL_EUNSUPPORTED,
                 "padded grid lengths must lie in [8, 2048] and be a power of two or 3, 5 or 7 "
                 "times a power of two >= 16");
    if (P[d] < Np[d]) return say(msg, msg_len, SCARL_EINVAL, "padded grid smaller than the tile");
  }
  const cudaStream_t s = (cudaStream_t)cuda_stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return say(msg, msg_len, SCARL_EDEVICE, "no usable current CUDA device");
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, out) != cudaSuccess ||
      (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) ||
      (pa.type == cudaMemoryTypeDevice && pa.device != dev)) {
    cudaGetLastError();
    return say(msg, msg_len, SCARL_EINVAL, "out must be device memory of the current GPU");
  }

  // ---- carve the fixed scratch array ----
  const int dt = dtype;
  const int Hx = P[0] / 2 + 1;
  const int Hpad = (Hx + 15) / 16 * 16;
  const int nb = spectrum_sum_blocks();
  const int ntab = Hx + P[1] + P[2];
  size_t off = 0;
  const size_t o_work = off;
  off += align256((size_t)Hpad * P[1] * Np[2] * 2 * dt);
  const size_t o_tw = off;
  off += align256((size_t)(P[0] + P[1] + P[2]) * 2 * dt);
  const size_t o_tab = off;
  off += align256((size_t)2 * ntab * dt);
  const size_t o_raw = off;
  off += align256((size_t)ntab * 8);
  const size_t o_part = off;
  off += align256((size_t)nb * 8);
  if (off > kScratchBytes) {
    char m[200];
    std::snprintf(m, sizeof m,
                  "request needs %zu bytes of scratch; the fixed scratch array holds %zu "
                  "(64 MiB): use smaller Np[2] or padded grid, or scarl_gen_padded",
                  off, kScratchBytes);
    return say(msg, msg_len, SCARL_EINVAL, m);
  }

  // ---- the array's address on this device (looked up once per device) ----
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return say(msg, msg_len, SCARL_EDEVICE, "cudaGetSymbolAddress of the scratch array failed");
      }
      g_dev_addr[dev] = p;
    }
    base = static_cast<unsigned char*>(g_dev_addr[dev]);
  }

  // ---- host tables (FP64), the same spectra as scarl_gen_padded ----
  const int n[3] = {Hx, P[1], P[2]};
  std::vector<double> raw;  // Gaussian: r_d(k); Matern: q_d(k)
  raw.reserve(ntab);
  double craw2 = 0.0, expo = 0.0;
  int amp;
  if (corrMod == SCARL_CM_GAUSSIAN) {
    amp = AMP_SEPARABLE;
    for (int d = 0; d < 3; ++d) {
      const double dk = 1.0 / ((double)P[d] * xStep[d]);
      for (int k = 0; k < n[d]; ++k) {
        const double f = freq(k, P[d], xStep[d]);
        raw.push_back(std::sqrt(corrL[d] * dk) * std::exp(-M_PI * corrL[d] * corrL[d] * f * f / 2.0));
      }
    }
  } else {
    const double v = (corrMod == SCARL_CM_EXPONENTIAL) ? 0.5 : nu;
    const double sc = std::tgamma(v) / (2.0 * std::sqrt(M_PI) * std::tgamma(v + 0.5));
    double a[3], dk3 = 1.0;
    for (int d = 0; d < 3; ++d) {
      a[d] = corrL[d] * sc;
      dk3 *= 1.0 / ((double)P[d] * xStep[d]);
    }
    craw2 = 8.0 * std::pow(M_PI, 1.5) * std::tgamma(v + 1.5) / std::tgamma(v) * a[0] * a[1] * a[2] * dk3;
    expo = -(v + 1.5) / 2.0;
    amp = (v == 0.5) ? AMP_RECIP : AMP_POW;
    for (int d = 0; d < 3; ++d)
      for (int k = 0; k < n[d]; ++k) {
        const double f = freq(k, P[d], xStep[d]);
        raw.push_back(4.0 * M_PI * M_PI * a[d] * a[d] * f * f);
      }
  }
  const double* r0 = reinterpret_cast<const double*>(base + o_raw);

  GenArgs ga;
  std::memset(&ga, 0, sizeof ga);
  for (int d = 0; d < 3; ++d) {
    ga.P[d] = P[d];
    ga.Nout[d] = Np[d];
  }
  ga.Hx = Hx;
  ga.Hpad = Hpad;
  ga.amp = amp;
  ga.expo = expo;

  // FP64 spectral normalisation on the GPU
  double norm = 1.0;
  if (normalise) {
    if (cudaMemcpyAsync(base + o_raw, raw.data(), raw.size() * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return say(msg, msg_len, SCARL_EDEVICE, "table upload failed");
    ga.qx = r0;
    ga.qy = r0 + n[0];
    ga.qz = r0 + n[0] + n[1];
    double* part = reinterpret_cast<double*>(base + o_part);
    if (launch_spectrum_sum(ga, r0, r0 + n[0], r0 + n[0] + n[1], craw2, part, nb, s) != cudaSuccess)
      return say(msg, msg_len, SCARL_EDEVICE, "spectrum sum launch failed");
    std::vector<double> h(nb);
    if (cudaMemcpyAsync(h.data(), part, (size_t)nb * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return say(msg, msg_len, SCARL_EDEVICE, "spectrum sum readback failed");
    norm = 0.0;
    for (double v : h) norm += v;
    if (!(norm > 0.0)) return say(msg, msg_len, SCARL_EINVAL, "spectrum sums to zero on this grid");
  }

  // tables in the pass precision: [ax | ay az (separable) or qx qy qz]
  const double inv = 1.0 / std::sqrt(norm);
  std::vector<double> tab;
  tab.reserve(2 * ntab);
  for (int k = 0; k < Hx; ++k) {
    const double g = (k == 0 || 2 * k == P[0]) ? 1.0 : M_SQRT1_2;
    tab.push_back((amp == AMP_SEPARABLE ? raw[k] : std::sqrt(craw2)) * g * inv);
  }
  if (amp == AMP_SEPARABLE) {
    tab.insert(tab.end(), raw.begin() + n[0], raw.end());
  } else {
    tab.insert(tab.end(), raw.begin(), raw.end());
  }
  // twiddles e^{2 pi i m / P_d}
  std::vector<double> tw;
  tw.reserve(2 * (size_t)(P[0] + P[1] + P[2]));
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int d = 0; d < 3; ++d)
    for (int m = 0; m < P[d]; ++m) {
      const long double ang = 2.0L * pi * (long double)m / (long double)P[d];
      tw.push_back((double)cosl(ang));
      tw.push_back((double)sinl(ang));
    }
  unsigned char* tabp = base + o_tab;
  unsigned char* twp = base + o_tw;
  cudaError_t e;
  if (dt == SCARL_F64) {
    e = cudaMemcpyAsync(tabp, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twp, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice, s);
  } else {
    std::vector<float> tf(tab.begin(), tab.end()), wf(tw.begin(), tw.end());
    e = cudaMemcpyAsync(tabp, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twp, wf.data(), wf.size() * 4, cudaMemcpyHostToDevice, s);
    // pageable sources: the copies have read the vectors when they return
  }
  if (e != cudaSuccess) return say(msg, msg_len, SCARL_EDEVICE, "table upload failed");

  const size_t es = (size_t)dt;
  ga.spec = SPEC_PHILOX;
  ga.ax = tabp;
  if (amp == AMP_SEPARABLE) {
    ga.ay = tabp + (size_t)Hx * es;
    ga.az = tabp + (size_t)(Hx + P[1]) * es;
    ga.qx = ga.qy = ga.qz = nullptr;
  } else {
    ga.ay = ga.az = nullptr;
    ga.qx = tabp + (size_t)Hx * es;
    ga.qy = tabp + (size_t)(2 * Hx) * es;
    ga.qz = tabp + (size_t)(2 * Hx + P[1]) * es;
  }
  ga.tw_x = twp;
  ga.tw_y = twp + (size_t)P[0] * 2 * es;
  ga.tw_z = twp + (size_t)(P[0] + P[1]) * 2 * es;
  ga.work = base + o_work;
  ga.k0 = (uint32_t)seed;
  ga.k1 = (uint32_t)(seed >> 32);
  ga.stream = stream;
  ga.epi.mode = 0;
  ga.epi.out = out;
  for (int pass = 1; pass <= 3; ++pass)
    if (launch_gen_pass(dt, pass, ga, s) != cudaSuccess)
      return say(msg, msg_len, SCARL_EDEVICE, "generator launch failed");
  return say(msg, msg_len, SCARL_OK, "");
}
