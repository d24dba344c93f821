// gen_padded.cu -- dispatch of the padded periodic-grid generator passes
// (kernels in gen_kernels.cuh, variants in gen_launch.cuh, instantiated per
// precision and line length by gen_inst.cu) and the FP64 spectral
// normalisation sum.
#include "gen_launch.cuh"

namespace scarl {

// Defined and explicitly instantiated in gen_inst.cu.
template <typename T, int N>
cudaError_t run_pass_len(int pass, int v, const GenArgs& a, const BatchMap* bm, int* nb,
                         cudaStream_t s);

template <typename T>
static cudaError_t run_pass_t(int pass, int v, const GenArgs& a, const BatchMap* bm, int* nb,
                              cudaStream_t s) {
  const int N = pass == 1 ? a.P[2] : (pass == 2 ? a.P[1] : a.P[0] / 2);
  switch (N) {
    case 4: return run_pass_len<T, 4>(pass, v, a, bm, nb, s);
    case 8: return run_pass_len<T, 8>(pass, v, a, bm, nb, s);
    case 16: return run_pass_len<T, 16>(pass, v, a, bm, nb, s);
    case 24: return run_pass_len<T, 24>(pass, v, a, bm, nb, s);
    case 32: return run_pass_len<T, 32>(pass, v, a, bm, nb, s);
    case 40: return run_pass_len<T, 40>(pass, v, a, bm, nb, s);
    case 48: return run_pass_len<T, 48>(pass, v, a, bm, nb, s);
    case 56: return run_pass_len<T, 56>(pass, v, a, bm, nb, s);
    case 64: return run_pass_len<T, 64>(pass, v, a, bm, nb, s);
    case 80: return run_pass_len<T, 80>(pass, v, a, bm, nb, s);
    case 96: return run_pass_len<T, 96>(pass, v, a, bm, nb, s);
    case 112: return run_pass_len<T, 112>(pass, v, a, bm, nb, s);
    case 128: return run_pass_len<T, 128>(pass, v, a, bm, nb, s);
    case 160: return run_pass_len<T, 160>(pass, v, a, bm, nb, s);
    case 192: return run_pass_len<T, 192>(pass, v, a, bm, nb, s);
    case 224: return run_pass_len<T, 224>(pass, v, a, bm, nb, s);
    case 256: return run_pass_len<T, 256>(pass, v, a, bm, nb, s);
    case 320: return run_pass_len<T, 320>(pass, v, a, bm, nb, s);
    case 384: return run_pass_len<T, 384>(pass, v, a, bm, nb, s);
    case 448: return run_pass_len<T, 448>(pass, v, a, bm, nb, s);
    case 512: return run_pass_len<T, 512>(pass, v, a, bm, nb, s);
    case 640: return run_pass_len<T, 640>(pass, v, a, bm, nb, s);
    case 768: return run_pass_len<T, 768>(pass, v, a, bm, nb, s);
    case 896: return run_pass_len<T, 896>(pass, v, a, bm, nb, s);
    case 1024: return run_pass_len<T, 1024>(pass, v, a, bm, nb, s);
    case 1280: return run_pass_len<T, 1280>(pass, v, a, bm, nb, s);
    case 1536: return run_pass_len<T, 1536>(pass, v, a, bm, nb, s);
    case 1792: return run_pass_len<T, 1792>(pass, v, a, bm, nb, s);
    case 2048: return run_pass_len<T, 2048>(pass, v, a, bm, nb, s);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t run_pass_dt(int dt, int pass, int v, const GenArgs& a, const BatchMap* bm,
                               int* nb, cudaStream_t s) {
  if (pass < 1 || pass > 3) return cudaErrorInvalidValue;
  return dt == 8 ? run_pass_t<double>(pass, v, a, bm, nb, s)
                 : run_pass_t<float>(pass, v, a, bm, nb, s);
}

void philox_schedule(GenArgs* a) {
  for (int r = 0; r < 10; ++r) {
    a->ks[r] = a->k0 + (uint32_t)r * 0x9E3779B9u;
    a->ks[10 + r] = a->k1 + (uint32_t)r * 0xBB67AE85u;
  }
}

cudaError_t launch_gen_pass(int dt, int pass, const GenArgs& a_in, cudaStream_t s) {
  if (pass < 1 || pass > 3) return cudaErrorInvalidValue;
  GenArgs a = a_in;
  philox_schedule(&a);
  if (pass == 1 && a.split && dt == 4 && a.spec == SPEC_PHILOX && gen_z_tc_supported(a.P[2]))
    return launch_gen_z_tc(a, s);
  if (pass == 3 && c2r_x_tc_used(dt, a)) return launch_c2r_x_tc(a, s);
  return run_pass_dt(dt, pass, a.var[pass - 1], a, nullptr, nullptr, s);
}

cudaError_t launch_gen_pass_batch(int dt, int pass, int v, const GenArgs& rep, const BatchMap& m,
                                  cudaStream_t s) {
  if (m.n < 1 || m.total < 1) return cudaErrorInvalidValue;
  return run_pass_dt(dt, pass, v, rep, &m, nullptr, s);
}

int gen_pass_blocks(int dt, int pass, int v, const GenArgs& a) {
  int nb = 0;
  if (run_pass_dt(dt, pass, v, a, nullptr, &nb, nullptr) != cudaSuccess) return -1;
  return nb;
}

// Every pass-3 kernel stores one moment pair a block.
int gen_pass3_partials(int dt, int v, const GenArgs& a) {
  if (c2r_x_tc_used(dt, a)) return c2r_x_tc_blocks(a);
  return gen_pass_blocks(dt, 3, v, a);
}

// The variant an untuned (precision, pass, length) runs: the FP32 pass 3 on
// the register transform with 32 lanes a line (else 16) where it serves the
// length and the status word exists; variant 0 otherwise.
int gen_default_variant(int dt, int pass, const GenArgs& a) {
  if (dt == 4 && pass == 3 && a.status) {
    for (int v : {RowVars<float>::n + 2, RowVars<float>::n + 1})
      if (gen_pass_blocks(dt, pass, v, a) > 0) return v;
  }
  return 0;
}

int gen_variant_count(int dt, int pass) {
  if (pass == 3) return dt == 8 ? RowVars<double>::n : RowVars<float>::n + kShflVars<float>;
  if (pass == 2 && dt == 4) return ColVars<float>::n + kDirectVars<float>;
  return dt == 8 ? ColVars<double>::n : ColVars<float>::n;
}

// ---------------------------------------------------------------------------
// FP64 spectral variance-normalisation sum over the full periodic grid.
// ---------------------------------------------------------------------------
constexpr int kSumThreads = 256;
int spectrum_sum_blocks() { return 148 * 8; }

__global__ void __launch_bounds__(kSumThreads) k_spec_sum(const GenArgs a, const double* rx,
                                                          const double* ry, const double* rz,
                                                          double craw2, double* partial) {
  const double* qx = static_cast<const double*>(a.qx);
  const double* qy = static_cast<const double*>(a.qy);
  const double* qz = static_cast<const double*>(a.qz);
  const int64_t total = (int64_t)a.Hx * a.P[1] * a.P[2];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(i % a.Hx);
    const int64_t r = i / a.Hx;
    const int ky = (int)(r % a.P[1]);
    const int kz = (int)(r / a.P[1]);
    const double c = (kx == 0 || 2 * kx == a.P[0]) ? 1.0 : 2.0;
    double v;
    if (a.amp == AMP_SEPARABLE) {
      const double A = rx[kx] * ry[ky] * rz[kz];
      v = A * A;
    } else {
      v = craw2 * pow(1.0 + qx[kx] + qy[ky] + qz[kz], 2.0 * a.expo);
    }
    acc += c * v;
  }
  __shared__ double red[kSumThreads / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kSumThreads / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

cudaError_t launch_spectrum_sum(const GenArgs& a, const double* rx, const double* ry,
                                const double* rz, double craw2, double* partial, int nblocks,
                                cudaStream_t s) {
  k_spec_sum<<<nblocks, kSumThreads, 0, s>>>(a, rx, ry, rz, craw2, partial);
  return cudaGetLastError();
}

}  // namespace scarl
