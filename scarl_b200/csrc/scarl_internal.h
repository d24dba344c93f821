// scarl_internal.h -- kernel argument blocks and launcher declarations shared
// between the CUDA translation units and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace scarl {

// Per-axis blend tables for one tile (device pointers, Np[d] entries each).
//   lo/hi : partition-of-unity factors of the low / high side (1.0 where the
//           side has no neighbour), multiplied low x,y,z then high x,y,z.
//   flags : bit0 = the tile contributes the point along this axis,
//           bit1 = first contributor, bit2 = last contributor.
struct BlendAxis {
  const double* lo;
  const double* hi;
  const uint8_t* flags;
  const double* sw64;  // sqrt(lo * hi): the axis' factor of sqrt(weight)
  const float* sw32;
};

struct Epilogue {
  int mode;            // 0 = plain crop, 1 = blend into a global field
  void* out;           // plain: Nx*Ny*Nz tile; blend: L0*L1*L2 global field
  int64_t L[3];        // global extent (blend)
  int64_t off[3];      // tile origin in the global field (blend)
  BlendAxis ax[3];
  int marginal;        // 0 none, 1 Gaussian (x*s+mu), 2 lognormal exp(x*s+mu)
  double ms, mmu;
  int apply_pou;
  double* mom;         // non-null: pass 3 stores per-block FP64 partial sums of the final
                       // values and their squares here (gen_pass3_partials pairs)
};

// Spectrum synthesis for the padded periodic grid.
enum SpecMode : int {
  SPEC_PHILOX = 0,  // canonical Philox normals times amplitude
  SPEC_INJECT = 1,  // caller-supplied normal pairs times amplitude
  SPEC_SHINO = 2,   // build_Sk_mtx phases (Park-Miller) and amplitude, literal
};
enum AmpKind : int {
  AMP_SEPARABLE = 0,  // A = ax[kx] * ay[ky] * az[kz]
  AMP_RECIP = 1,      // A = ax[kx] / (1 + qx + qy + qz)
  AMP_POW = 2,        // A = ax[kx] * (1 + qx + qy + qz)^expo
};

struct GenArgs {
  int P[3];
  int Hx, Hpad;
  int Nout[3];
  void* work;            // complex intermediate, Hpad * P1 * Nout2 entries
  const void* tw_z;      // e^{2 pi i m / P2}
  const void* tw_y;      // e^{2 pi i m / P1}
  const void* tw_x;      // e^{2 pi i m / P0}
  // spectrum
  int spec;              // SpecMode
  int amp;               // AmpKind
  const void* ax;        // separable: amplitude factors; Matern: g(kx)/sqrt(norm) prefactor
  const void* ay;
  const void* az;
  const void* qx;        // Matern: 4 pi^2 a_d^2 f_d^2 per axis
  const void* qy;
  const void* qz;
  double expo;           // Matern: -(nu + 3/2) / 2
  uint32_t k0, k1, stream;
  uint32_t ks[20];       // Philox round keys k0 + r C0 (r < 10), k1 + r C1 (philox_schedule)
  const void* xi;        // injected normal pairs (SPEC_INJECT)
  // literal Shino spectrum (FP64 tables)
  int sz[3];
  uint32_t pm_s1;        // Park-Miller state after the first step
  const uint32_t* pm_pw; // 16807^(2^b) mod (2^31-1)
  double de[3];          // (PI^2/2) delta_k^2
  double shino_scale;    // sqrt(8) and 2 sqrt(prod delta_k) applied in order
  double shino_f;
  Epilogue epi;
  int var[3];            // launch variant of each pass (autotuned, 0 = default)
  int split;             // FP32, split BF16 on the tensor cores: bit 0 pass 1's z DFT, bit 1 pass 3's x DFT
  int* status;           // device word, bit 0 set when a bounded tensor-core wait expired
  int wait_test;         // test hook: the tensor-core pass issues no MMA and waits 20 ms
};

// One batched launch of a pass over several realisations that share the
// pass' line length: block b of the flat grid belongs to items[i] where
// start[i] <= b < start[i + 1] (device arrays, n + 1 offsets).
struct BatchMap {
  const GenArgs* args;   // argument blocks of every realisation (device)
  const int* items;      // realisations of this launch (device, n entries)
  const int* start;      // block offsets (device, n + 1 entries)
  int n;
  int total;             // start[n], the launch's grid size
};

// Fills a->ks from a->k0, a->k1 (the launchers call it; batched argument
// blocks must have it filled before upload).
void philox_schedule(GenArgs* a);

// Launchers (return cudaSuccess or the launch error).  dt: 4 = FP32, 8 = FP64.
// pass: 1 = synthesis + z, 2 = y, 3 = C2R x + epilogue.
cudaError_t launch_gen_pass(int dt, int pass, const GenArgs& a, cudaStream_t s);
// Batched form: rep is the host copy of one member's arguments (line length
// and spectrum mode), v the launch variant.
cudaError_t launch_gen_pass_batch(int dt, int pass, int v, const GenArgs& rep, const BatchMap& m,
                                  cudaStream_t s);
// Pass 1 with the z-axis DFT as split-BF16 tensor-core matrix products
// (gen_tc.cu): FP32, Philox spectrum, line lengths with gen_z_tc_supported.
bool gen_z_tc_supported(int N);
cudaError_t launch_gen_z_tc(const GenArgs& a, cudaStream_t s);
// Batched form over realisations sharing the z length (m.start: offsets in
// work items, gen_z_tc_items per realisation; rep: any member).
int gen_z_tc_items(const GenArgs& a);
cudaError_t launch_gen_z_tc_batch(const GenArgs& rep, const BatchMap& m, cudaStream_t s);
// Pass 3 with the x-axis DFT as split-BF16 tensor-core matrix products
// (c2r_tc.cu): FP32, single-tile launches, half lengths P0 / 2 with
// c2r_x_tc_supported; c2r_x_tc_blocks is its CTA count (one FP64 moment pair
// each).  launch_gen_pass takes it for pass 3 when bit 1 of a.split is set
// (SCARL_SPLIT_BF16_X).
bool c2r_x_tc_supported(int N);
cudaError_t launch_c2r_x_tc(const GenArgs& a, cudaStream_t s);
int c2r_x_tc_blocks(const GenArgs& a);
// True when pass 3 of a runs on the tensor cores.
inline bool c2r_x_tc_used(int dt, const GenArgs& a) {
  return (a.split & 2) && dt == 4 && a.status && c2r_x_tc_supported(a.P[0] / 2);
}
// Blocks one realisation needs in a pass with launch variant v.
int gen_pass_blocks(int dt, int pass, int v, const GenArgs& a);
// Number of launch variants of a pass (valid ones depend on the line length).
int gen_variant_count(int dt, int pass);
// Variant of an untuned (precision, pass, line length) for the grid of a.
int gen_default_variant(int dt, int pass, const GenArgs& a);
// FP64 partial pairs (sum x, sum x^2) a single-tile pass-3 launch of variant v
// writes at a.epi.mom (-1: the variant does not serve the grid).
int gen_pass3_partials(int dt, int v, const GenArgs& a);
// out[0..1] = sums of the n pairs at pairs (device), in a fixed order; part:
// 2 pair_sum_parts() doubles of device scratch.
cudaError_t launch_pair_sum(const double* pairs, int64_t n, double* part, double* out, cudaStream_t s);
int pair_sum_parts();
// FP64 sum over the full periodic grid of S(k) dk^3: separable tables r*
// (A_raw = rx ry rz) or Matern q tables with A_raw^2 = craw2 (1+q)^(2 expo).
cudaError_t launch_spectrum_sum(const GenArgs& a, const double* rx, const double* ry,
                                const double* rz, double craw2, double* partial, int nblocks,
                                cudaStream_t s);
int spectrum_sum_blocks();

// Literal DCT-III path (FP64).
struct DctArgs {
  int Np[3];
  int K[3];
  const double* cx;  // per-axis corrL * exp(-PI k^2) factors, order of the reference
  const double* cy;
  const double* cz;
  double corrL[3];
  const double* phi;    // injected phases (K0*K1*K2) or null (Philox uniforms)
  const double* gamma;  // injected amplitudes or null (1)
  uint32_t k0, k1, stream;
  double* sk;           // K0*K1*K2 spectrum
  double* t1;           // N0*K1*K2
  double* t2;           // N0*N1*K2
  double* out;          // N0*N1*N2
  const double* ctab[3];  // 2*cos(pi m / (2 N)) (and 1 at i = 0), m < 4N
};
cudaError_t launch_dct_literal(const DctArgs& a, cudaStream_t s);

// Post steps.
cudaError_t launch_blend_tile(int dt, const void* tile, const int Np[3], const Epilogue& e,
                              cudaStream_t s);
cudaError_t launch_apply_pou(int dt, void* field, const int Np[3], const BlendAxis ax[3],
                             cudaStream_t s);
cudaError_t launch_add_overlap(const double* in, double* out, const int Np[3],
                               const int Np_ovlp[3], const int topo[3], cudaStream_t s);
cudaError_t launch_marginal(int dt, void* f, int64_t n, int kind, double sc, double mu,
                            cudaStream_t s);
cudaError_t launch_affine(int dt, void* f, int64_t n, double sub, double div, cudaStream_t s);
// FP64 sums of x and x^2 over nmc blocks of xN values; partial has
// nmc * nb * 2 doubles.
cudaError_t launch_sums(int dt, const void* f, int64_t xN, int nmc, double* partial, int nb,
                        cudaStream_t s);
int sums_blocks(int64_t xN);

// Directional circular autocovariance of the standardised, windowed field.
cudaError_t launch_lag_cov(int dt, const void* f, const int L[3], int dir, double avg,
                           double sd, const double* win, int nkeep, double* partial, int nparts,
                           cudaStream_t s);
int lag_cov_parts(const int L[3], int dir);

// Streamed axis covariance (cov.cu): per-block FP64 power of the centred,
// zero-padded lines along axis dir (complex length N, padded length 2N),
// then S(h) for h <= maxlag.  bins holds N + 1 doubles.
int axis_power_blocks(int dt, const int L[3], int dir, int N);
// status: the context's device status word (bit 0: a bounded copy wait of
// the TMA form expired); null runs the forms without bulk copies.
cudaError_t launch_axis_power(int dt, const void* f, const int L[3], int dir, int N, double mu,
                              const void* tw, double* partial, int nblocks, cudaStream_t s,
                              int* status = nullptr);
cudaError_t launch_cov_lags(const double* partial, int nblocks, int N, int maxlag,
                            const double* tw64, double* bins, double* S, cudaStream_t s);

// Learned padding (mlp.cu).  One axis of one configuration: kind 1 =
// Gaussian, 2 = Matern (nu; exponential is nu = 1/2); ell in grid points;
// q = 4 pi^2 a^2 (Matern).  N <= 256.
struct PadLabelIn {
  int kind, N;
  double ell, nu, q;
};
struct PadLabelOut {
  int P, W, saturated;
};
cudaError_t launch_pad_labels(const PadLabelIn* in, PadLabelOut* out, int n, double tol,
                              cudaStream_t s);
cudaError_t launch_pad_error(const PadLabelIn* in, const int* P, double* err, int n,
                             cudaStream_t s);
constexpr int kMlpIn = 16, kMlpHidden = 64, kMlpOut = 2;
constexpr int kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden +
                           kMlpHidden + kMlpOut * kMlpHidden + kMlpOut;
cudaError_t launch_mlp_train(const void* X, const float* T, int n, const void* wb, const float* p,
                             float* grad, double* loss, cudaStream_t s);
cudaError_t launch_mlp_infer(const void* X, int n, const void* wb, const float* p, float* Y,
                             cudaStream_t s);
cudaError_t launch_mlp_adam(float* p, float* g, float* m, float* v, void* wb, float lr, int t,
                            cudaStream_t s);
cudaError_t launch_to_bf16(const float* a, void* b, int n, cudaStream_t s);

}  // namespace scarl
