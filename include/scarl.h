/*
 * scarl.h -- C ABI of scarl_b200, a B200 (sm_100a) implementation of the
 * ScaRL random-field path: spectral generation on a padded periodic grid (or
 * the reference's DCT-III generator), partition-of-unity blending of
 * overlapping subdomain tiles, the marginal transform, and the Stat_ScaRL
 * moment / covariance estimators.
 *
 * Conventions
 *  - Arrays are column-major (Fortran order, x fastest), as in ScaRL.
 *  - Every call returns an int status (SCARL_OK = 0); the library never exits
 *    or traps.  scarl_last_error(ctx) holds the message of the last failure.
 *  - Field pointers may be host memory (pageable or pinned) or device memory
 *    of the context's GPU; the library detects which and copies as needed.
 *  - Device work runs on the context's stream (its own, or one set with
 *    scarl_ctx_set_stream).  Calls with host pointers return after the
 *    results are in host memory; calls with device pointers return after the
 *    work is enqueued (use scarl_sync).
 *  - One context per host thread.  Contexts own all device scratch memory
 *    (grown on demand up to the budget given at creation, then reused).
 *  - Functions marked [host] compute on the CPU and need no GPU; they accept
 *    ctx == NULL.
 */
#ifndef SCARL_H
#define SCARL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SCARL_OK 0
#define SCARL_EINVAL 1       /* invalid argument (verify_inputs rules, sizes) */
#define SCARL_ENOMEM 2       /* device memory budget or allocation exhausted */
#define SCARL_EDEVICE 3      /* CUDA error */
#define SCARL_ETIMEOUT 4     /* a bounded device wait expired */
#define SCARL_EUNSUPPORTED 5 /* valid in the reference but not provided here */
#define SCARL_EIO 6          /* file could not be read */

/* ---- enumerations: values of SRC_F/constants_ScaRL.f90:12-19 ---- */
#define SCARL_FFT 1          /* gen_meth: FFT with localization */
#define SCARL_FFT_MPI 2      /* gen_meth: slab FFTW-MPI (layout only here) */
#define SCARL_CM_GAUSSIAN 1
#define SCARL_CM_VON_KARMAN 2
#define SCARL_CM_EXPONENTIAL 3 /* no counterpart in the reference */
#define SCARL_FOM_GAUSSIAN 1
#define SCARL_FOM_LOGNORMAL 2

/* ---- precisions ---- */
#define SCARL_F32 4
#define SCARL_F64 8
/* Flag OR'ed into SCARL_F32 for the padded generator (scarl_gen_padded,
 * scarl_generate_sample's opts.dtype): the z-axis DFT of pass 1 runs on the
 * tensor cores as split-BF16 matrix products (head + tail of every operand,
 * three products, FP32 accumulation), a field error near 4e-6 relative L2
 * against FP64 (bounded by 1e-5).  Padded z lengths without a tensor-core
 * kernel, and injected or literal spectra, run the FP32 pass instead.  No
 * counterpart in the reference. */
#define SCARL_SPLIT_BF16 0x100
/* Flag OR'ed into SCARL_F32 (implies SCARL_SPLIT_BF16): pass 3's Hermitian
 * C2R along x also runs on the tensor cores, its half length N = P0 / 2 as two
 * split-BF16 DFT stages N1 x N2 (N2 = 32 with N1 = 2..8, or N2 = 16 with N1 =
 * 2, 3, 5, 7), in front of the same crop / blend epilogue; other half lengths
 * and batched ensembles keep the CUDA-core pass 3.  Field error bounded by
 * 1e-5 relative L2 against FP64.  Slower than the CUDA-core pass 3 on B200
 * (0.151 against 0.109 ms per tile of the 513^3 headline field), so it is
 * not part of SCARL_SPLIT_BF16.  No counterpart in the reference. */
#define SCARL_SPLIT_BF16_X 0x200

/* ---- generators for scarl_generate_sample ---- */
#define SCARL_GEN_DCT 1      /* gen_std_gauss_FFT, SRC_F/fftw_ScaRL.f90:261 */
#define SCARL_GEN_SHINO 2    /* gen_std_gauss_Shino_FFT, SRC_F/fftw_ScaRL.f90:157 */
#define SCARL_GEN_PADDED 3   /* padded periodic C2R, normalised spectra */

/* ---- padded grid policies ---- */
#define SCARL_PAD_FULL 0     /* 2^ceil(log2(2 Np)), SRC_F/fftw_ScaRL.f90:194 */
#define SCARL_PAD_AUTO 1     /* smallest power of two with image error <= tol */
#define SCARL_PAD_LEARNED 2  /* the context's trained predictor, full padding as fallback */
#define SCARL_PAD_SMOOTH 3   /* as AUTO over every supported length: powers of two and
                                3, 5, 7 x 2^a (2^a >= 16), at most 2048 */

typedef struct scarl_ctx scarl_ctx;

/* One deck entry: the 11 per-sample lines of input_ScaRL.txt
 * (SRC_F/read_input.f90:257-299), plus the von Karman order nu. */
typedef struct {
  char name[256];
  double xMinGlob[3];
  double xMaxGlob[3];
  double corrL[3];
  double overlap[3];      /* in correlation lengths */
  int pointsPerCorrL[3];
  int corrMod;
  int margiFirst;
  double avg;
  double std_dev;
  int seedBase;
  double nu;              /* von Karman smoothness (0.5 = exponential) */
} scarl_sample;

/* Index maps of one sample (SRC_F/main_ScaRL.f90:100-176). */
typedef struct {
  int L[3];               /* global points after the re-fit of :176 */
  int Np[3];              /* points per tile */
  int Np_ovlp[3];         /* overlap points */
  int topo_shape[3];      /* tiles per axis */
  int nb_tiles;           /* product(topo_shape) */
  double xStep[3];
} scarl_layout;

/* Geometry of one tile (SRC_F/main_ScaRL.f90:455-468). */
typedef struct {
  int topo_pos[3];
  int pos_0[3];           /* 1-based, like the reference */
  int pos_N[3];
  double coord_0[3];
  double coord_N[3];
  double xRange[3];
} scarl_tile;

/* Options of scarl_generate_sample; zero-initialise for the defaults. */
typedef struct {
  int generator;          /* SCARL_GEN_*, 0 = SCARL_GEN_PADDED */
  int dtype;              /* SCARL_F32 / SCARL_F64, 0 = SCARL_F32 */
  int nb_procs;           /* tiles requested (mpirun -np), 0 = 1 */
  int topo_shape[3];      /* explicit topology (extra_config_ScaRL.txt); 0 = decide */
  int pad[3];             /* explicit padded grid per axis; 0 = chosen by pad_policy */
  int pad_policy;         /* SCARL_PAD_FULL (default), _AUTO, _LEARNED or _SMOOTH */
  double pad_tol;         /* SCARL_PAD_AUTO / _SMOOTH image tolerance, 0 = 1e-3 */
  int no_spectral_normalisation; /* 1 = raw Riemann-sum amplitudes */
  int normalize_field;    /* 1 = normalize_field (disabled in the reference) */
  uint32_t stream;        /* realisation stream (ensembles), 0 by default */
  int autotune;           /* 1 = autotune each new grid shape on first use */
  const double* phiK;     /* DCT generator: injected phases, nb x (Np/2)^3 */
  int gen_meth;           /* SCARL_FFT (0 = default): overlapping tiles blended by the
                             partition of unity; SCARL_FFT_MPI: the whole re-fitted grid as
                             one global transform (DCT: spectrum over every kz, phases
                             L0/2 x L1/2 x L2) */
  double* moments;        /* non-NULL (host, 2 values): receives sum f and sum f^2 over
                             the output field in FP64, accumulated inside the C2R pass as
                             each point becomes final (no second read of the field;
                             padded and Shino generators, not with normalize_field) */
} scarl_gen_opts;

/* ------------------------------------------------------------------ */
/* Context                                                             */
/* ------------------------------------------------------------------ */
int scarl_ctx_create(int device, size_t budget_bytes, scarl_ctx** ctx);
int scarl_ctx_destroy(scarl_ctx* ctx);
const char* scarl_last_error(const scarl_ctx* ctx);
int scarl_ctx_set_stream(scarl_ctx* ctx, void* cuda_stream);
int scarl_sync(scarl_ctx* ctx);
/* Autotuner (no counterpart in the reference): times every launch variant
 * (values per thread, lines per block) of the three generator passes on
 * padded grid P and tile Np, keeps the fastest per (dtype, pass, line
 * length) in the context, and merges the choices into cache_path (text
 * lines "dtype pass N variant"; NULL = no file).  Contexts also load the
 * file named by the environment variable SCARL_TUNE_CACHE when created.
 * FP32 pass 3 has three more variants after the shared-memory engine's five
 * (5, 6, 7: the line transform in registers and warp shuffles with 8, 16
 * and 32 lanes a line, for half lengths N = N2 L with N2 <= 32 of the form
 * 2^a, 3, 5 or 7 x 2^a); an untuned FP32 pass 3 runs variant 7, else 6,
 * where it serves the length.  scarl_tune_get gives the stored choice (-1
 * when the triple has none); scarl_tune_set with variant -1 forgets it. */
int scarl_autotune(scarl_ctx* ctx, int dtype, int corrMod, double nu, const int P[3],
                   const int Np[3], const double xStep[3], const double corrL[3],
                   const char* cache_path);
int scarl_tune_get(scarl_ctx* ctx, int dtype, int pass, int N, int* variant);
int scarl_tune_set(scarl_ctx* ctx, int dtype, int pass, int N, int variant);
/* Test hook of the tensor-core pass's bounded waits (no counterpart in the
 * reference): while enabled, SCARL_SPLIT_BF16 tiles issue no matrix product,
 * so every CTA's wait on the tensor core runs out after 20 ms; the kernel
 * raises the context's status word, frees its tensor memory and returns, and
 * the call (or the next scarl_sync) returns SCARL_ETIMEOUT.  The context stays
 * usable. */
int scarl_tc_wait_test(scarl_ctx* ctx, int enable);
/* Kernels launched and bytes copied host->device / device->host by this
 * context since its creation. */
int scarl_counters(scarl_ctx* ctx, long long* launches, unsigned long long* h2d_bytes,
                   unsigned long long* d2h_bytes);
/* Per-kernel device time (CUDA events around each launch) while enabled;
 * enable = 2 clears the accumulated times. */
int scarl_profile(scarl_ctx* ctx, int enable);
int scarl_profile_read(scarl_ctx* ctx, int idx, char* name, size_t name_len,
                       double* total_ms, long long* launches);
const char* scarl_version(void);

/* ------------------------------------------------------------------ */
/* [host] Index maps, topology, weights (bit-exact restatements)       */
/* ------------------------------------------------------------------ */
/* SRC_F/main_ScaRL.f90:271-340 (verify_inputs): 0 or SCARL_EINVAL with the
 * reference's message in msg.  corrMod 2/3 are accepted (new models). */
int scarl_verify_inputs(const scarl_sample* s, int gen_meth, char* msg, size_t msg_len);
/* SRC_F/main_ScaRL.f90:788-897 (decide_topo_shape, localization branch). */
int scarl_decide_topo_shape(int nb_procs, const int L[3], const int Np_ovlp[3],
                            long long pointsPerBlockIdeal, int topo_shape[3]);
/* SRC_F/main_ScaRL.f90:747-782 (get_topo_pos / get_topo_rank). */
int scarl_get_topo_pos(int rank, const int topo_shape[3], int topo_pos[3]);
int scarl_get_topo_rank(const int topo_shape[3], const int topo_pos[3]);
/* SRC_F/main_ScaRL.f90:100-176: xStep, L, Np_ovlp, topology, Np, re-fitted L.
 * topo_shape_in = NULL decides the topology for nb_procs tiles. */
int scarl_sample_layout(const scarl_sample* s, int gen_meth, int nb_procs,
                        const int* topo_shape_in, scarl_layout* out);
/* SRC_F/main_ScaRL.f90:455-459 (pos_0, pos_N, coord_0, coord_N, xRange). */
int scarl_tile_geometry(const scarl_layout* lay, const double xMinGlob[3], int rank,
                        scarl_tile* out);
/* SRC_F/main_ScaRL.f90:1236-1294: the Np[0]*Np[1]*Np[2] weight array. */
int scarl_unity_partition_weights(const int Np[3], const int Np_ovlp[3], int partitionType,
                                  const int topo_pos[3], const int topo_shape[3], double* w);
/* SRC_F/fftw_ScaRL.f90:194 and SRC_F/spectra_ScaRL.f90:44-56: padded grid,
 * spectrum box and delta_k of the Shino generator (k_cut clamped to k_max). */
int scarl_shino_sizes(const int Np[3], const double xRange[3], const double corrL[3],
                      int sz_c[3], int sz_Sk[3], double delta_k[3]);

/* Padded periodic grid of a tile (no counterpart in the reference beyond
 * the FULL rule of SRC_F/fftw_ScaRL.f90:194).  AUTO: smallest power of two
 * P >= 8 per axis with C((P - Np + 1) xStep) <= tol, C the target model's
 * unit-variance correlation along that axis. */
int scarl_pad_size(int policy, int corrMod, double nu, const double corrL[3],
                   const double xStep[3], const int Np[3], double tol, int P[3]);
/* Target model correlation at lag r along an axis of integral scale l. */
double scarl_axis_correlation(int corrMod, double nu, double l, double r);

/* ------------------------------------------------------------------ */
/* [host] Input decks (SRC_F/read_input.f90)                           */
/* ------------------------------------------------------------------ */
/* read_config_ScaRL :26-102; a missing file gives the defaults of :74-83. */
int scarl_read_config(const char* path, int* gen_meth, int* c_info_file, int* d_sample,
                      int* one_file, int* one_hdf_ds, char* input_file, size_t len);
/* read_extra_config_ScaRL :108-149; *found = 0 when the file is absent. */
int scarl_read_extra_config(const char* path, int* found, int topo_shape[3]);
/* read_input_ScaRL :159-348.  Call with samples = NULL to get the count. */
int scarl_read_input(const char* path, char* output_folder, size_t folder_len,
                     int* nSamples, scarl_sample* samples, int max_samples);
/* read_input_SEM :354-559 (random.spec + domains.txt in folder). */
int scarl_read_input_sem(const char* folder, char* output_folder, size_t folder_len,
                         int* nSamples, scarl_sample* samples, int max_samples);

/* ------------------------------------------------------------------ */
/* Generation                                                          */
/* ------------------------------------------------------------------ */
/* Drop-in for gen_std_gauss_FFT (SRC_F/fftw_ScaRL.f90:261-418), FP64.
 * data_real_3D: Np[0]*Np[1]*Np[2] doubles (caller-allocated, overwritten).
 * phiK / gammaK: the (Np/2)^3 phase and amplitude arrays the reference draws
 * with random_number (:364-367); phiK = NULL draws Philox uniforms keyed by
 * seed + rank, gammaK = NULL uses 1 (the reference's :367).  corrMod must be
 * SCARL_CM_GAUSSIAN (the only model of this routine). */
int scarl_gen_std_gauss_fft(scarl_ctx* ctx, double* data_real_3D, const int Np[3],
                            const double xRange[3], const double corrL[3], int corrMod,
                            int seed, int rank, const double* phiK, const double* gammaK);

/* Drop-in for gen_Std_Gauss_FFT_MPI (SRC_F/fftw_ScaRL.f90:424-583) on one GPU:
 * the global DCT-III over the L grid of the spectrum on (L0/2, L1/2, L2), Gaussian
 * model, FP64.  The MPI communicator has no counterpart: the whole transform runs
 * on the GPU, so Np must equal L (one rank).  phiK / gammaK: injected
 * (L0/2)(L1/2)L2 phases / amplitudes or NULL (Philox uniforms / 1). */
int scarl_gen_std_gauss_fft_mpi(scarl_ctx* ctx, double* data_real_3D, const double xRange[3],
                                const double corrL[3], int corrMod, int seed, int rank,
                                const int L[3], const int Np[3], const double* phiK,
                                const double* gammaK);

/* Drop-in for gen_std_gauss_Shino_FFT + build_Sk_mtx (SRC_F/fftw_ScaRL.f90:
 * 157-255, SRC_F/spectra_ScaRL.f90:10-142), FP64: Park-Miller phases from
 * seed + 1000000, the reference's amplitude and scaling, padded grid
 * 2^ceil(log2(2 Np)), real part cropped to Np.  The quadrant placement uses
 * the full first axis of the spectrum box (the reference's :204 halves it). */
int scarl_gen_std_gauss_shino_fft(scarl_ctx* ctx, double* data_real_3D, const int Np[3],
                                  const double xRange[3], const double corrL[3],
                                  const int pointsPerCorrL[3], int corrMod, int seed, int rank);

/* Padded periodic method, one tile, no blending: Np[0]*Np[1]*Np[2] values of
 * dtype written to out.  Grid spacing xStep, padded grid pad (0 entries =
 * 2^ceil(log2(2 Np))).  corrMod 1/2/3 with nu for 2.  normalise = 1 scales
 * the spectrum so the periodic field has unit variance (FP64 sum on the
 * GPU).  xi = NULL draws Philox normals keyed by (seed, stream); otherwise xi
 * holds (P0/2+1)*P1*P2 pairs (re, im) of dtype, mode index kx fastest. */
int scarl_gen_padded(scarl_ctx* ctx, void* out, int dtype, const int Np[3], const int pad[3],
                     const double xStep[3], const double corrL[3], int corrMod, double nu,
                     int normalise, uint64_t seed, uint32_t stream, const void* xi);

/* No counterpart in the reference.  scarl_gen_padded for callers that
 * cannot allocate GPU memory (a host code whose device memory belongs to its
 * own pool allocator, or a running time-critical loop that must not call
 * cudaMalloc): no context, no allocation.  Its scratch is a fixed 64 MiB
 * device array reserved on every GPU that loads this library until the
 * process exits; requests whose intermediate and tables do not fit (the
 * intermediate is round_up(P0/2+1, 16) * P1 * Np[2] complex values: about
 * 8.3 M in FP32, 4.1 M in FP64, e.g. a 256^3 padded grid with Np[2] <= 225 in
 * FP32) return SCARL_EINVAL with the needed size in msg.  Padded lengths and
 * their default are those of scarl_gen_padded (SCARL_EUNSUPPORTED outside
 * them); dtype SCARL_F32 or SCARL_F64.
 * out must be device memory of the current GPU (a pointer to another GPU's
 * memory returns SCARL_EINVAL); work is enqueued on cuda_stream (NULL = the
 * legacy default stream).  The first call on a device looks up the array's
 * address: make it before any stream capture.  Every call uploads its
 * tables from host memory; with normalise = 1 the host also waits for the
 * FP64 spectral sum on cuda_stream before the passes are enqueued.
 * Calls share the array: calls whose GPU work may overlap race and must be
 * serialised.  Output equals scarl_gen_padded with xi = NULL. */
int scarl_gen_padded_noalloc(void* out, int dtype, const int Np[3], const int pad[3],
                             const double xStep[3], const double corrL[3], int corrMod, double nu,
                             int normalise, uint64_t seed, uint32_t stream, void* cuda_stream,
                             char* msg, size_t msg_len);

/* One deck sample end to end on the GPU (SRC_F/main_ScaRL.f90:95-214 +
 * create_fields :345-583 without file output): layout, every tile generated,
 * PoU-weighted, overlap-summed and assembled into the global field
 * L[0]*L[1]*L[2] (layout from scarl_sample_layout), marginal transformed.
 * global: dtype values. */
int scarl_generate_sample(scarl_ctx* ctx, const scarl_sample* s, const scarl_gen_opts* opts,
                          void* global);

/* ------------------------------------------------------------------ */
/* Ensembles (no counterpart in the reference, which generates one     */
/* sample per run, SRC_F/main_ScaRL.f90:82-214)                        */
/* ------------------------------------------------------------------ */
#define SCARL_ENS_AUTOTUNE 1  /* time the launch variants of every batched launch once */
#define SCARL_ENS_NO_GRAPH 2  /* launch eagerly instead of replaying the CUDA graph */

/* [host] Shapes and isotropic correlation lengths of realisations
 * first..first+n-1: realisation r reads the four words w of Philox4x32-10 at
 * counter {r, r >> 32, 0, 2}, key {seed, seed >> 32}; axis d gets
 * choices[floor(w_d * nchoices / 2^32)] points, the correlation length is
 * lmin + (lmax - lmin) (w_3 + 1/2) 2^-32.  Np and corrL receive 3 n values. */
int scarl_ensemble_draw(uint64_t seed, long long first, int n, const int* choices, int nchoices,
                        double lmin, double lmax, int* Np, double* corrL);

/* n independent padded-method realisations of uneven grids, one tile each
 * (dtype SCARL_F32, SCARL_F64 or SCARL_F32 | SCARL_SPLIT_BF16):
 * realisation i has Np[3i..3i+2] points of spacing xStep[3i..], correlation
 * lengths corrL[3i..], Philox key seeds[i] (NULL: i) and stream streams[i]
 * (NULL: 0).  Its field, column-major, starts at element
 * sum_{j<i} Np_j0 Np_j1 Np_j2 of out (device or host pointer).  Padded grids
 * follow pad_policy (SCARL_PAD_FULL, _AUTO or _SMOOTH) / pad_tol per realisation; margiFirst 0 leaves the
 * standard field, 1 / 2 apply the Gaussian / lognormal marginal of avg,
 * std_dev.  Realisations are grouped by line length in each of the three
 * passes and every group runs as one batched launch (with SCARL_SPLIT_BF16
 * the pass-1 groups whose z length has a tensor-core kernel run it,
 * persistent over the group's realisations); the first call for a
 * list of shapes builds the plan (FP64 spectral sums, tables, workspace) and
 * captures the launches in a CUDA graph that later calls replay. */
int scarl_gen_ensemble(scarl_ctx* ctx, void* out, int dtype, int n, const int* Np,
                       const double* xStep, const double* corrL, int corrMod, double nu,
                       int pad_policy, double pad_tol, const uint64_t* seeds,
                       const uint32_t* streams, int margiFirst, double avg, double std_dev,
                       int flags);

/* ------------------------------------------------------------------ */
/* Post steps (device kernels; FP64 fields in place)                   */
/* ------------------------------------------------------------------ */
/* apply_UnityPartition_mtx (SRC_F/main_ScaRL.f90:1216-1301), bit-exact. */
int scarl_apply_unity_partition(scarl_ctx* ctx, double* field, const int Np[3],
                                const int Np_ovlp[3], int partitionType, const int topo_pos[3],
                                const int topo_shape[3]);
/* add_overlap (SRC_F/main_ScaRL.f90:984-1210) over every tile at once:
 * tiles holds nb = prod(topo_shape) consecutive Np blocks in rank order;
 * each block receives its neighbours' overlap regions, bit-exact. */
int scarl_add_overlap(scarl_ctx* ctx, double* tiles, const int Np[3], const int Np_ovlp[3],
                      const int topo_shape[3]);
/* multiVariateTransformation (SRC_F/main_ScaRL.f90:1355-1395). */
int scarl_multivariate_transformation(scarl_ctx* ctx, void* field, int dtype, long long n,
                                      double avg, double std_dev, int margiFirst);
/* normalize_field (SRC_F/main_ScaRL.f90:903-953) on an assembled global
 * field (every point counted once): standardise, FP64 sums on the GPU. */
int scarl_normalize_field(scarl_ctx* ctx, void* field, int dtype, long long n, double* avg,
                          double* std_dev);

/* ------------------------------------------------------------------ */
/* Estimators (Stat_ScaRL), FP64 accumulation on the GPU               */
/* ------------------------------------------------------------------ */
/* calculate_average_and_stdVar_MPI (SRC_F/Stat_ScaRL/statistics_RF.f90:
 * 18-174): field is xNTotal x Nmc; per-realisation and global mean and
 * population standard deviation sqrt(E[x^2] - E[x]^2). */
int scarl_moments(scarl_ctx* ctx, const void* field, int dtype, long long xNTotal, int Nmc,
                  double* evntAvg, double* evntStdDev, double* globalAvg,
                  double* globalStdDev);
/* rebuild_Sk_FFT + rebuild_Sk (statistics_RF.f90:180-462) for one field
 * L[0]*L[1]*L[2]: per direction the circular autocovariance of the
 * standardised, Tukey-windowed field averaged over lines, first floor(L/2)
 * lags kept.  SkTot receives floor(L0/2)+floor(L1/2)+floor(L2/2) values.
 * tukey_literal = 1 reproduces the reference's window (single-precision
 * r_tukey, taper formula over every ratio > r); 0 the standard Tukey window. */
int scarl_rebuild_sk(scarl_ctx* ctx, const void* field, int dtype, const int L[3], double avg,
                     double stdDev, int tukey_literal, double* SkTot);
/* Mean, variance and the covariance along each axis up to lag maxlag of
 * one field L[0] x L[1] x L[2] (column-major, device or host pointer), FP64
 * accumulation on the GPU:
 *   cov[d (maxlag + 1) + h] = sum over point pairs (x, x + h e_d) of
 *       (f(x) - m)(f(x + h e_d) - m) / number of such pairs,
 * m = *known_mean when given (an ensemble of known mean), else the mean over
 * all points; *mean receives the sample mean, var = cov[0].  One moment pass plus one pass per
 * axis over the field.  No direct counterpart: rebuild_Sk_FFT
 * (statistics_RF.f90:258-462) windows and wraps each line; this is the
 * plain linear estimator a covariance model is checked against.  Needs
 * maxlag < L[d] and L[d] + maxlag <= 4096.  FP32 fields whose lines start on
 * 16-byte boundaries stage their lines through TMA bulk copies with bounded
 * waits: a wait that runs out returns SCARL_ETIMEOUT (the results are then
 * invalid). */
int scarl_axis_cov(scarl_ctx* ctx, const void* field, int dtype, const int L[3], int maxlag,
                   const double* known_mean, double* mean, double* var, double* cov);
/* scarl_axis_cov with the field's sums already known: sums = (sum f,
 * sum f^2), as scarl_gen_opts.moments streams them out of the generator's
 * C2R pass, so that only the per-axis passes read the field. */
int scarl_axis_cov_sums(scarl_ctx* ctx, const void* field, int dtype, const int L[3], int maxlag,
                        const double sums[2], double* mean, double* var, double* cov);
/* [host] rebuild_corrL (statistics_RF.f90:468-486). */
int scarl_rebuild_corrL(const double* SkTot, const int L[3], const double xStep[3],
                        double corrL_out[3]);

/* ------------------------------------------------------------------ */
/* Learned padding / overlap predictor (no counterpart in the          */
/* reference)                                                          */
/* ------------------------------------------------------------------ */
/* Labels from the method's expected axis covariance (FP64, GPU): for axis
 * i (corrMod[i], nu[i], correlation length ell_pts[i] in grid points, N[i]
 * <= 256 points) the smallest padded length P[i] whose covariance differs
 * by <= 0.01 from the infinitely padded method's over lags 0..N-1, and the
 * smallest overlap W[i] whose partition-of-unity blend keeps the covariance
 * error <= 0.01.  saturated[i] = 1 when even 16 N did not reach it. */
int scarl_pad_labels(scarl_ctx* ctx, int n, const int* corrMod, const double* nu,
                     const double* ell_pts, const int* N, int* P, int* W, int* saturated);
/* The same covariance error at given padded lengths P[i] (N <= P <= 8192). */
int scarl_pad_error(scarl_ctx* ctx, int n, const int* corrMod, const double* nu,
                    const double* ell_pts, const int* N, const int* P, double* err);
/* [host] Network inputs (16 per axis) and targets (log2 of the image
 * distance P - N + 1 and of W, in correlation lengths; 2 per axis). */
int scarl_mlp_features(int n, const int* corrMod, const double* nu, const double* ell_pts,
                       const int* N, float* X);
int scarl_mlp_targets(int n, const double* ell_pts, const int* N, const int* P, const int* W,
                      float* T);
/* The context's MLP (16 -> 64 -> 64 -> 2, ReLU; BF16 weights and
 * activations, FP32 accumulation; 5378 FP32 master parameters in the order
 * W1[64][16] b1 W2[64][64] b2 W3[2][64] b3). */
int scarl_mlp_init(scarl_ctx* ctx, uint64_t seed);
int scarl_mlp_params(scarl_ctx* ctx, float* get, const float* set);
/* Mean-squared-error loss and its gradient over n samples (no update). */
int scarl_mlp_grad(scarl_ctx* ctx, const float* X, const float* T, int n, float* grad,
                   double* loss);
/* steps full-batch Adam steps (learning rate lr); loss_hist: steps losses or NULL. */
int scarl_mlp_train(scarl_ctx* ctx, const float* X, const float* T, int n, int steps, float lr,
                    double* loss_hist);
int scarl_mlp_predict(scarl_ctx* ctx, const float* X, int n, float* Y);
/* Padded grid and overlap width per axis from the trained model, with a
 * 2^0.25 safety margin, rounded up to the next length the generator runs
 * (powers of two, 3, 5, 7 times a power of two >= 16); full padding
 * (SRC_F/fftw_ScaRL.f90:194) when the
 * inputs leave the trained range or the prediction exceeds it (fallback:
 * bit 0 out of range, bit 1 capped).  W may be NULL. */
int scarl_pad_size_learned(scarl_ctx* ctx, int corrMod, double nu, const double corrL[3],
                           const double xStep[3], const int Np[3], int P[3], int W[3],
                           int* fallback);

/* ------------------------------------------------------------------ */
/* Output files (SRC_F/write_output.f90, SRC_F/hdf5_ScaRL.f90)         */
/* ------------------------------------------------------------------ */
/* HDF5 + XDMF files of one generated sample, the three layouts of
 * SRC_F/main_ScaRL.f90:590-668: one_file && one_hdf_ds -> folder/name.h5
 * with dataset "samples" (write_hdf5_multi_proc_3D_1ds, :313-451) and
 * name.xmf; one_file only -> name.h5 with one dataset "sample_1_p<rank>" per
 * tile (write_hdf5_multi_proc_3D) and a global name.xmf; neither -> one
 * file name_proc_<rank, 5 digits>.h5/.xmf per tile (write_hdf5_single_proc_3D)
 * and the global name.xmf.  Every .h5 carries the root attributes of
 * write_HDF5_attributes (:722-813); with ntimes > 0 also "times" (1 x ntimes)
 * and "time_labels" (ntimes strings of 20 characters, time_labels holds
 * ntimes x 20 characters, space or NUL padded) as write_time_on_hdf5 does.
 * field: the L0 x L1 x L2 global field (device or host), written in its own
 * precision (the reference writes FP64).  The files use the classic HDF5
 * format (superblock 0, symbol-table groups, contiguous datasets) written by
 * this library's own encoder; no HDF5 library is needed. */
int scarl_write_sample_h5(scarl_ctx* ctx, const char* folder, const char* output_name,
                          const void* field, int dtype, const scarl_sample* s,
                          const scarl_layout* lay, int one_file, int one_hdf_ds,
                          const char* time_labels, const double* times, int ntimes);
/* [host] write_constant_field (SRC_F/write_output.f90:144-178), the output
 * of a sample with std_dev = 0: folder/name.h5 holding a 2 x 2 x 2 dataset
 * "samples" of avg with the reference's attribute values, and name.xmf. */
int scarl_write_constant_field_h5(const char* folder, const char* output_name,
                                  const double xMinGlob[3], const double xMaxGlob[3], double avg);
/* Stat_ScaRL's step for one result file (SRC_F/Stat_ScaRL/main_Stat.f90:59-104)
 * on the GPU: the sample attributes and dataset dset_name are read, the FP64
 * mean and standard deviation computed (calculate_average_and_stdVar_MPI);
 * with calc_corrL also the directional spectra (rebuild_Sk, literal Tukey
 * window) and correlation lengths (rebuild_corrL), which are then added to
 * the result file's root attributes (write_StatisticsOnH5: globalAvg,
 * globalStdDev, evntAvg, evntStdDev, corrL_out, Sk_1..Sk_3).  Always writes
 * folder/STAT_<file name> (makeStatFile).  corrL_out may be NULL. */
int scarl_stat_file(scarl_ctx* ctx, const char* res_path, const char* dset_name, int calc_corrL,
                    double* globalAvg, double* globalStdDev, double* corrL_out);
/* [host] Dataset names of a classic-format HDF5 file, one per line. */
int scarl_h5_list(const char* path, char* names, size_t len, char* msg, size_t msg_len);
/* [host] Overwrites the raw bytes of a contiguous dataset in place (nbytes
 * must equal its size), as write_time_on_hdf5 (SRC_F/write_output.f90:
 * 819-911) reopens a result file to write its times. */
int scarl_h5_overwrite_dataset(const char* path, const char* name, const void* data,
                               unsigned long long nbytes, char* msg, size_t msg_len);
/* [host] A numeric dataset of a classic-format HDF5 file (contiguous
 * layout), converted to dtype into out; dims receives its extents in
 * column-major order (HDF5 order reversed, 1 for missing axes), rank its
 * rank.  out == NULL: extents only. */
int scarl_h5_read_dataset(const char* path, const char* name, void* out, int dtype,
                          long long dims[3], int* rank, char* msg, size_t msg_len);
/* [host] A numeric attribute of the root group (object NULL or "") or of a
 * dataset, as doubles; count receives its number of elements. */
int scarl_h5_read_attr(const char* path, const char* object, const char* name, double* out,
                       int max_count, int* count, char* msg, size_t msg_len);

#ifdef __cplusplus
}
#endif
#endif
