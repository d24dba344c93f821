/*
 * scarl_oracle.h -- CPU FP64 restatement of the ScaRL random-field path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA implementation in scarl_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity pinning:
 *   - Park-Miller generator: pinned to the known-answer table in
 *     SRC_F/normal_ScaRL.f90:762-769.
 *   - FFTW 3.3.4/3.3.7 (not vendored in the reference, not installed here):
 *     the transforms are restated from FFTW's documented definitions
 *     (REDFT01 = unnormalised DCT-III, BACKWARD = unnormalised e^{+i}) and
 *     checked against scipy.fft.dct(type=3) / numpy.fft in tests/.
 *   - Fortran intrinsic random_number (compiler specific): not reproducible;
 *     both codes are fed the same injected arrays instead.
 *   - Philox4x32-10: checked against the Random123 published known-answer
 *     vectors in tests/.
 *   The reference itself (Fortran + MPI + FFTW + HDF5) cannot be compiled in
 *   this environment, so field-level parity is partially pinned: through the
 *   definitions above, not through reference output.
 *
 * Arrays are column-major (Fortran order, x fastest) like the reference.
 */
#ifndef SCARL_ORACLE_H
#define SCARL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* constants_ScaRL.f90:5 -- the reference's own (truncated) value of pi. */
#define SO_PI_REF 3.1415926535898

/* ---------------- random numbers ---------------- */
int32_t so_pm_step(int32_t seed);
void so_r8vec_uniform_01(int n, int32_t* seed, double* r);
void so_r8vec_normal_01(int n, int32_t* seed, double* x);
int32_t so_pm_jump(int32_t state, uint64_t n);
void so_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void so_normals(uint64_t seed, uint32_t stream, const int P[3], double* re_im);
void so_uniforms(uint64_t seed, uint32_t stream, uint64_t first, uint64_t n, double* u);
void so_ensemble_draw(uint64_t seed, int64_t first, int n, const int* choices, int nchoices,
                      double lmin, double lmax, int* Np, double* corrL);

/* ---------------- index maps ---------------- */
int so_verify_inputs(const double xMin[3], const double xMax[3], const double corrL[3],
                     const double overlap[3], double avg, double std_dev, int corrMod,
                     int margiFirst, const int ppcl[3], int gen_meth);
void so_find_factors(int n, int d[100]);
void so_decide_topo_shape(int nb_procs, const int L[3], const int ovlp[3],
                          int64_t ppbi, int topo[3]);
void so_get_topo_pos(int rank, const int shape[3], int pos[3]);
int so_get_topo_rank(const int shape[3], const int pos[3]);
int so_sample_layout(const double xMin[3], const double xMax[3], const double corrL[3],
                     const double overlap[3], const int ppcl[3], int gen_meth,
                     int nb_procs, const int* topo_in, int L[3], int Np[3],
                     int Np_ovlp[3], int topo[3], double xStep[3]);
void so_tile_geometry(const int Np[3], const int Np_ovlp[3], const int topo_pos[3],
                      const double xStep[3], const double xMin[3], int pos_0[3],
                      int pos_N[3], double coord_0[3], double coord_N[3], double xRange[3]);

/* ---------------- post steps ---------------- */
void so_unity_partition_weights(const int Np[3], const int Np_ovlp[3], int partitionType,
                                const int topo_pos[3], const int topo_shape[3], double* w);
void so_apply_unity_partition(const int Np[3], const int Np_ovlp[3], int partitionType,
                              const int topo_pos[3], const int topo_shape[3], double* f);
void so_add_overlap(double* const* RF, const int Np[3], const int Np_ovlp[3],
                    const int topo_shape[3]);
void so_normalize_field(double* const* RF, const int Np[3], const int Np_ovlp[3],
                        const int topo_shape[3], double* avg_out, double* std_out);
int so_multivariate_transformation(double avg, double std_dev, int margiFirst,
                                   double* f, int64_t n);
void so_assemble_global(double* const* RF, const int Np[3], const int Np_ovlp[3],
                        const int topo_shape[3], const int L[3], double* global);

/* ---------------- transforms ---------------- */
void so_fft1d(double* re_im, int n, int sign);
void so_dct3_1d(const double* in, double* out, int n);
void so_dct3_3d(const double* in, double* out, const int n[3]);
void so_c2c_3d(double* re_im, const int n[3], int sign);
void so_c2r_3d_crop(const double* H, const int P[3], const int Nout[3], double* out);

/* ---------------- generators ---------------- */
void so_gen_std_gauss_fft(double* out, const int Np[3], const double xRange[3],
                          const double corrL[3], const double* phiK, const double* gammaK);
void so_gen_std_gauss_fft_mpi(double* out, const int L[3], const double xRange[3],
                              const double corrL[3], const double* phiK, const double* gammaK);
int so_padded_size_literal(int Np);
int so_shino_sizes(const int Np[3], const double xRange[3], const double corrL[3],
                   int sz_c[3], int sz_Sk[3], double delta_k[3]);
void so_build_sk_mtx(int32_t seed, const int sz_Sk[3], const double delta_k[3], double* Sk);
void so_gen_std_gauss_shino_fft(double* out, const int Np[3], const double xRange[3],
                                const double corrL[3], int32_t seed, int via_c2c);
double so_spectrum(int corrMod, double nu, const double corrL[3], const double f[3]);
double so_spectrum_sum(int corrMod, double nu, const int P[3], const double dx[3],
                       const double corrL[3]);
void so_padded_spectrum(int corrMod, double nu, const int P[3], const double dx[3],
                        const double corrL[3], int normalise, uint64_t seed, uint32_t stream,
                        const double* xi, double* H);
void so_gen_padded(double* out, const int Np[3], const int P[3], const double dx[3],
                   const double corrL[3], int corrMod, double nu, int normalise,
                   uint64_t seed, uint32_t stream, const double* xi);
void so_gen_padded_stream(double* out, const int Np[3], const int P[3], const double dx[3],
                          const double corrL[3], int corrMod, double nu, double norm,
                          uint64_t seed, uint32_t stream, int line_stride);
int so_generate_sample(int generator, const double xMin[3], const double xMax[3],
                       const double corrL[3], const double overlap[3], const int ppcl[3],
                       int corrMod, double nu, int margiFirst, double avg, double std_dev,
                       int seedBase, int nb_procs, const int* topo_in, const int* pad,
                       int normalise_spectrum, int normalize_field, const double* phiK_all,
                       double* global);

/* ---------------- estimators ---------------- */
void so_moments(const double* f, int64_t xN, int nmc, double* evntAvg, double* evntStd,
                double* gAvg, double* gStd);
void so_tukey(int n, int literal, double* w);
/* Plain linear covariance along each axis, lags 0..maxlag, of the field
 * centred by its global mean (direct FP64 sums; cov has 3 (maxlag + 1)). */
void so_axis_cov(const double* f, const int L[3], int maxlag, double* mean, double* cov);
void so_rebuild_sk_fft(const double* f, const int L[3], int dir, double avg, double stdDev,
                       int tukey_literal, double* Sk);
void so_rebuild_corrL(const double* SkTot, const int nkeep[3], const double xStep[3],
                      double corrL_out[3]);

#ifdef __cplusplus
}
#endif
#endif
