/*
 * scarl_oracle.c -- CPU FP64 restatement of the ScaRL random-field path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for scarl_b200 and the timed
 * CPU baseline of bench.py.  Never linked into the product.
 * Each routine cites the reference routine it restates (paths relative to the
 * ScaRL source tree).  Parity pinning status is described in scarl_oracle.h.
 */
#include "scarl_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex zc;

#define SO_PM_M 2147483647
#define SO_PM_A 16807

/* ======================================================================== */
/* Random numbers                                                           */
/* ======================================================================== */

/* One Park-Miller step with Schrage's factorisation, exactly as
 * SRC_F/normal_ScaRL.f90:827-833 (int32 arithmetic, never overflows). */
int32_t so_pm_step(int32_t seed) {
  int32_t k = seed / 127773;
  seed = 16807 * (seed - k * 127773) - k * 2836;
  if (seed < 0) seed = seed + 2147483647;
  return seed;
}

/* SRC_F/normal_ScaRL.f90:1435-1516 (r8vec_uniform_01). */
void so_r8vec_uniform_01(int n, int32_t* seed, double* r) {
  for (int i = 0; i < n; ++i) {
    *seed = so_pm_step(*seed);
    r[i] = (double)(*seed) * 4.656612875E-10;
  }
}

/* SRC_F/normal_ScaRL.f90:1138-1259 (r8vec_normal_01, Box-Muller pairs). */
void so_r8vec_normal_01(int n, int32_t* seed, double* x) {
  const double r8_pi = 3.141592653589793;
  if (n <= 0) return;
  if (n == 1) {
    double r0, r1;
    so_r8vec_uniform_01(1, seed, &r0);
    so_r8vec_uniform_01(1, seed, &r1);
    x[0] = sqrt(-2.0 * log(r0)) * cos(2.0 * r8_pi * r1);
    return;
  }
  int hi = n; /* 1-based x_hi_index */
  int odd = ((hi - 1) % 2 == 0); /* mod(x_hi - x_lo, 2) == 0 -> odd count */
  if (!odd) {
    int m = n / 2;
    double* r = (double*)malloc(sizeof(double) * 2 * m);
    so_r8vec_uniform_01(2 * m, seed, r);
    for (int i = 0; i < m; ++i) {
      x[2 * i] = sqrt(-2.0 * log(r[2 * i])) * cos(2.0 * r8_pi * r[2 * i + 1]);
      x[2 * i + 1] = sqrt(-2.0 * log(r[2 * i])) * sin(2.0 * r8_pi * r[2 * i + 1]);
    }
    free(r);
  } else {
    int xh = n - 1;
    int m = xh / 2 + 1;
    double* r = (double*)malloc(sizeof(double) * 2 * m);
    so_r8vec_uniform_01(2 * m, seed, r);
    for (int i = 0; i < m - 1; ++i) {
      x[2 * i] = sqrt(-2.0 * log(r[2 * i])) * cos(2.0 * r8_pi * r[2 * i + 1]);
      x[2 * i + 1] = sqrt(-2.0 * log(r[2 * i])) * sin(2.0 * r8_pi * r[2 * i + 1]);
    }
    x[n - 1] = sqrt(-2.0 * log(r[2 * m - 2])) * cos(2.0 * r8_pi * r[2 * m - 1]);
    free(r);
  }
}

/* Jump-ahead for the Park-Miller recursion: 16807^n * state mod (2^31-1).
 * Valid for 0 <= state < 2^31-1 (every state after the first Schrage step),
 * where Schrage's formula and the modular product agree. */
int32_t so_pm_jump(int32_t state, uint64_t n) {
  uint64_t r = 1, b = SO_PM_A;
  while (n) {
    if (n & 1) r = (r * b) % SO_PM_M;
    b = (b * b) % SO_PM_M;
    n >>= 1;
  }
  return (int32_t)(((uint64_t)(uint32_t)state * r) % SO_PM_M);
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC11).  Counter-based: out = Philox(ctr, key). */
void so_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform in (0,1) from two 32-bit words: 52 random bits, half-offset, so
 * the value is exactly representable and never 0 or 1. */
static inline double so_u01(uint32_t hi, uint32_t lo) {
  uint64_t a = ((uint64_t)hi << 32) | lo;
  return (double)(a >> 12) * 0x1p-52 + 0x1p-53;
}

/* Box-Muller pair from two 32-bit words: u = (w + 1/2) 2^-32. */
static inline void so_bm(uint32_t a, uint32_t b, double* re, double* im) {
  double u1 = (double)a * 0x1p-32 + 0x1p-33;
  double u2 = (double)b * 0x1p-32 + 0x1p-33;
  double r = sqrt(-2.0 * log(u1));
  *re = r * cos(2.0 * M_PI * u2);
  *im = r * sin(2.0 * M_PI * u2);
}

/* Canonical standard normals of the padded spectrum: modes (kx, ky, kz0) and
 * (kx, ky, kz0 + P2/2), kz0 < P2/2, share the draw
 * Philox(ctr = {c_lo, c_hi, stream, 0}, key = {seed_lo, seed_hi}) with
 * c = kx + Hx (ky + P1 kz0); words (0,1) feed the first mode, (2,3) the
 * second.  out = {re0, im0, re1, im1}. */
static inline void so_mode_pair(const uint32_t key[2], uint32_t stream, int kx, int ky, int kz0,
                                int Hx, int P1, double out[4]) {
  const uint64_t c = (uint64_t)kx + (uint64_t)Hx * ((uint64_t)ky + (uint64_t)P1 * kz0);
  uint32_t ctr[4] = {(uint32_t)c, (uint32_t)(c >> 32), stream, 0u};
  uint32_t o[4];
  so_philox4x32_10(ctr, key, o);
  so_bm(o[0], o[1], out, out + 1);
  so_bm(o[2], o[3], out + 2, out + 3);
}

/* All canonical normals of a padded grid P, pairs in mode order
 * m = kx + Hx (ky + P1 kz). */
void so_normals(uint64_t seed, uint32_t stream, const int P[3], double* re_im) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const int Hx = P[0] / 2 + 1, h = P[2] / 2;
#pragma omp parallel for collapse(2) schedule(static)
  for (int kz0 = 0; kz0 < h; ++kz0)
    for (int ky = 0; ky < P[1]; ++ky)
      for (int kx = 0; kx < Hx; ++kx) {
        double o[4];
        so_mode_pair(key, stream, kx, ky, kz0, Hx, P[1], o);
        int64_t m0 = kx + (int64_t)Hx * (ky + (int64_t)P[1] * kz0);
        int64_t m1 = kx + (int64_t)Hx * (ky + (int64_t)P[1] * (kz0 + h));
        re_im[2 * m0] = o[0]; re_im[2 * m0 + 1] = o[1];
        re_im[2 * m1] = o[2]; re_im[2 * m1 + 1] = o[3];
      }
}

/* Canonical uniform phases (counter word 3 = 1) used when the DCT-path
 * generator is not given injected phases. */
void so_uniforms(uint64_t seed, uint32_t stream, uint64_t first, uint64_t n, double* u) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    uint64_t m = first + (uint64_t)i;
    uint32_t ctr[4] = {(uint32_t)m, (uint32_t)(m >> 32), stream, 1u};
    uint32_t o[4];
    so_philox4x32_10(ctr, key, o);
    u[i] = so_u01(o[0], o[1]);
  }
}

/* Shapes and correlation lengths of an ensemble of realisations (no
 * counterpart in the reference, which generates one sample per run,
 * SRC_F/main_ScaRL.f90:82-214).  Realisation r = first + i draws the four
 * words of Philox4x32-10 at counter {r, r >> 32, 0, 2}, key {seed, seed >> 32}:
 * axis d takes choices[floor(w_d * nchoices / 2^32)] points and the
 * isotropic correlation length is lmin + (lmax - lmin) (w_3 + 1/2) 2^-32. */
void so_ensemble_draw(uint64_t seed, int64_t first, int n, const int* choices, int nchoices,
                      double lmin, double lmax, int* Np, double* corrL) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int i = 0; i < n; ++i) {
    const uint64_t r = (uint64_t)(first + i);
    uint32_t ctr[4] = {(uint32_t)r, (uint32_t)(r >> 32), 0u, 2u};
    uint32_t w[4];
    so_philox4x32_10(ctr, key, w);
    for (int d = 0; d < 3; ++d)
      Np[3 * i + d] = choices[(int)(((uint64_t)w[d] * (uint64_t)nchoices) >> 32)];
    const double u = (double)w[3] * 0x1p-32 + 0x1p-33;
    const double l = lmin + (lmax - lmin) * u;
    corrL[3 * i] = corrL[3 * i + 1] = corrL[3 * i + 2] = l;
  }
}

/* ======================================================================== */
/* Index maps                                                               */
/* ======================================================================== */

/* SRC_F/main_ScaRL.f90:271-340 (verify_inputs).  Returns 0 when valid, else
 * the number of the failed rule (1..8). */
int so_verify_inputs(const double xMin[3], const double xMax[3], const double corrL[3],
                     const double overlap[3], double avg, double std_dev, int corrMod,
                     int margiFirst, const int ppcl[3], int gen_meth) {
  (void)overlap; /* negative overlap is only a warning in the reference */
  for (int d = 0; d < 3; ++d) if (xMin[d] >= xMax[d]) return 1;
  for (int d = 0; d < 3; ++d) if (corrL[d] < 0.0) return 2;
  if (corrMod != 1 && corrMod != 2 && corrMod != 3) return 3;
  if (margiFirst != 1 && margiFirst != 2) return 4;
  if (gen_meth != 1 && gen_meth != 2) return 5;
  if (avg <= 0.0 && margiFirst == 2) return 6;
  if (std_dev < 0.0) return 7;
  for (int d = 0; d < 3; ++d) if (ppcl[d] < 2) return 8;
  return 0;
}

/* SRC_F/main_ScaRL.f90:959-978 (find_factors). */
void so_find_factors(int n, int d[100]) {
  for (int i = 0; i < 100; ++i) d[i] = 0;
  int i = 0, div = 2, next = 3, rest = n;
  while (rest != 1 && rest > 0) {
    while (rest % div == 0) { d[i++] = div; rest /= div; }
    div = next; next += 2;
  }
}

static int so_maxloc3(const int v[3]) {
  int p = 0;
  for (int d = 1; d < 3; ++d) if (v[d] > v[p]) p = d;
  return p;
}

/* SRC_F/main_ScaRL.f90:834-893 (decide_topo_shape, localization branch).
 * vol_surf_factor is uninitialised in the reference; it starts at 0 here. */
void so_decide_topo_shape(int nb_procs, const int L[3], const int ovlp[3],
                          int64_t ppbi, int topo[3]) {
  int nBlocks[3] = {1, 1, 1}, nPPP[3], nBlocksIdeal[3], nFieldsIdeal[3];
  int nFieldsChosen[3] = {1, 1, 1};
  for (;;) {
    int64_t tot = 1;
    for (int d = 0; d < 3; ++d) {
      int nPoints = L[d] + (nBlocks[d] - 1) * ovlp[d];
      nPPP[d] = (int)ceil((double)nPoints / (double)nBlocks[d]);
      tot *= (int64_t)nPPP[d];
    }
    if (tot <= ppbi) break;
    if (nBlocks[0] * nBlocks[1] * nBlocks[2] >= nb_procs) break;
    nBlocks[so_maxloc3(nPPP)] += 1;
  }
  memcpy(nBlocksIdeal, nBlocks, sizeof nBlocks);
  int np_start = (int)ceilf(0.75f * (float)nb_procs);
  double vsf = 0.0;
  for (int np = np_start; np <= nb_procs; ++np) {
    int f[100];
    memcpy(nBlocks, nBlocksIdeal, sizeof nBlocks);
    nFieldsIdeal[0] = nFieldsIdeal[1] = nFieldsIdeal[2] = 1;
    so_find_factors(np, f);
    for (int i = 99; i >= 0; --i) {
      if (f[i] == 0) continue;
      if (nBlocks[0] == 1 && nBlocks[1] == 1 && nBlocks[2] == 1) break;
      int pos = so_maxloc3(nBlocks);
      nFieldsIdeal[pos] *= f[i];
      nBlocks[pos] = (int)ceil((double)nBlocks[pos] / (double)f[i]);
    }
    double vst = (double)(nFieldsIdeal[0] * nFieldsIdeal[1] * nFieldsIdeal[2]) /
                 (double)(2 * (nFieldsIdeal[0] * nFieldsIdeal[1] +
                               nFieldsIdeal[1] * nFieldsIdeal[2] +
                               nFieldsIdeal[2] * nFieldsIdeal[0]));
    if (vst >= vsf) { vsf = vst; memcpy(nFieldsChosen, nFieldsIdeal, sizeof nFieldsIdeal); }
  }
  memcpy(topo, nFieldsChosen, sizeof nFieldsChosen);
}

/* SRC_F/main_ScaRL.f90:747-764 (get_topo_pos). */
void so_get_topo_pos(int rank, const int shape[3], int pos[3]) {
  int rest = rank;
  pos[2] = rest / (shape[0] * shape[1]);
  rest -= pos[2] * shape[0] * shape[1];
  pos[1] = rest / shape[0];
  rest -= pos[1] * shape[0];
  pos[0] = rest;
}

/* SRC_F/main_ScaRL.f90:770-782 (get_topo_rank). */
int so_get_topo_rank(const int shape[3], const int pos[3]) {
  return shape[0] * shape[1] * pos[2] + shape[0] * pos[1] + pos[0];
}

/* SRC_F/main_ScaRL.f90:100-111 and 157-176: xStep, L, Np_ovlp, topology,
 * Np (with the overlap clamps) and the re-fitted L.  gen_meth 2 (FFT_MPI)
 * uses FFTW-MPI's block slab count along axis 3 (decide_topo_shape :818-833). */
int so_sample_layout(const double xMin[3], const double xMax[3], const double corrL[3],
                     const double overlap[3], const int ppcl[3], int gen_meth,
                     int nb_procs, const int* topo_in, int L[3], int Np[3],
                     int Np_ovlp[3], int topo[3], double xStep[3]) {
  for (int d = 0; d < 3; ++d) {
    xStep[d] = corrL[d] / ((double)(ppcl[d] - 1));
    L[d] = 1 + (int)ceil((xMax[d] - xMin[d]) / xStep[d]);
    Np_ovlp[d] = (gen_meth == 2) ? 0 : 1 + (int)ceil(overlap[d] * (double)(ppcl[d] - 1));
  }
  if (topo_in) {
    if (topo_in[0] * topo_in[1] * topo_in[2] != nb_procs) return -1;
    memcpy(topo, topo_in, 3 * sizeof(int));
  } else if (gen_meth == 2) {
    int blk = (L[2] + nb_procs - 1) / nb_procs;
    topo[0] = 1; topo[1] = 1; topo[2] = (L[2] + blk - 1) / blk;
  } else {
    so_decide_topo_shape(nb_procs, L, Np_ovlp, 1, topo);
  }
  for (int d = 0; d < 3; ++d) {
    Np[d] = (int)ceil((double)(L[d] + (topo[d] - 1) * Np_ovlp[d]) / (double)topo[d]);
    if (topo[d] == 2 && Np[d] < Np_ovlp[d]) Np[d] = Np_ovlp[d];
    if (topo[d] >= 3 && Np[d] < 2 * Np_ovlp[d]) Np[d] = 2 * Np_ovlp[d];
    L[d] = Np[d] * topo[d] - (topo[d] - 1) * Np_ovlp[d];
  }
  return 0;
}

/* SRC_F/main_ScaRL.f90:455-459 (create_fields: pos_0, pos_N, coord_0/N, xRange). */
void so_tile_geometry(const int Np[3], const int Np_ovlp[3], const int topo_pos[3],
                      const double xStep[3], const double xMin[3], int pos_0[3],
                      int pos_N[3], double coord_0[3], double coord_N[3], double xRange[3]) {
  for (int d = 0; d < 3; ++d) {
    pos_0[d] = (Np[d] - Np_ovlp[d]) * topo_pos[d] + 1;
    pos_N[d] = pos_0[d] + Np[d] - 1;
    coord_0[d] = (double)(pos_0[d] - 1) * xStep[d] + xMin[d];
    coord_N[d] = (double)(pos_N[d] - 1) * xStep[d] + xMin[d];
    xRange[d] = coord_N[d] - coord_0[d];
  }
}

/* ======================================================================== */
/* Post steps                                                               */
/* ======================================================================== */

/* SRC_F/main_ScaRL.f90:1236-1294: the full partition-of-unity weight array,
 * multiplied in the reference's order (low side x,y,z then high side x,y,z). */
void so_unity_partition_weights(const int Np[3], const int Np_ovlp[3], int partitionType,
                                const int topo_pos[3], const int topo_shape[3], double* w) {
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) w[i] = 1.0;
  for (int jj = 1; jj <= 2; ++jj) {
    for (int ii = 0; ii < 3; ++ii) {
      int shift = (jj == 1) ? -1 : 1;
      if (Np_ovlp[ii] < 2) continue;
      if (topo_pos[ii] + shift < 0 || topo_pos[ii] + shift > topo_shape[ii] - 1) continue;
      int no = Np_ovlp[ii];
      double* pat = (double*)malloc(sizeof(double) * no);
      for (int kk = 0; kk < no; ++kk) pat[kk] = (double)kk / (double)(no - 1);
      if (jj == 1)
        for (int a = 0, b = no - 1; a < b; ++a, --b) { double t = pat[a]; pat[a] = pat[b]; pat[b] = t; }
      if (partitionType == 1)
        for (int kk = 0; kk < no; ++kk) pat[kk] = (1.0 + cos(SO_PI_REF * pat[kk])) / 2.0;
      int D = (jj == 1) ? 0 : Np[ii] - no;
      /* every point of plane D + t (index ii) takes factor pat[t]; a point
       * lies in one plane per (jj, ii), so the product order per point is
       * the reference's */
#pragma omp parallel for schedule(static)
      for (int k = 0; k < Np[2]; ++k)
        for (int j = 0; j < Np[1]; ++j)
          for (int i = 0; i < Np[0]; ++i) {
            const int c = ii == 0 ? i : (ii == 1 ? j : k);
            if (c < D || c >= D + no) continue;
            w[i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)] *= pat[c - D];
          }
      free(pat);
    }
  }
}

/* SRC_F/main_ScaRL.f90:1216-1301 (apply_UnityPartition_mtx): field *= sqrt(w). */
void so_apply_unity_partition(const int Np[3], const int Np_ovlp[3], int partitionType,
                              const int topo_pos[3], const int topo_shape[3], double* f) {
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  double* w = (double*)malloc(sizeof(double) * n);
  so_unity_partition_weights(Np, Np_ovlp, partitionType, topo_pos, topo_shape, w);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) f[i] = f[i] * sqrt(w[i]);
  free(w);
}

static void so_region(const int s[3], const int Np[3], const int Np_ovlp[3], int minP[3],
                      int maxP[3]) {
  for (int d = 0; d < 3; ++d) {
    minP[d] = 1; maxP[d] = Np[d];
    if (s[d] == 1) minP[d] = Np[d] - Np_ovlp[d] + 1;
    if (s[d] == -1) maxP[d] = Np_ovlp[d];
  }
}

/* SRC_F/main_ScaRL.f90:984-1210 (add_overlap) over simulated ranks: every
 * rank sends its region for direction s to rank+s and accumulates what rank-s
 * sent, in the reference's 27-direction order; then RF = RF + accumulated. */
void so_add_overlap(double* const* RF, const int Np[3], const int Np_ovlp[3],
                    const int topo_shape[3]) {
  const int nb = topo_shape[0] * topo_shape[1] * topo_shape[2];
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  double** acc = (double**)malloc(sizeof(double*) * nb);
  for (int r = 0; r < nb; ++r) acc[r] = (double*)calloc(n, sizeof(double));
  for (int r = 0; r < nb; ++r) {
    int pos[3];
    so_get_topo_pos(r, topo_shape, pos);
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          int s[3] = {ii, jj, kk};
          int ms[3] = {-ii, -jj, -kk};
          int src[3] = {pos[0] - ii, pos[1] - jj, pos[2] - kk};
          int dst[3] = {pos[0] - ii, pos[1] - jj, pos[2] - kk};
          (void)dst;
          /* receiver side: neigh_rank(op_dir) == rank when rank-s is outside */
          int inside = 1;
          for (int d = 0; d < 3; ++d) if (src[d] < 0 || src[d] > topo_shape[d] - 1) inside = 0;
          if (!inside) continue;
          if (ii == 0 && jj == 0 && kk == 0) continue;
          int minR[3], maxR[3], minS[3], maxS[3];
          so_region(ms, Np, Np_ovlp, minR, maxR);
          so_region(s, Np, Np_ovlp, minS, maxS);
          int degen = 0;
          for (int d = 0; d < 3; ++d) if (maxR[d] <= minR[d]) degen = 1;
          if (degen) continue;
          const double* sf = RF[so_get_topo_rank(topo_shape, src)];
          for (int k = 0; k <= maxR[2] - minR[2]; ++k)
            for (int j = 0; j <= maxR[1] - minR[1]; ++j)
              for (int i = 0; i <= maxR[0] - minR[0]; ++i) {
                int64_t ir = (minR[0] - 1 + i) + (int64_t)Np[0] * ((minR[1] - 1 + j) + (int64_t)Np[1] * (minR[2] - 1 + k));
                int64_t is = (minS[0] - 1 + i) + (int64_t)Np[0] * ((minS[1] - 1 + j) + (int64_t)Np[1] * (minS[2] - 1 + k));
                acc[r][ir] = acc[r][ir] + sf[is];
              }
        }
  }
  for (int r = 0; r < nb; ++r) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) RF[r][i] = RF[r][i] + acc[r][i];
    free(acc[r]);
  }
  free(acc);
}

/* SRC_F/main_ScaRL.f90:903-953 (normalize_field, disabled in the reference's
 * driver at :565-567) over simulated ranks, reductions summed in rank order. */
void so_normalize_field(double* const* RF, const int Np[3], const int Np_ovlp[3],
                        const int topo_shape[3], double* avg_out, double* std_out) {
  const int nb = topo_shape[0] * topo_shape[1] * topo_shape[2];
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  int64_t xNTotal = 1;
  for (int d = 0; d < 3; ++d)
    xNTotal *= (int64_t)topo_shape[d] * (Np[d] - Np_ovlp[d]) + Np_ovlp[d];
  double* part = (double*)malloc(sizeof(double) * nb);
  int maxPos[3];
  for (int r = 0; r < nb; ++r) {
    int pos[3];
    so_get_topo_pos(r, topo_shape, pos);
    for (int d = 0; d < 3; ++d) maxPos[d] = (pos[d] != topo_shape[d] - 1) ? Np[d] - Np_ovlp[d] : Np[d];
    double s = 0.0;
    for (int k = 0; k < maxPos[2]; ++k)
      for (int j = 0; j < maxPos[1]; ++j)
        for (int i = 0; i < maxPos[0]; ++i) s += RF[r][i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)];
    part[r] = s;
  }
  double tot = 0.0;
  for (int r = 0; r < nb; ++r) tot += part[r];
  double avg = tot / (double)xNTotal;
  for (int r = 0; r < nb; ++r) for (int64_t i = 0; i < n; ++i) RF[r][i] = RF[r][i] - avg;
  for (int r = 0; r < nb; ++r) {
    int pos[3];
    so_get_topo_pos(r, topo_shape, pos);
    for (int d = 0; d < 3; ++d) maxPos[d] = (pos[d] != topo_shape[d] - 1) ? Np[d] - Np_ovlp[d] : Np[d];
    double s = 0.0;
    for (int k = 0; k < maxPos[2]; ++k)
      for (int j = 0; j < maxPos[1]; ++j)
        for (int i = 0; i < maxPos[0]; ++i) {
          double v = RF[r][i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)];
          s += v * v;
        }
    part[r] = s;
  }
  tot = 0.0;
  for (int r = 0; r < nb; ++r) tot += part[r];
  double sd = sqrt(tot / (double)xNTotal);
  for (int r = 0; r < nb; ++r) for (int64_t i = 0; i < n; ++i) RF[r][i] = RF[r][i] / sd;
  free(part);
  if (avg_out) *avg_out = avg;
  if (std_out) *std_out = sd;
}

/* SRC_F/main_ScaRL.f90:1355-1395 (multiVariateTransformation). */
int so_multivariate_transformation(double avg, double std_dev, int margiFirst,
                                   double* f, int64_t n) {
  double normalVar, normalAvg;
  if (margiFirst == 1) {
    normalVar = std_dev * std_dev;
    normalAvg = avg;
  } else if (margiFirst == 2) {
    if (avg <= 0.0) return -1;
    double cv = std_dev / avg;
    normalVar = log(1.0 + cv * cv);
    normalAvg = log(avg) - normalVar / 2.0;
  } else {
    return -2;
  }
  double s = sqrt(normalVar);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double v = f[i] * s + normalAvg;
    f[i] = (margiFirst == 2) ? exp(v) : v;
  }
  return 0;
}

/* SRC_F/write_output.f90:373-431 (write_hdf5_multi_proc_3D_1ds): every rank's
 * block is written at pos_0-1 in rank order; later ranks overwrite. */
void so_assemble_global(double* const* RF, const int Np[3], const int Np_ovlp[3],
                        const int topo_shape[3], const int L[3], double* global) {
  const int nb = topo_shape[0] * topo_shape[1] * topo_shape[2];
  for (int r = 0; r < nb; ++r) {
    int pos[3];
    so_get_topo_pos(r, topo_shape, pos);
    int o[3];
    for (int d = 0; d < 3; ++d) o[d] = (Np[d] - Np_ovlp[d]) * pos[d];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Np[2]; ++k)
      for (int j = 0; j < Np[1]; ++j)
        for (int i = 0; i < Np[0]; ++i)
          global[(o[0] + i) + (int64_t)L[0] * ((o[1] + j) + (int64_t)L[1] * (o[2] + k))] =
              RF[r][i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)];
  }
}

/* ======================================================================== */
/* Transforms (FFTW definitions restated; FFTW itself is not available)      */
/* ======================================================================== */

typedef struct {
  int n;
  int pow2;
  int nf, fac[32]; /* mixed radix: radices 4, 2, 3, 5, 7 whose product is n (nf > 0) */
  zc* tw;      /* e^{-2 pi i k / n}, k < n (pow2 and mixed radix) */
  int* rev;
  int m;       /* Bluestein convolution length */
  zc* chirp;   /* e^{-i pi k^2 / n} */
  zc* bfft;    /* FFT_m of the conjugate chirp, wrapped */
} so_plan;

#define SO_MAX_PLANS 64
static so_plan* so_plans[SO_MAX_PLANS];
static int so_nplans = 0;

static void so_fft_pow2(const so_plan* p, zc* x) {
  int n = p->n;
  for (int i = 0; i < n; ++i) {
    int j = p->rev[i];
    if (j > i) { zc t = x[i]; x[i] = x[j]; x[j] = t; }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int s = 0; s < n; s += len)
      for (int k = 0; k < half; ++k) {
        zc w = p->tw[k * step];
        zc a = x[s + k], b = x[s + k + half] * w;
        x[s + k] = a + b;
        x[s + k + half] = a - b;
      }
  }
}

static so_plan* so_plan_get(int n);

/* n as a product of the radices 4, 2, 3, 5, 7 (fours first); 0 when n has
 * another prime factor. */
static int so_factor(int n, int fac[32], int* nf) {
  int k = 0;
  const int rad[5] = {4, 2, 3, 5, 7};
  for (int i = 0; i < 5 && n > 1; ++i)
    while (n % rad[i] == 0 && k < 32) { fac[k++] = rad[i]; n /= rad[i]; }
  *nf = n == 1 ? k : 0;
  return n == 1;
}

/* Unnormalised forward DFT by Stockham autosort over the plan's radices
 * (Govindaraju et al., SC08): stage s with span Ns reads x[j + q n / R],
 * twiddles by e^{-2 pi i q (j mod Ns) / (Ns R)}, takes a length-R DFT and
 * writes y[(j / Ns) Ns R + (j mod Ns) + u Ns]. */
static void so_fft_mixed(const so_plan* p, zc* x) {
  const int n = p->n;
  zc* buf = (zc*)malloc(sizeof(zc) * n);
  zc* a = x;
  zc* b = buf;
  int Ns = 1;
  for (int s = 0; s < p->nf; ++s) {
    const int R = p->fac[s], stride = n / R, tstep = n / (Ns * R);
    for (int j = 0; j < stride; ++j) {
      zc v[8], y[8];
      const int k = j % Ns;
      for (int q = 0; q < R; ++q) v[q] = a[j + q * stride] * p->tw[q * k * tstep];
      if (R == 2) {
        y[0] = v[0] + v[1];
        y[1] = v[0] - v[1];
      } else if (R == 4) {
        const zc t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3], d = v[1] - v[3];
        const zc t3 = cimag(d) - I * creal(d); /* -i (v1 - v3) */
        y[0] = t0 + t2; y[2] = t0 - t2; y[1] = t1 + t3; y[3] = t1 - t3;
      } else {
        for (int u = 0; u < R; ++u) {
          zc acc = v[0];
          for (int q = 1; q < R; ++q) acc += v[q] * p->tw[((u * q) % R) * stride];
          y[u] = acc;
        }
      }
      const int d = (j / Ns) * Ns * R + k;
      for (int u = 0; u < R; ++u) b[d + u * Ns] = y[u];
    }
    zc* t = a; a = b; b = t;
    Ns *= R;
  }
  if (a != x) memcpy(x, a, sizeof(zc) * n);
  free(buf);
}

static so_plan* so_plan_make(int n) {
  so_plan* p = (so_plan*)calloc(1, sizeof(so_plan));
  p->n = n;
  p->pow2 = (n & (n - 1)) == 0;
  if (p->pow2) {
    p->tw = (zc*)malloc(sizeof(zc) * n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      p->tw[k] = cos(a) + I * sin(a);
    }
    p->rev = (int*)malloc(sizeof(int) * n);
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      p->rev[i] = r;
    }
  } else if (so_factor(n, p->fac, &p->nf)) {
    p->tw = (zc*)malloc(sizeof(zc) * n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      p->tw[k] = cos(a) + I * sin(a);
    }
  } else {
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (zc*)malloc(sizeof(zc) * n);
    for (int k = 0; k < n; ++k) {
      int64_t q = ((int64_t)k * k) % (2 * (int64_t)n);
      double a = -M_PI * (double)q / (double)n;
      p->chirp[k] = cos(a) + I * sin(a);
    }
    p->bfft = (zc*)calloc(m, sizeof(zc));
    for (int k = 0; k < n; ++k) {
      p->bfft[k] = conj(p->chirp[k]);
      if (k) p->bfft[m - k] = conj(p->chirp[k]);
    }
    so_fft_pow2(so_plan_get(m), p->bfft);
  }
  return p;
}

static so_plan* so_plan_get(int n) {
  so_plan* p = NULL;
#pragma omp critical(so_plan_cache)
  {
    for (int i = 0; i < so_nplans; ++i) if (so_plans[i]->n == n) { p = so_plans[i]; break; }
  }
  if (p) return p;
  so_plan* q = so_plan_make(n);
#pragma omp critical(so_plan_cache)
  {
    for (int i = 0; i < so_nplans; ++i) if (so_plans[i]->n == n) { p = so_plans[i]; break; }
    if (!p && so_nplans < SO_MAX_PLANS) { so_plans[so_nplans++] = q; p = q; q = NULL; }
  }
  if (q) { /* lost the race or cache full: keep the fresh plan leaked-free */
    if (!p) p = q; else { free(q->tw); free(q->rev); free(q->chirp); free(q->bfft); free(q); }
  }
  return p;
}

/* Unnormalised forward (sign -1) DFT of length n, any n. */
static void so_fft_fwd(zc* x, int n) {
  if (n <= 1) return;
  so_plan* p = so_plan_get(n);
  if (p->pow2) { so_fft_pow2(p, x); return; }
  if (p->nf) { so_fft_mixed(p, x); return; }
  /* Bluestein: X_k = c_k * sum_j (x_j c_j) conj(c_{k-j}) */
  int m = p->m;
  so_plan* pm = so_plan_get(m);
  zc* a = (zc*)calloc(m, sizeof(zc));
  for (int k = 0; k < n; ++k) a[k] = x[k] * p->chirp[k];
  so_fft_pow2(pm, a);
  for (int k = 0; k < m; ++k) a[k] *= p->bfft[k];
  for (int k = 0; k < m; ++k) a[k] = conj(a[k]);
  so_fft_pow2(pm, a);
  for (int k = 0; k < m; ++k) a[k] = conj(a[k]) / (double)m;
  for (int k = 0; k < n; ++k) x[k] = a[k] * p->chirp[k];
  free(a);
}

static void so_fft_sign(zc* x, int n, int sign) {
  if (sign < 0) { so_fft_fwd(x, n); return; }
  for (int i = 0; i < n; ++i) x[i] = conj(x[i]);
  so_fft_fwd(x, n);
  for (int i = 0; i < n; ++i) x[i] = conj(x[i]);
}

/* FFTW_FORWARD (sign -1) / FFTW_BACKWARD (sign +1), unnormalised. */
void so_fft1d(double* re_im, int n, int sign) { so_fft_sign((zc*)re_im, n, sign); }

/* FFTW REDFT01 (DCT-III): y_k = x_0 + 2 sum_{j>=1} x_j cos(pi j (2k+1) / (2n)),
 * with an exactly reduced angle index. */
static void so_dct3_line(const double* x, int stride_in, double* y, int stride_out, int n,
                         const double* ctab) {
  int last = -1;
  for (int j = n - 1; j >= 0; --j) if (x[(int64_t)j * stride_in] != 0.0) { last = j; break; }
  for (int k = 0; k < n; ++k) {
    double s = x[0];
    for (int j = 1; j <= last; ++j) {
      int64_t m = ((int64_t)j * (2 * k + 1)) % (4 * (int64_t)n);
      s += 2.0 * x[(int64_t)j * stride_in] * ctab[m];
    }
    y[(int64_t)k * stride_out] = (last < 0) ? 0.0 : s;
  }
}

static double* so_dct_table(int n) {
  double* c = (double*)malloc(sizeof(double) * 4 * n);
  for (int m = 0; m < 4 * n; ++m) c[m] = cos(M_PI * (double)m / (2.0 * (double)n));
  return c;
}

void so_dct3_1d(const double* in, double* out, int n) {
  double* c = so_dct_table(n);
  so_dct3_line(in, 1, out, 1, n, c);
  free(c);
}

/* 3D REDFT01 (fftw_plan_r2r_3d with REDFT01 on all axes), out of place. */
void so_dct3_3d(const double* in, double* out, const int n[3]) {
  const int64_t N = (int64_t)n[0] * n[1] * n[2];
  double* a = (double*)malloc(sizeof(double) * N);
  double* b = (double*)malloc(sizeof(double) * N);
  memcpy(a, in, sizeof(double) * N);
  double* c0 = so_dct_table(n[0]);
  double* c1 = so_dct_table(n[1]);
  double* c2 = so_dct_table(n[2]);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j) {
      int64_t o = (int64_t)n[0] * (j + (int64_t)n[1] * k);
      so_dct3_line(a + o, 1, b + o, 1, n[0], c0);
    }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < n[2]; ++k)
    for (int i = 0; i < n[0]; ++i) {
      int64_t o = i + (int64_t)n[0] * n[1] * k;
      so_dct3_line(b + o, n[0], a + o, n[0], n[1], c1);
    }
#pragma omp parallel for collapse(2) schedule(static)
  for (int j = 0; j < n[1]; ++j)
    for (int i = 0; i < n[0]; ++i) {
      int64_t o = i + (int64_t)n[0] * j;
      so_dct3_line(a + o, n[0] * n[1], out + o, n[0] * n[1], n[2], c2);
    }
  free(a); free(b); free(c0); free(c1); free(c2);
}

/* 3D complex DFT (FFTW_FORWARD/BACKWARD, unnormalised), in place. */
void so_c2c_3d(double* re_im, const int n[3], int sign) {
  zc* x = (zc*)re_im;
  so_plan_get(n[0]); so_plan_get(n[1]); so_plan_get(n[2]);
  for (int ax = 0; ax < 3; ++ax) {
    int len = n[ax];
    int64_t stride = ax == 0 ? 1 : (ax == 1 ? n[0] : (int64_t)n[0] * n[1]);
    int o1 = ax == 0 ? n[1] : n[0];
    int o2 = ax == 2 ? n[1] : n[2];
    int64_t s1 = ax == 0 ? n[0] : 1;
    int64_t s2 = ax == 2 ? n[0] : (int64_t)n[0] * n[1];
#pragma omp parallel for collapse(2) schedule(static)
    for (int b = 0; b < o2; ++b)
      for (int a = 0; a < o1; ++a) {
        zc* line = (zc*)malloc(sizeof(zc) * len);
        int64_t base = a * s1 + b * s2;
        for (int t = 0; t < len; ++t) line[t] = x[base + t * stride];
        so_fft_sign(line, len, sign);
        for (int t = 0; t < len; ++t) x[base + t * stride] = line[t];
        free(line);
      }
  }
}

/* Real output of the padded periodic grid, cropped to Nout:
 *   out(n) = Re sum_{kx=0}^{P0/2} w(kx) sum_{ky,kz} H e^{+2 pi i k.n / P},
 * w = 1 on the kx = 0 and kx = P0/2 planes and 2 elsewhere (numpy irfftn
 * semantics times prod(P)).  H is stored kx fastest with Hx = P0/2+1.  Only
 * the outputs inside the crop are formed: z-lines keep z < Nout[2], then
 * y-lines keep y < Nout[1], then x-lines keep x < Nout[0]. */
void so_c2r_3d_crop(const double* Hd, const int P[3], const int Nout[3], double* out) {
  const zc* H = (const zc*)Hd;
  const int Hx = P[0] / 2 + 1;
  const int Nz = Nout[2], Ny = Nout[1], Nx = Nout[0];
  zc* T = (zc*)malloc(sizeof(zc) * (int64_t)Hx * P[1] * Nz);
  so_plan_get(P[0]); so_plan_get(P[1]); so_plan_get(P[2]);
#pragma omp parallel
  {
    zc* line = (zc*)malloc(sizeof(zc) * (P[0] > P[1] ? (P[0] > P[2] ? P[0] : P[2]) : (P[1] > P[2] ? P[1] : P[2])));
#pragma omp for collapse(2) schedule(static)
    for (int ky = 0; ky < P[1]; ++ky)
      for (int kx = 0; kx < Hx; ++kx) {
        for (int kz = 0; kz < P[2]; ++kz) line[kz] = H[kx + (int64_t)Hx * (ky + (int64_t)P[1] * kz)];
        so_fft_sign(line, P[2], +1);
        for (int z = 0; z < Nz; ++z) T[kx + (int64_t)Hx * (ky + (int64_t)P[1] * z)] = line[z];
      }
#pragma omp for collapse(2) schedule(static)
    for (int z = 0; z < Nz; ++z)
      for (int kx = 0; kx < Hx; ++kx) {
        for (int ky = 0; ky < P[1]; ++ky) line[ky] = T[kx + (int64_t)Hx * (ky + (int64_t)P[1] * z)];
        so_fft_sign(line, P[1], +1);
        for (int y = 0; y < Ny; ++y) T[kx + (int64_t)Hx * (y + (int64_t)P[1] * z)] = line[y];
      }
#pragma omp for collapse(2) schedule(static)
    for (int z = 0; z < Nz; ++z)
      for (int y = 0; y < Ny; ++y) {
        const zc* X = T + (int64_t)Hx * (y + (int64_t)P[1] * z);
        for (int k = 0; k < P[0]; ++k) {
          if (k == 0) line[k] = creal(X[0]);
          else if (2 * k == P[0]) line[k] = creal(X[k]);
          else if (k < Hx) line[k] = X[k];
          else line[k] = conj(X[P[0] - k]);
        }
        so_fft_sign(line, P[0], +1);
        for (int x = 0; x < Nx; ++x) out[x + (int64_t)Nx * (y + (int64_t)Ny * z)] = creal(line[x]);
      }
    free(line);
  }
  free(T);
}

/* ======================================================================== */
/* Generators                                                               */
/* ======================================================================== */

/* SRC_F/fftw_ScaRL.f90:261-418 (gen_std_gauss_FFT), Gaussian model:
 *   delta_x = xRange/(Np-1), k_max = 1/delta_x, delta_k = k_max/(Np-1)
 *   k_i = (i-1) delta_k / corrL on the (Np/2)^3 octant
 *   S = prod_d corrL_d exp(-PI k_d^2), Sk = gamma sqrt(S) cos(2 PI phi)
 *   out = unnormalised 3D REDFT01 of Sk over Np.
 * The region outside the octant is uninitialised in the reference
 * (:317, :370); it is zero here.  gamma is the injected amplitude (the
 * reference overwrites it with 1, :367): gammaK == NULL means 1. */
static void so_dct_generator(double* out, const int Np[3], const double xRange[3],
                             const double corrL[3], const double* phiK, const double* gammaK,
                             int full_z) {
  int K[3];
  double dk[3];
  for (int d = 0; d < 3; ++d) {
    K[d] = (full_z && d == 2) ? Np[d] : Np[d] / 2;
    double delta_x = xRange[d] / (double)(Np[d] - 1);
    double k_max = 1.0 / delta_x;
    dk[d] = k_max / (double)(Np[d] - 1);
  }
  const int64_t N = (int64_t)Np[0] * Np[1] * Np[2];
  double* Sk = (double*)calloc(N, sizeof(double));
  for (int k = 0; k < K[2]; ++k)
    for (int j = 0; j < K[1]; ++j)
      for (int i = 0; i < K[0]; ++i) {
        int idx[3] = {i, j, k};
        double S = 1.0;
        for (int d = 0; d < 3; ++d) {
          double kp = (double)idx[d] * dk[d] / corrL[d];
          S = S * corrL[d] * exp(-SO_PI_REF * (kp * kp));
        }
        int64_t o = i + (int64_t)K[0] * (j + (int64_t)K[1] * k);
        double g = gammaK ? gammaK[o] : 1.0;
        Sk[i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)] = g * sqrt(S) * cos(2.0 * SO_PI_REF * phiK[o]);
      }
  so_dct3_3d(Sk, out, Np);
  free(Sk);
}

void so_gen_std_gauss_fft(double* out, const int Np[3], const double xRange[3],
                          const double corrL[3], const double* phiK, const double* gammaK) {
  so_dct_generator(out, Np, xRange, corrL, phiK, gammaK, 0);
}

/* gen_Std_Gauss_FFT_MPI (SRC_F/fftw_ScaRL.f90:424-583) for one rank: the same
 * spectrum and DCT-III with the spectrum over every kz (:469-476); phases
 * (L0/2)(L1/2)L2 in x-fastest order. */
void so_gen_std_gauss_fft_mpi(double* out, const int L[3], const double xRange[3],
                              const double corrL[3], const double* phiK, const double* gammaK) {
  so_dct_generator(out, L, xRange, corrL, phiK, gammaK, 1);
}

/* SRC_F/fftw_ScaRL.f90:194: sz_c = 2**ceiling(log(dble(2*Np))/log(2d0)). */
int so_padded_size_literal(int Np) {
  return 1 << (int)ceil(log((double)(2 * Np)) / log(2.0));
}

/* SRC_F/spectra_ScaRL.f90:44-56 (build_Sk_mtx sizes, Gaussian).  The
 * reference's coarse-mesh branch (:50-54) raises k_cut on the fine axes and
 * leaves the coarse ones past the padded grid; k_cut is clamped to k_max here
 * (the truncation its message announces).  Returns 1 when clamped. */
int so_shino_sizes(const int Np[3], const double xRange[3], const double corrL[3],
                   int sz_c[3], int sz_Sk[3], double delta_k[3]) {
  int clamped = 0;
  for (int d = 0; d < 3; ++d) {
    double xr = xRange[d] / corrL[d];
    sz_c[d] = so_padded_size_literal(Np[d]);
    double delta_x = xr / (double)(Np[d] - 1);
    double k_max = 1.0 / delta_x;
    delta_k[d] = k_max / (double)(sz_c[d] / 2);
    double k_cut = 7.355;
    if (k_max < k_cut) { k_cut = k_max; clamped = 1; }
    sz_Sk[d] = (int)ceil(k_cut / delta_k[d]);
    if (sz_Sk[d] > sz_c[d] / 2) sz_Sk[d] = sz_c[d] / 2;
  }
  return clamped;
}

/* SRC_F/spectra_ScaRL.f90:74-117 (build_Sk_mtx, Gaussian): unit phases from
 * Park-Miller(seed + 1000000) over the (sz1, 2 sz2, 2 sz3) array, rounded to
 * default (single precision) complex by CMPLX (:80), boundary planes zeroed,
 * mirrored Gaussian amplitude, then sqrt(8) and 2 sqrt(prod delta_k).
 * Sk is complex (re, im interleaved), column-major. */
void so_build_sk_mtx(int32_t seed, const int sz_Sk[3], const double delta_k[3], double* Skd) {
  zc* Sk = (zc*)Skd;
  const int n1 = sz_Sk[0], n2 = 2 * sz_Sk[1], n3 = 2 * sz_Sk[2];
  const int64_t N = (int64_t)n1 * n2 * n3;
  int32_t s = (int32_t)((uint32_t)seed + 1000000u);
  for (int64_t e = 0; e < N; ++e) {
    s = so_pm_step(s);
    double u = (double)s * 4.656612875E-10;
    double ph = 2.0 * SO_PI_REF * u;
    Sk[e] = (double)(float)cos(ph) + I * (double)(float)sin(ph);
  }
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i)
        if (i == 0 || j == 0 || k == 0 || j == n2 - 1 || k == n3 - 1)
          Sk[i + (int64_t)n1 * (j + (int64_t)n2 * k)] = 0.0;
  double de[3];
  for (int d = 0; d < 3; ++d) de[d] = ((SO_PI_REF * SO_PI_REF) / 2.0) * (delta_k[d] * delta_k[d]);
  for (int ii = 2; ii <= sz_Sk[0]; ++ii)
    for (int jj = 2; jj <= sz_Sk[1]; ++jj)
      for (int kk = 2; kk <= sz_Sk[2]; ++kk) {
        double a = (double)(ii - 1), b = (double)(jj - 1), c = (double)(kk - 1);
        double sv = sqrt(exp(-((a * a * de[0] + b * b * de[1]) + c * c * de[2])));
        int jm = n2 - jj + 1, km = n3 - kk + 1;
#define SKI(I_, J_, K_) Sk[((I_) - 1) + (int64_t)n1 * (((J_) - 1) + (int64_t)n2 * ((K_) - 1))]
        SKI(ii, jj, kk) *= sv;
        SKI(ii, jm, kk) *= sv;
        SKI(ii, jj, km) *= sv;
        SKI(ii, jm, km) *= sv;
#undef SKI
      }
  double pdk = (delta_k[0] * delta_k[1]) * delta_k[2];
  double f = 2.0 * sqrt(pdk);
  for (int64_t e = 0; e < N; ++e) {
    Sk[e] = sqrt(8.0) * Sk[e];
    Sk[e] = f * Sk[e];
  }
}

/* SRC_F/fftw_ScaRL.f90:157-255 (gen_std_gauss_Shino_FFT): place the
 * half-spectrum in the four (+,+/-,+/-) quadrants of the padded grid, inverse
 * c2c, keep the real part over Np.  The quadrant sizes use the full first
 * axis of Sk (:204 halves it, leaving :218-232 non-conforming).
 * via_c2c = 1 uses the full complex transform; 0 the equivalent C2R with H =
 * Sk/2 on kx >= 1 (the kx = 0 plane is zero). */
void so_gen_std_gauss_shino_fft(double* out, const int Np[3], const double xRange[3],
                                const double corrL[3], int32_t seed, int via_c2c) {
  int sz_c[3], sz[3];
  double dk[3];
  so_shino_sizes(Np, xRange, corrL, sz_c, sz, dk);
  const int n1 = sz[0], n2 = 2 * sz[1], n3 = 2 * sz[2];
  zc* Sk = (zc*)malloc(sizeof(zc) * (int64_t)n1 * n2 * n3);
  so_build_sk_mtx(seed, sz, dk, (double*)Sk);
  if (via_c2c) {
    const int64_t N = (int64_t)sz_c[0] * sz_c[1] * sz_c[2];
    zc* c = (zc*)calloc(N, sizeof(zc));
    for (int k = 0; k < n3; ++k)
      for (int j = 0; j < n2; ++j)
        for (int i = 0; i < n1; ++i) {
          int cj = j < sz[1] ? j : sz_c[1] - n2 + j;
          int ck = k < sz[2] ? k : sz_c[2] - n3 + k;
          c[i + (int64_t)sz_c[0] * (cj + (int64_t)sz_c[1] * ck)] = Sk[i + (int64_t)n1 * (j + (int64_t)n2 * k)];
        }
    so_c2c_3d((double*)c, sz_c, +1);
    for (int k = 0; k < Np[2]; ++k)
      for (int j = 0; j < Np[1]; ++j)
        for (int i = 0; i < Np[0]; ++i)
          out[i + (int64_t)Np[0] * (j + (int64_t)Np[1] * k)] = creal(c[i + (int64_t)sz_c[0] * (j + (int64_t)sz_c[1] * k)]);
    free(c);
  } else {
    const int Hx = sz_c[0] / 2 + 1;
    zc* H = (zc*)calloc((int64_t)Hx * sz_c[1] * sz_c[2], sizeof(zc));
    for (int k = 0; k < n3; ++k)
      for (int j = 0; j < n2; ++j)
        for (int i = 1; i < n1; ++i) {
          int cj = j < sz[1] ? j : sz_c[1] - n2 + j;
          int ck = k < sz[2] ? k : sz_c[2] - n3 + k;
          H[i + (int64_t)Hx * (cj + (int64_t)sz_c[1] * ck)] = 0.5 * Sk[i + (int64_t)n1 * (j + (int64_t)n2 * k)];
        }
    so_c2r_3d_crop((const double*)H, sz_c, Np, out);
    free(H);
  }
  free(Sk);
}

/* Target spectral densities (cycles per unit length), corrL = integral scale
 * along each axis (the quantity the Stat estimator rebuild_corrL returns):
 *   1 Gaussian:     C(r) = exp(-pi sum (r_d/l_d)^2)
 *   3 exponential:  C(r) = exp(-|r/a|), a = l/2
 *   2 von Karman:   Matern(nu) with a = l Gamma(nu) / (2 sqrt(pi) Gamma(nu+1/2)) */
/* The model constants of so_spectrum, prepared once per grid; so_spec_eval
 * forms each product in the order so_spectrum always has, so its values are
 * those of so_spectrum bit for bit. */
typedef struct {
  int corrMod;
  double corrL[3], t[3], c, p;
} so_spec;

static void so_spec_prep(so_spec* s, int corrMod, double nu, const double corrL[3]) {
  s->corrMod = corrMod;
  for (int d = 0; d < 3; ++d) s->corrL[d] = corrL[d];
  if (corrMod == 1) return;
  if (corrMod == 3) { nu = 0.5; }
  double sc = tgamma(nu) / (2.0 * sqrt(M_PI) * tgamma(nu + 0.5)), a[3];
  for (int d = 0; d < 3; ++d) { a[d] = corrL[d] * sc; s->t[d] = 4.0 * M_PI * M_PI * a[d] * a[d]; }
  s->c = 8.0 * pow(M_PI, 1.5) * tgamma(nu + 1.5) / tgamma(nu) * a[0] * a[1] * a[2];
  s->p = -(nu + 1.5);
}

static double so_spec_eval(const so_spec* s, const double f[3]) {
  if (s->corrMod == 1) {
    double S = 1.0;
    for (int d = 0; d < 3; ++d)
      S *= s->corrL[d] * exp(-M_PI * s->corrL[d] * s->corrL[d] * f[d] * f[d]);
    return S;
  }
  double q = 0.0;
  for (int d = 0; d < 3; ++d) q += s->t[d] * f[d] * f[d];
  return s->c * pow(1.0 + q, s->p);
}

double so_spectrum(int corrMod, double nu, const double corrL[3], const double f[3]) {
  so_spec s;
  so_spec_prep(&s, corrMod, nu, corrL);
  return so_spec_eval(&s, f);
}

static inline double so_freq(int k, int P, double dx) {
  int s = (2 * k <= P) ? k : k - P;
  return (double)s / ((double)P * dx);
}

/* sum over the full periodic grid of S(k) dk^3 (FP64, deterministic order). */
double so_spectrum_sum(int corrMod, double nu, const int P[3], const double dx[3],
                       const double corrL[3]) {
  const int Hx = P[0] / 2 + 1;
  const double dk3 = (1.0 / (P[0] * dx[0])) * (1.0 / (P[1] * dx[1])) * (1.0 / (P[2] * dx[2]));
  double* part = (double*)calloc(P[2], sizeof(double));
  so_spec sp;
  so_spec_prep(&sp, corrMod, nu, corrL);
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < P[2]; ++kz) {
    double s = 0.0;
    for (int ky = 0; ky < P[1]; ++ky)
      for (int kx = 0; kx < Hx; ++kx) {
        double f[3] = {so_freq(kx, P[0], dx[0]), so_freq(ky, P[1], dx[1]), so_freq(kz, P[2], dx[2])};
        double c = (kx == 0 || 2 * kx == P[0]) ? 1.0 : 2.0;
        s += c * so_spec_eval(&sp, f) * dk3;
      }
    part[kz] = s;
  }
  double t = 0.0;
  for (int kz = 0; kz < P[2]; ++kz) t += part[kz];
  free(part);
  return t;
}

/* Half spectrum of the padded periodic grid (corrected, normalised method):
 *   H(m) = sqrt(S(k_m) dk^3 / norm) g(kx) (xi_re + i xi_im),
 *   g = 1 on the kx = 0 and kx = P0/2 planes, 1/sqrt(2) elsewhere,
 * so that the C2R output has variance sum_m S dk^3 / norm (1 when
 * normalised).  xi: injected pairs, or canonical Philox normals. */
static void so_padded_spectrum_n(int corrMod, double nu, const int P[3], const double dx[3],
                                 const double corrL[3], double norm, uint64_t seed,
                                 uint32_t stream, const double* xi, double* Hd) {
  zc* H = (zc*)Hd;
  const int Hx = P[0] / 2 + 1;
  const int64_t M = (int64_t)Hx * P[1] * P[2];
  const double dk3 = (1.0 / (P[0] * dx[0])) * (1.0 / (P[1] * dx[1])) * (1.0 / (P[2] * dx[2]));
  so_spec sp;
  so_spec_prep(&sp, corrMod, nu, corrL);
  double* own = NULL;
  if (!xi) {
    own = (double*)malloc(sizeof(double) * 2 * M);
    so_normals(seed, stream, P, own);
    xi = own;
  }
#pragma omp parallel for schedule(static)
  for (int kz = 0; kz < P[2]; ++kz)
    for (int ky = 0; ky < P[1]; ++ky)
      for (int kx = 0; kx < Hx; ++kx) {
        int64_t m = kx + (int64_t)Hx * (ky + (int64_t)P[1] * kz);
        double f[3] = {so_freq(kx, P[0], dx[0]), so_freq(ky, P[1], dx[1]), so_freq(kz, P[2], dx[2])};
        double g = (kx == 0 || 2 * kx == P[0]) ? 1.0 : M_SQRT1_2;
        double A = sqrt(so_spec_eval(&sp, f) * dk3 / norm) * g;
        H[m] = A * xi[2 * m] + I * (A * xi[2 * m + 1]);
      }
  free(own);
}

void so_padded_spectrum(int corrMod, double nu, const int P[3], const double dx[3],
                        const double corrL[3], int normalise, uint64_t seed, uint32_t stream,
                        const double* xi, double* Hd) {
  double norm = normalise ? so_spectrum_sum(corrMod, nu, P, dx, corrL) : 1.0;
  so_padded_spectrum_n(corrMod, nu, P, dx, corrL, norm, seed, stream, xi, Hd);
}

/* so_gen_padded with the normalisation sum given (tiles of one sample share
 * their padded grid, so the sum is formed once per sample). */
static void so_gen_padded_n(double* out, const int Np[3], const int P[3], const double dx[3],
                            const double corrL[3], int corrMod, double nu, double norm,
                            uint64_t seed, uint32_t stream, const double* xi) {
  const int Hx = P[0] / 2 + 1;
  double* H = (double*)malloc(sizeof(double) * 2 * (int64_t)Hx * P[1] * P[2]);
  so_padded_spectrum_n(corrMod, nu, P, dx, corrL, norm, seed, stream, xi, H);
  so_c2r_3d_crop(H, P, Np, out);
  free(H);
}

void so_gen_padded(double* out, const int Np[3], const int P[3], const double dx[3],
                   const double corrL[3], int corrMod, double nu, int normalise,
                   uint64_t seed, uint32_t stream, const double* xi) {
  double norm = normalise ? so_spectrum_sum(corrMod, nu, P, dx, corrL) : 1.0;
  so_gen_padded_n(out, Np, P, dx, corrL, corrMod, nu, norm, seed, stream, xi);
}

/* so_gen_padded with the spectrum synthesised inside the z pass (no full
 * half-spectrum array) and the normalisation sum given; line_stride > 1
 * processes every line_stride-th line of each pass only (a timing sample
 * whose output is not a field). */
void so_gen_padded_stream(double* out, const int Np[3], const int P[3], const double dx[3],
                          const double corrL[3], int corrMod, double nu, double norm,
                          uint64_t seed, uint32_t stream, int line_stride) {
  const int Hx = P[0] / 2 + 1;
  const int Nz = Np[2], Ny = Np[1], Nx = Np[0];
  const double dk3 = (1.0 / (P[0] * dx[0])) * (1.0 / (P[1] * dx[1])) * (1.0 / (P[2] * dx[2]));
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const int st = line_stride < 1 ? 1 : line_stride;
  zc* T = (zc*)calloc((size_t)Hx * P[1] * Nz, sizeof(zc));
  so_plan_get(P[0]); so_plan_get(P[1]); so_plan_get(P[2]);
  so_spec sp;
  so_spec_prep(&sp, corrMod, nu, corrL);
  int mx = P[0] > P[1] ? P[0] : P[1];
  if (P[2] > mx) mx = P[2];
#pragma omp parallel
  {
    zc* line = (zc*)malloc(sizeof(zc) * mx);
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)Hx * P[1]; l += st) {
      const int kx = (int)(l % Hx), ky = (int)(l / Hx);
      const int h = P[2] / 2;
      for (int kz0 = 0; kz0 < h; ++kz0) {
        double nv[4];
        so_mode_pair(key, stream, kx, ky, kz0, Hx, P[1], nv);
        for (int half = 0; half < 2; ++half) {
          const int kz = kz0 + half * h;
          double f[3] = {so_freq(kx, P[0], dx[0]), so_freq(ky, P[1], dx[1]), so_freq(kz, P[2], dx[2])};
          double g = (kx == 0 || 2 * kx == P[0]) ? 1.0 : M_SQRT1_2;
          double A = sqrt(so_spec_eval(&sp, f) * dk3 / norm) * g;
          line[kz] = A * nv[2 * half] + I * (A * nv[2 * half + 1]);
        }
      }
      so_fft_sign(line, P[2], +1);
      for (int z = 0; z < Nz; ++z) T[kx + (int64_t)Hx * (ky + (int64_t)P[1] * z)] = line[z];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)Hx * Nz; l += st) {
      const int kx = (int)(l % Hx), z = (int)(l / Hx);
      for (int ky = 0; ky < P[1]; ++ky) line[ky] = T[kx + (int64_t)Hx * (ky + (int64_t)P[1] * z)];
      so_fft_sign(line, P[1], +1);
      for (int y = 0; y < Ny; ++y) T[kx + (int64_t)Hx * (y + (int64_t)P[1] * z)] = line[y];
    }
#pragma omp for schedule(static)
    for (int64_t l = 0; l < (int64_t)Ny * Nz; l += st) {
      const int y = (int)(l % Ny), z = (int)(l / Ny);
      const zc* X = T + (int64_t)Hx * (y + (int64_t)P[1] * z);
      for (int k = 0; k < P[0]; ++k) {
        if (k == 0) line[k] = creal(X[0]);
        else if (2 * k == P[0]) line[k] = creal(X[k]);
        else if (k < Hx) line[k] = X[k];
        else line[k] = conj(X[P[0] - k]);
      }
      so_fft_sign(line, P[0], +1);
      for (int x = 0; x < Nx; ++x) out[x + (int64_t)Nx * (y + (int64_t)Ny * z)] = creal(line[x]);
    }
    free(line);
  }
  free(T);
}

static int so_pow2_pad(int n) {
  int p = 1;
  while (p < 2 * n) p <<= 1;
  return p;
}

/* One deck sample through the localization method (SRC_F/main_ScaRL.f90:
 * 95-185 layout, create_fields :455-576): per simulated rank generate the
 * tile, apply sqrt(PoU), add overlaps, optionally normalize (disabled in the
 * reference), transform the marginal, assemble the global block in rank
 * order.  generator: 1 = gen_std_gauss_FFT (DCT-III), 2 = Shino padded c2c
 * (Park-Miller phases), 3 = corrected padded method (Philox normals).
 * Returns 0, the verify_inputs rule number (1..8) or -1 (topology). */
int so_generate_sample(int generator, const double xMin[3], const double xMax[3],
                       const double corrL[3], const double overlap[3], const int ppcl[3],
                       int corrMod, double nu, int margiFirst, double avg, double std_dev,
                       int seedBase, int nb_procs, const int* topo_in, const int* pad,
                       int normalise_spectrum, int normalize_field, const double* phiK_all,
                       double* global) {
  int rc = so_verify_inputs(xMin, xMax, corrL, overlap, avg, std_dev, corrMod, margiFirst, ppcl, 1);
  if (rc) return rc;
  int L[3], Np[3], No[3], topo[3];
  double xStep[3];
  if (so_sample_layout(xMin, xMax, corrL, overlap, ppcl, 1, nb_procs, topo_in, L, Np, No, topo, xStep))
    return -1;
  const int64_t NG = (int64_t)L[0] * L[1] * L[2];
  if (std_dev == 0.0) { /* write_constant_field, SRC_F/main_ScaRL.f90:145-155 */
    for (int64_t i = 0; i < NG; ++i) global[i] = avg;
    return 0;
  }
  const int nb = topo[0] * topo[1] * topo[2];
  const int64_t n = (int64_t)Np[0] * Np[1] * Np[2];
  double** RF = (double**)malloc(sizeof(double*) * nb);
  int Ppad[3];
  for (int d = 0; d < 3; ++d) Ppad[d] = pad ? pad[d] : so_pow2_pad(Np[d]);
  const double norm = (generator == 3 && normalise_spectrum)
                          ? so_spectrum_sum(corrMod, nu, Ppad, xStep, corrL) : 1.0;
  for (int r = 0; r < nb; ++r) {
    RF[r] = (double*)malloc(sizeof(double) * n);
    int pos[3], p0[3], pN[3];
    double c0[3], cN[3], xr[3];
    so_get_topo_pos(r, topo, pos);
    so_tile_geometry(Np, No, pos, xStep, xMin, p0, pN, c0, cN, xr);
    int seedStart = seedBase + 1 + r;
    if (generator == 1) {
      int64_t K = (int64_t)(Np[0] / 2) * (Np[1] / 2) * (Np[2] / 2);
      double* ph = NULL;
      const double* phi;
      if (phiK_all) phi = phiK_all + K * r;
      else { ph = (double*)malloc(sizeof(double) * (K ? K : 1)); so_uniforms((uint64_t)(uint32_t)seedStart, 0, 0, K, ph); phi = ph; }
      so_gen_std_gauss_fft(RF[r], Np, xr, corrL, phi, NULL);
      free(ph);
    } else if (generator == 2) {
      so_gen_std_gauss_shino_fft(RF[r], Np, xr, corrL, seedStart, 0);
    } else {
      so_gen_padded_n(RF[r], Np, Ppad, xStep, corrL, corrMod, nu, norm,
                      (uint64_t)(uint32_t)seedStart, 0, NULL);
    }
    so_apply_unity_partition(Np, No, 1, pos, topo, RF[r]);
  }
  so_add_overlap(RF, Np, No, topo);
  if (normalize_field) so_normalize_field(RF, Np, No, topo, NULL, NULL);
  for (int r = 0; r < nb; ++r) so_multivariate_transformation(avg, std_dev, margiFirst, RF[r], n);
  so_assemble_global(RF, Np, No, topo, L, global);
  for (int r = 0; r < nb; ++r) free(RF[r]);
  free(RF);
  return 0;
}

/* ======================================================================== */
/* Estimators (Stat_ScaRL)                                                  */
/* ======================================================================== */

/* SRC_F/Stat_ScaRL/statistics_RF.f90:18-174 (calculate_average_and_stdVar_MPI)
 * for one process: f is (xN, nmc) column-major. */
void so_moments(const double* f, int64_t xN, int nmc, double* evntAvg, double* evntStd,
                double* gAvg, double* gStd) {
  double S = 0.0, S2 = 0.0;
  for (int e = 0; e < nmc; ++e) {
    double s = 0.0, s2 = 0.0;
    for (int64_t i = 0; i < xN; ++i) { double v = f[e * xN + i]; s += v; s2 += v * v; }
    evntAvg[e] = s / (double)xN;
    evntStd[e] = sqrt(s2 / (double)xN - evntAvg[e] * evntAvg[e]);
    S += s; S2 += s2;
  }
  *gAvg = S / (double)(xN * nmc);
  *gStd = sqrt(S2 / (double)(xN * nmc) - (*gAvg) * (*gAvg));
}

/* SRC_F/Stat_ScaRL/statistics_RF.f90:277,325-351 (Tukey windows).  literal = 1
 * restates the reference: r_tukey is the single-precision literal 0.1 and the
 * high-side taper formula covers every ratio > r_tukey.  literal = 0 is the
 * standard Tukey window with taper fraction r_tukey (flat middle). */
void so_tukey(int n, int literal, double* w) {
  const double r = (double)0.1f;
  for (int i = 0; i < n; ++i) {
    double ratio = (double)i / (double)(n - 1);
    w[i] = 1.0;
    if (literal) {
      if (ratio < r) w[i] = 1.0 / 2.0 * (1 + cos(2.0 * SO_PI_REF / r * (ratio - r / 2.0)));
      else if (ratio > r) w[i] = 1.0 / 2.0 * (1 + cos(2.0 * SO_PI_REF / r * (ratio - 1.0 + r / 2.0)));
    } else {
      if (ratio < r / 2.0) w[i] = 1.0 / 2.0 * (1 + cos(2.0 * M_PI / r * (ratio - r / 2.0)));
      else if (ratio > 1.0 - r / 2.0) w[i] = 1.0 / 2.0 * (1 + cos(2.0 * M_PI / r * (ratio - 1.0 + r / 2.0)));
    }
  }
}

/* SRC_F/Stat_ScaRL/statistics_RF.f90:258-462 (rebuild_Sk_FFT, nDim = 3):
 * standardise, window along dir, forward FFT per line, /L(dir), |.|^2,
 * mean over the other two axes in the reference's order, backward FFT,
 * real part.  Sk has L[dir] entries. */
void so_rebuild_sk_fft(const double* f, const int L[3], int dir, double avg, double stdDev,
                       int tukey_literal, double* Sk) {
  const int n = L[dir];
  const int64_t N = (int64_t)L[0] * L[1] * L[2];
  double* P2 = (double*)malloc(sizeof(double) * N); /* |X/n|^2 */
  double* w = (double*)malloc(sizeof(double) * n);
  so_tukey(n, tukey_literal, w);
  int o1 = dir == 0 ? L[1] : L[0];
  int o2 = dir == 2 ? L[1] : L[2];
  int64_t s1 = dir == 0 ? L[0] : 1;
  int64_t s2 = dir == 2 ? L[0] : (int64_t)L[0] * L[1];
  int64_t st = dir == 0 ? 1 : (dir == 1 ? L[0] : (int64_t)L[0] * L[1]);
  so_plan_get(n);
#pragma omp parallel
  {
    zc* line = (zc*)malloc(sizeof(zc) * n);
#pragma omp for collapse(2) schedule(static)
    for (int b = 0; b < o2; ++b)
      for (int a = 0; a < o1; ++a) {
        int64_t base = a * s1 + b * s2;
        for (int t = 0; t < n; ++t) line[t] = ((f[base + t * st] - avg) / stdDev) * w[t];
        so_fft_sign(line, n, -1);
        for (int t = 0; t < n; ++t) {
          zc v = line[t] / (double)n;
          P2[base + t * st] = creal(v * conj(v));
        }
      }
    free(line);
  }
  zc* acc = (zc*)calloc(n, sizeof(zc));
  if (dir == 0) {
    for (int i = 0; i < L[0]; ++i) {
      double outer = 0.0;
      for (int k = 0; k < L[2]; ++k) {
        double s = 0.0;
        for (int j = 0; j < L[1]; ++j) s += P2[i + (int64_t)L[0] * (j + (int64_t)L[1] * k)];
        outer += s / L[1];
      }
      acc[i] = outer / L[2];
    }
  } else if (dir == 1) {
    for (int j = 0; j < L[1]; ++j) {
      double outer = 0.0;
      for (int k = 0; k < L[2]; ++k) {
        double s = 0.0;
        for (int i = 0; i < L[0]; ++i) s += P2[i + (int64_t)L[0] * (j + (int64_t)L[1] * k)];
        outer += s / L[0];
      }
      acc[j] = outer / L[2];
    }
  } else {
    for (int k = 0; k < L[2]; ++k) {
      double outer = 0.0;
      for (int j = 0; j < L[1]; ++j) {
        double s = 0.0;
        for (int i = 0; i < L[0]; ++i) s += P2[i + (int64_t)L[0] * (j + (int64_t)L[1] * k)];
        outer += s / L[0];
      }
      acc[k] = outer / L[1];
    }
  }
  so_fft_sign(acc, n, +1);
  for (int t = 0; t < n; ++t) Sk[t] = creal(acc[t]);
  free(acc); free(P2); free(w);
}

/* SRC_F/Stat_ScaRL/statistics_RF.f90:468-486 (rebuild_corrL) over the kept
 * half of each direction (rebuild_Sk :207-222 keeps floor(L/2) lags). */
void so_rebuild_corrL(const double* SkTot, const int nkeep[3], const double xStep[3],
                      double corrL_out[3]) {
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int t = 0; t < nkeep[d]; ++t) s += SkTot[off + t];
    corrL_out[d] = 2.0 * (s - ((SkTot[off] + SkTot[off + nkeep[d] - 1]) / 2.0)) * xStep[d];
    off += nkeep[d];
  }
}

/* Direct restatement of the linear axis covariance: for each axis d and lag
 * h, the mean over all point pairs (x, x + h e_d) of (f - mu)(f' - mu), mu
 * the mean over all points.  Test infrastructure for scarl_axis_cov. */
void so_axis_cov(const double* f, const int L[3], int maxlag, double* mean, double* cov) {
  const int64_t n = (int64_t)L[0] * L[1] * L[2];
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += f[i];
  const double mu = s / (double)n;
  *mean = mu;
  const int64_t st[3] = {1, L[0], (int64_t)L[0] * L[1]};
  for (int d = 0; d < 3; ++d) {
#pragma omp parallel for schedule(dynamic)
    for (int h = 0; h <= maxlag; ++h) {
      double acc = 0.0;
      int64_t pairs = 0;
      for (int z = 0; z < L[2]; ++z)
        for (int y = 0; y < L[1]; ++y)
          for (int x = 0; x < L[0]; ++x) {
            const int c[3] = {x, y, z};
            if (c[d] + h >= L[d]) continue;
            const int64_t i = x + (int64_t)L[0] * (y + (int64_t)L[1] * z);
            acc += (f[i] - mu) * (f[i + (int64_t)h * st[d]] - mu);
            ++pairs;
          }
      cov[d * (maxlag + 1) + h] = acc / (double)pairs;
    }
  }
}
