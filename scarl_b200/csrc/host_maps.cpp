// host_maps.cpp -- host-side logic of the ScaRL driver: input validation,
// index maps, topology, tile geometry, partition-of-unity weights, the
// Shino spectrum sizes and the plain-text deck readers.  Pure C++ on the
// CPU; every routine restates the reference routine it cites so the maps
// come out bit-identical.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/scarl.h"
#include "host_maps.h"

namespace scarl {

constexpr double kPiRefH = 3.1415926535898;  // SRC_F/constants_ScaRL.f90:5

static void set_msg(char* msg, size_t len, const char* text) {
  if (msg && len) {
    std::snprintf(msg, len, "%s", text);
  }
}

// SRC_F/main_ScaRL.f90:286-333.  Exponential (3) and von Karman (2) are
// accepted: they are the new spectra of the padded generator.
int verify_inputs(const scarl_sample* s, int gen_meth, char* msg, size_t len) {
  for (int d = 0; d < 3; ++d)
    if (s->xMinGlob[d] >= s->xMaxGlob[d]) { set_msg(msg, len, "ERROR: xMinGlob >= xMaxGlob"); return SCARL_EINVAL; }
  for (int d = 0; d < 3; ++d)
    if (s->corrL[d] < 0.0) { set_msg(msg, len, "ERROR: corrL < 0d0"); return SCARL_EINVAL; }
  if (s->corrMod != SCARL_CM_GAUSSIAN && s->corrMod != SCARL_CM_VON_KARMAN &&
      s->corrMod != SCARL_CM_EXPONENTIAL) {
    set_msg(msg, len, "ERROR: Correlation model not implemented");
    return SCARL_EINVAL;
  }
  if (s->margiFirst != SCARL_FOM_GAUSSIAN && s->margiFirst != SCARL_FOM_LOGNORMAL) {
    set_msg(msg, len, "ERROR: First-order marginal not implemented");
    return SCARL_EINVAL;
  }
  if (gen_meth != SCARL_FFT && gen_meth != SCARL_FFT_MPI) {
    set_msg(msg, len, "ERROR: Generation Method  not implemented");
    return SCARL_EINVAL;
  }
  if (s->avg <= 0.0 && s->margiFirst == SCARL_FOM_LOGNORMAL) {
    set_msg(msg, len, "ERROR: When using lognormal first-order marginal density the average should be greater than 0");
    return SCARL_EINVAL;
  }
  if (s->std_dev < 0.0) {
    set_msg(msg, len, "ERROR: Standard deviation should not be smaller than 0d0");
    return SCARL_EINVAL;
  }
  for (int d = 0; d < 3; ++d)
    if (s->pointsPerCorrL[d] < 2) { set_msg(msg, len, "ERROR: PointsPerCorrL < 2"); return SCARL_EINVAL; }
  if (s->corrMod == SCARL_CM_VON_KARMAN && !(s->nu > 0.0)) {
    set_msg(msg, len, "ERROR: von Karman order nu must be > 0");
    return SCARL_EINVAL;
  }
  set_msg(msg, len, "");
  return SCARL_OK;
}

// SRC_F/main_ScaRL.f90:959-978.
static void find_factors(int n, int d[100]) {
  for (int i = 0; i < 100; ++i) d[i] = 0;
  int i = 0, div = 2, next = 3, rest = n;
  while (rest > 1) {
    while (rest % div == 0) { d[i++] = div; rest /= div; }
    div = next;
    next += 2;
  }
}

static int first_maxloc(const int v[3]) {
  int p = 0;
  for (int d = 1; d < 3; ++d)
    if (v[d] > v[p]) p = d;
  return p;
}

// SRC_F/main_ScaRL.f90:834-893.  The reference leaves vol_surf_factor
// uninitialised; it starts at zero here.
void decide_topo_shape(int nb_procs, const int L[3], const int ovlp[3], long long ppbi,
                       int topo[3]) {
  int nBlocks[3] = {1, 1, 1}, nPerProc[3];
  for (;;) {
    long long tot = 1;
    for (int d = 0; d < 3; ++d) {
      const int nPoints = L[d] + (nBlocks[d] - 1) * ovlp[d];
      nPerProc[d] = (int)std::ceil((double)nPoints / (double)nBlocks[d]);
      tot *= (long long)nPerProc[d];
    }
    if (tot <= ppbi) break;
    if (nBlocks[0] * nBlocks[1] * nBlocks[2] >= nb_procs) break;
    nBlocks[first_maxloc(nPerProc)] += 1;
  }
  const int ideal[3] = {nBlocks[0], nBlocks[1], nBlocks[2]};
  const int np_start = (int)std::ceil(0.75f * (float)nb_procs);
  double best = 0.0;
  int chosen[3] = {1, 1, 1};
  for (int np = np_start; np <= nb_procs; ++np) {
    int f[100], nb[3] = {ideal[0], ideal[1], ideal[2]}, nf[3] = {1, 1, 1};
    find_factors(np, f);
    for (int i = 99; i >= 0; --i) {
      if (f[i] == 0) continue;
      if (nb[0] == 1 && nb[1] == 1 && nb[2] == 1) break;
      const int pos = first_maxloc(nb);
      nf[pos] *= f[i];
      nb[pos] = (int)std::ceil((double)nb[pos] / (double)f[i]);
    }
    const double v = (double)(nf[0] * nf[1] * nf[2]) /
                     (double)(2 * (nf[0] * nf[1] + nf[1] * nf[2] + nf[2] * nf[0]));
    if (v >= best) {
      best = v;
      chosen[0] = nf[0]; chosen[1] = nf[1]; chosen[2] = nf[2];
    }
  }
  topo[0] = chosen[0]; topo[1] = chosen[1]; topo[2] = chosen[2];
}

void get_topo_pos(int rank, const int shape[3], int pos[3]) {
  int rest = rank;
  pos[2] = rest / (shape[0] * shape[1]);
  rest -= pos[2] * shape[0] * shape[1];
  pos[1] = rest / shape[0];
  rest -= pos[1] * shape[0];
  pos[0] = rest;
}

int get_topo_rank(const int shape[3], const int pos[3]) {
  return shape[0] * shape[1] * pos[2] + shape[0] * pos[1] + pos[0];
}

// SRC_F/main_ScaRL.f90:100-111, 119-127 and 157-176.
int sample_layout(const scarl_sample* s, int gen_meth, int nb_procs, const int* topo_in,
                  scarl_layout* o) {
  if (nb_procs < 1) return SCARL_EINVAL;
  for (int d = 0; d < 3; ++d) {
    if (s->pointsPerCorrL[d] < 2) return SCARL_EINVAL;
    o->xStep[d] = s->corrL[d] / ((double)(s->pointsPerCorrL[d] - 1));
    const double span = std::ceil((s->xMaxGlob[d] - s->xMinGlob[d]) / o->xStep[d]);
    if (!(span >= 0.0) || span > 1.0e9) return SCARL_EINVAL;
    o->L[d] = 1 + (int)span;
    o->Np_ovlp[d] = (gen_meth == SCARL_FFT_MPI)
                        ? 0
                        : 1 + (int)std::ceil(s->overlap[d] * (double)(s->pointsPerCorrL[d] - 1));
  }
  if (topo_in) {
    if (topo_in[0] < 1 || topo_in[1] < 1 || topo_in[2] < 1) return SCARL_EINVAL;
    if (topo_in[0] * topo_in[1] * topo_in[2] != nb_procs) return SCARL_EINVAL;
    for (int d = 0; d < 3; ++d) o->topo_shape[d] = topo_in[d];
  } else if (gen_meth == SCARL_FFT_MPI) {
    // FFTW-MPI's default slab distribution of the last axis (block ceil(L3/np)).
    const int blk = (o->L[2] + nb_procs - 1) / nb_procs;
    o->topo_shape[0] = 1;
    o->topo_shape[1] = 1;
    o->topo_shape[2] = (o->L[2] + blk - 1) / blk;
  } else {
    decide_topo_shape(nb_procs, o->L, o->Np_ovlp, 1, o->topo_shape);
  }
  for (int d = 0; d < 3; ++d) {
    const int T = o->topo_shape[d];
    int Np = (int)std::ceil((double)(o->L[d] + (T - 1) * o->Np_ovlp[d]) / (double)T);
    if (T == 2 && Np < o->Np_ovlp[d]) Np = o->Np_ovlp[d];
    if (T >= 3 && Np < 2 * o->Np_ovlp[d]) Np = 2 * o->Np_ovlp[d];
    o->Np[d] = Np;
    o->L[d] = Np * T - (T - 1) * o->Np_ovlp[d];
  }
  o->nb_tiles = o->topo_shape[0] * o->topo_shape[1] * o->topo_shape[2];
  return SCARL_OK;
}

// SRC_F/main_ScaRL.f90:455-459.
void tile_geometry(const scarl_layout* lay, const double xMin[3], int rank, scarl_tile* t) {
  get_topo_pos(rank, lay->topo_shape, t->topo_pos);
  for (int d = 0; d < 3; ++d) {
    t->pos_0[d] = (lay->Np[d] - lay->Np_ovlp[d]) * t->topo_pos[d] + 1;
    t->pos_N[d] = t->pos_0[d] + lay->Np[d] - 1;
    t->coord_0[d] = (double)(t->pos_0[d] - 1) * lay->xStep[d] + xMin[d];
    t->coord_N[d] = (double)(t->pos_N[d] - 1) * lay->xStep[d] + xMin[d];
    t->xRange[d] = t->coord_N[d] - t->coord_0[d];
  }
}

// One side's partition-of-unity pattern along one axis
// (SRC_F/main_ScaRL.f90:1257-1270): empty when the side does not apply.
std::vector<double> pou_pattern(int Np_ovlp, int side, int topo_pos, int topo_shape,
                                int partitionType) {
  std::vector<double> p;
  const int shift = side == 0 ? -1 : 1;
  if (Np_ovlp < 2) return p;
  if (topo_pos + shift < 0 || topo_pos + shift > topo_shape - 1) return p;
  p.resize(Np_ovlp);
  for (int k = 0; k < Np_ovlp; ++k) p[k] = (double)k / (double)(Np_ovlp - 1);
  if (side == 0) std::reverse(p.begin(), p.end());
  if (partitionType == 1)
    for (int k = 0; k < Np_ovlp; ++k) p[k] = (1.0 + std::cos(kPiRefH * p[k])) / 2.0;
  return p;
}

// Per-axis factor tables: lo[x] / hi[x] carry the pattern on the planes it
// covers and 1.0 elsewhere, so the product lo_x lo_y lo_z hi_x hi_y hi_z
// multiplies exactly the factors the reference multiplies, in its order.
void pou_axis_tables(int Np, int Np_ovlp, int topo_pos, int topo_shape, int partitionType,
                     double* lo, double* hi) {
  for (int x = 0; x < Np; ++x) { lo[x] = 1.0; hi[x] = 1.0; }
  std::vector<double> pl = pou_pattern(Np_ovlp, 0, topo_pos, topo_shape, partitionType);
  for (size_t t = 0; t < pl.size(); ++t) lo[t] = pl[t];
  std::vector<double> ph = pou_pattern(Np_ovlp, 1, topo_pos, topo_shape, partitionType);
  for (size_t t = 0; t < ph.size(); ++t) hi[Np - Np_ovlp + (int)t] = ph[t];
}

// Blend roles along one axis.  A point shared with the previous / next tile
// is summed only when the overlap is wider than one point (add_overlap skips
// degenerate regions, :1133,:1168); a one-point overlap keeps the value of the
// higher-ranked tile, which the one-dataset writer stores last
// (SRC_F/write_output.f90:412-427).
void blend_axis_flags(int Np, int Np_ovlp, int topo_pos, int topo_shape, uint8_t* flags) {
  for (int x = 0; x < Np; ++x) {
    const bool has_prev = topo_pos > 0 && x < Np_ovlp;
    const bool has_next = topo_pos < topo_shape - 1 && x >= Np - Np_ovlp;
    const bool summed = Np_ovlp >= 2;
    bool participate = true, first = true, last = true;
    if (has_next) {
      if (summed) last = false;
      else participate = false;
    }
    if (has_prev && summed) first = false;
    flags[x] = (uint8_t)((participate ? 1 : 0) | (first ? 2 : 0) | (last ? 4 : 0));
  }
}

// SRC_F/main_ScaRL.f90:1236-1294: full weight array, reference order.
void unity_partition_weights(const int Np[3], const int No[3], int partitionType,
                             const int pos[3], const int shape[3], double* w) {
  const size_t n = (size_t)Np[0] * Np[1] * Np[2];
  for (size_t i = 0; i < n; ++i) w[i] = 1.0;
  for (int side = 0; side < 2; ++side)
    for (int ax = 0; ax < 3; ++ax) {
      std::vector<double> p = pou_pattern(No[ax], side, pos[ax], shape[ax], partitionType);
      if (p.empty()) continue;
      const int D = side == 0 ? 0 : Np[ax] - No[ax];
      for (int k = 0; k < Np[2]; ++k)
        for (int j = 0; j < Np[1]; ++j)
          for (int i = 0; i < Np[0]; ++i) {
            const int c = ax == 0 ? i : (ax == 1 ? j : k);
            if (c < D || c >= D + No[ax]) continue;
            w[i + (size_t)Np[0] * (j + (size_t)Np[1] * k)] *= p[c - D];
          }
    }
}

// SRC_F/fftw_ScaRL.f90:193-194 and SRC_F/spectra_ScaRL.f90:44-56.
int shino_sizes(const int Np[3], const double xRange[3], const double corrL[3], int sz_c[3],
                int sz_Sk[3], double delta_k[3]) {
  int clamped = 0;
  for (int d = 0; d < 3; ++d) {
    const double xr = xRange[d] / corrL[d];
    sz_c[d] = 1 << (int)std::ceil(std::log((double)(2 * Np[d])) / std::log(2.0));
    const double delta_x = xr / (double)(Np[d] - 1);
    const double k_max = 1.0 / delta_x;
    delta_k[d] = k_max / (double)(sz_c[d] / 2);
    double k_cut = 7.355;
    if (k_max < k_cut) { k_cut = k_max; clamped = 1; }
    sz_Sk[d] = (int)std::ceil(k_cut / delta_k[d]);
    if (sz_Sk[d] > sz_c[d] / 2) sz_Sk[d] = sz_c[d] / 2;
  }
  return clamped;
}

// ---------------------------------------------------------------------------
// Padded grid sizes
// ---------------------------------------------------------------------------
// K_nu(x) from K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt (trapezoid;
// the integrand is smooth and decays doubly exponentially).
static double bessel_k(double nu, double x) {
  const double h = 1.0 / 64.0;
  double s = 0.5 * std::exp(-x);
  for (int i = 1; i < 64 * 40; ++i) {
    const double t = i * h;
    const double e = x * std::cosh(t);
    if (e > 745.0) break;
    s += std::exp(-e) * std::cosh(nu * t);
  }
  return s * h;
}

// Unit-variance correlation at lag r along an axis with integral scale l.
double axis_correlation(int corrMod, double nu, double l, double r) {
  if (r <= 0.0) return 1.0;
  if (corrMod == SCARL_CM_GAUSSIAN) return std::exp(-M_PI * r * r / (l * l));
  if (corrMod == SCARL_CM_EXPONENTIAL) return std::exp(-2.0 * r / l);
  const double a = l * std::tgamma(nu) / (2.0 * std::sqrt(M_PI) * std::tgamma(nu + 0.5));
  const double x = r / a;
  if (x > 700.0) return 0.0;
  return std::pow(2.0, 1.0 - nu) / std::tgamma(nu) * std::pow(x, nu) * bessel_k(nu, x);
}

bool fft_length_supported(int n) {
  if (n < 8 || n > 2048) return false;
  int m = n;
  while (m % 2 == 0) m /= 2;
  if (m == 1) return true;
  return (m == 3 || m == 5 || m == 7) && n / m >= 16;
}

// Smallest supported length >= n (power of two, or m 2^a with m = 3, 5, 7 and
// 2^a >= 16); 0 above 2048.
static int next_smooth(int n) {
  for (int p = std::max(n, 8); p <= 2048; ++p)
    if (fft_length_supported(p)) return p;
  return 0;
}

// policy 0: the reference's 2^ceil(log2(2 Np)) (SRC_F/fftw_ScaRL.f90:194).
// policy 1: smallest power of two P >= 8 with C((P - Np + 1) dx) <= tol along
// each axis: the nearest periodic image of the farthest pair of tile points
// then contributes at most tol to the covariance.
// policy 3: the same rule over every supported length (powers of two and
// 3, 5, 7 times a power of two >= 16, up to 2048).
int pad_size(int policy, int corrMod, double nu, const double corrL[3], const double xStep[3],
             const int Np[3], double tol, int P[3]) {
  for (int d = 0; d < 3; ++d) {
    if (Np[d] < 1) return SCARL_EINVAL;
    int p = 8;
    if (policy == 0) {
      while (p < 2 * Np[d]) p <<= 1;
    } else if (policy == 1) {
      if (!(tol > 0.0 && tol < 1.0) || !(corrL[d] > 0.0) || !(xStep[d] > 0.0)) return SCARL_EINVAL;
      while (p < Np[d] || axis_correlation(corrMod, nu, corrL[d], (p - Np[d] + 1) * xStep[d]) > tol) {
        p <<= 1;
        if (p > (1 << 24)) return SCARL_EINVAL;
      }
    } else if (policy == 3) {
      if (!(tol > 0.0 && tol < 1.0) || !(corrL[d] > 0.0) || !(xStep[d] > 0.0)) return SCARL_EINVAL;
      p = next_smooth(Np[d]);
      while (p && axis_correlation(corrMod, nu, corrL[d], (p - Np[d] + 1) * xStep[d]) > tol)
        p = next_smooth(p + 1);
      if (!p) return SCARL_EINVAL;  // beyond the largest supported length
    } else {
      return SCARL_EINVAL;
    }
    P[d] = p;
  }
  return SCARL_OK;
}

// ---------------------------------------------------------------------------
// Plain-text decks: getLine (SRC_F/read_input.f90:565-585) plus Fortran
// list-directed reads of the returned record.
// ---------------------------------------------------------------------------
class Deck {
 public:
  explicit Deck(const char* path) : in_(path) {}
  bool ok() const { return (bool)in_; }
  // Next record whose first non-blank character is not '#'; "eof_gl" at EOF.
  std::string line() {
    std::string s;
    for (int i = 0; i < 200; ++i) {
      if (!std::getline(in_, s)) return "eof_gl";
      if (!s.empty() && s.back() == '\r') s.pop_back();
      size_t p = s.find_first_not_of(" \t");
      s = (p == std::string::npos) ? std::string() : s.substr(p);
      if (s.empty() || s[0] != '#') return s;
    }
    return s;
  }
  void rewind() { in_.clear(); in_.seekg(0); }

 private:
  std::ifstream in_;
};

// Split a record into list-directed items: blanks/commas separate, '/' ends
// the record, quoted strings keep their content, r*value repeats.
static std::vector<std::string> items(const std::string& rec) {
  std::vector<std::string> out;
  size_t i = 0, n = rec.size();
  while (i < n) {
    while (i < n && (rec[i] == ' ' || rec[i] == '\t' || rec[i] == ',')) ++i;
    if (i >= n || rec[i] == '/') break;
    std::string tok;
    if (rec[i] == '"' || rec[i] == '\'') {
      const char q = rec[i++];
      while (i < n) {
        if (rec[i] == q) {
          if (i + 1 < n && rec[i + 1] == q) { tok += q; i += 2; continue; }
          ++i;
          break;
        }
        tok += rec[i++];
      }
      out.push_back(tok);
      continue;
    }
    while (i < n && rec[i] != ' ' && rec[i] != '\t' && rec[i] != ',' && rec[i] != '/') tok += rec[i++];
    const size_t star = tok.find('*');
    if (star != std::string::npos && star > 0 &&
        std::all_of(tok.begin(), tok.begin() + star, [](char c) { return std::isdigit((unsigned char)c); })) {
      const int r = std::atoi(tok.substr(0, star).c_str());
      const std::string v = tok.substr(star + 1);
      for (int k = 0; k < r; ++k) out.push_back(v);
    } else {
      out.push_back(tok);
    }
  }
  return out;
}

static bool to_double(const std::string& t, double* v) {
  std::string s = t;
  for (char& c : s)
    if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
  if (s.empty()) return false;
  char* end = nullptr;
  *v = std::strtod(s.c_str(), &end);
  return end && *end == '\0';
}

static bool to_int(const std::string& t, int* v) {
  if (t.empty()) return false;
  char* end = nullptr;
  const long r = std::strtol(t.c_str(), &end, 10);
  if (!end || *end != '\0') return false;
  *v = (int)r;
  return true;
}

static bool read_ints(Deck& dk, int* v, int n) {
  std::vector<std::string> it = items(dk.line());
  if ((int)it.size() < n) return false;
  for (int i = 0; i < n; ++i)
    if (!to_int(it[i], v + i)) return false;
  return true;
}

static bool read_doubles(Deck& dk, double* v, int n) {
  std::vector<std::string> it = items(dk.line());
  if ((int)it.size() < n) return false;
  for (int i = 0; i < n; ++i)
    if (!to_double(it[i], v + i)) return false;
  return true;
}

static bool read_string(Deck& dk, std::string* v) {
  std::vector<std::string> it = items(dk.line());
  if (it.empty()) return false;
  *v = it[0];
  return true;
}

static void copy_str(char* dst, size_t len, const std::string& s) {
  if (dst && len) std::snprintf(dst, len, "%s", s.c_str());
}

int read_config(const char* path, int* gen_meth, int* c_info, int* d_sample, int* one_file,
                int* one_hdf_ds, char* input_file, size_t len) {
  Deck dk(path);
  if (!dk.ok()) {  // defaults, SRC_F/read_input.f90:74-83
    *gen_meth = 1; *c_info = 0; *d_sample = 0; *one_file = 1; *one_hdf_ds = 1;
    copy_str(input_file, len, "./input_ScaRL.txt");
    return SCARL_OK;
  }
  int v;
  if (!read_ints(dk, gen_meth, 1)) return SCARL_EIO;
  if (!read_ints(dk, &v, 1)) return SCARL_EIO;
  *c_info = v == 1;
  if (!read_ints(dk, &v, 1)) return SCARL_EIO;
  *d_sample = v == 1;
  if (!read_ints(dk, &v, 1)) return SCARL_EIO;
  *one_file = v == 1;
  if (!read_ints(dk, &v, 1)) return SCARL_EIO;
  *one_hdf_ds = v == 1;
  std::string f;
  if (!read_string(dk, &f)) return SCARL_EIO;
  copy_str(input_file, len, f);
  return SCARL_OK;
}

int read_extra_config(const char* path, int* found, int topo[3]) {
  topo[0] = topo[1] = topo[2] = -1;
  *found = 0;
  Deck dk(path);
  if (!dk.ok()) return SCARL_OK;
  *found = 1;
  return read_ints(dk, topo, 3) ? SCARL_OK : SCARL_EIO;
}

int read_input(const char* path, char* folder, size_t flen, int* nSamples, scarl_sample* out,
               int max_samples) {
  Deck dk(path);
  if (!dk.ok()) return SCARL_EIO;
  std::string f;
  if (!read_string(dk, &f)) return SCARL_EIO;
  copy_str(folder, flen, f);
  int n;
  if (!read_ints(dk, &n, 1) || n < 0) return SCARL_EIO;
  *nSamples = n;
  if (!out) return SCARL_OK;
  if (n > max_samples) return SCARL_EINVAL;
  for (int s = 0; s < n; ++s) {
    scarl_sample& q = out[s];
    std::memset(&q, 0, sizeof q);
    std::string name;
    if (!read_string(dk, &name)) return SCARL_EIO;
    copy_str(q.name, sizeof q.name, name);
    if (!read_doubles(dk, q.xMinGlob, 3)) return SCARL_EIO;
    if (!read_doubles(dk, q.xMaxGlob, 3)) return SCARL_EIO;
    if (!read_doubles(dk, q.corrL, 3)) return SCARL_EIO;
    if (!read_doubles(dk, q.overlap, 3)) return SCARL_EIO;
    if (!read_ints(dk, q.pointsPerCorrL, 3)) return SCARL_EIO;
    if (!read_ints(dk, &q.corrMod, 1)) return SCARL_EIO;
    if (!read_ints(dk, &q.margiFirst, 1)) return SCARL_EIO;
    if (!read_doubles(dk, &q.avg, 1)) return SCARL_EIO;
    if (!read_doubles(dk, &q.std_dev, 1)) return SCARL_EIO;
    if (!read_ints(dk, &q.seedBase, 1)) return SCARL_EIO;
    q.nu = 0.5;
  }
  return SCARL_OK;
}

// SRC_F/read_input.f90:354-559.
int read_input_sem(const char* folderp, char* out_folder, size_t flen, int* nSamples,
                   scarl_sample* out, int max_samples) {
  const std::string folder = folderp ? folderp : ".";
  Deck dk((folder + "/random.spec").c_str());
  if (!dk.ok()) return SCARL_EIO;
  int nMat;
  if (!read_ints(dk, &nMat, 1) || nMat < 0) return SCARL_EIO;
  std::vector<int> nb_Mat(nMat), nProp(nMat);
  for (int m = 0; m < nMat; ++m) {
    if (!read_ints(dk, &nb_Mat[m], 1)) return SCARL_EIO;
    dk.line();  // VP_VS_RHO flag and values
    if (!read_ints(dk, &nProp[m], 1)) return SCARL_EIO;
    for (int j = 0; j < nProp[m]; ++j) dk.line();
  }
  int total = 0;
  for (int m = 0; m < nMat; ++m) total += nProp[m];
  *nSamples = total;
  if (!out) return SCARL_OK;
  if (total > max_samples) return SCARL_EINVAL;
  struct Prop { int mat; std::string name; double avg; int corrMod; double corrL[3]; int margiF; double CV; int seed; };
  std::vector<Prop> props;
  dk.rewind();
  dk.line();
  for (int m = 0; m < nMat; ++m) {
    dk.line();
    std::vector<std::string> it = items(dk.line());
    int flag = 0;
    double VP = 0, VS = 0, RHO = 0;
    if (it.empty() || !to_int(it[0], &flag)) return SCARL_EIO;
    if (flag == 1) {
      if (it.size() < 4 || !to_double(it[1], &VP) || !to_double(it[2], &VS) || !to_double(it[3], &RHO))
        return SCARL_EIO;
    }
    dk.line();
    for (int j = 0; j < nProp[m]; ++j) {
      std::vector<std::string> p = items(dk.line());
      if (p.size() < 9) return SCARL_EIO;
      Prop q;
      q.mat = nb_Mat[m];
      q.name = p[0];
      if (!to_double(p[1], &q.avg) || !to_int(p[2], &q.corrMod) || !to_double(p[3], &q.corrL[0]) ||
          !to_double(p[4], &q.corrL[1]) || !to_double(p[5], &q.corrL[2]) || !to_int(p[6], &q.margiF) ||
          !to_double(p[7], &q.CV) || !to_int(p[8], &q.seed))
        return SCARL_EIO;
      if (flag == 1) {
        if (q.name == "Lambda") q.avg = 2.0 * RHO * (VS * VS);
        else if (q.name == "Kappa") q.avg = RHO * (VP * VP - 4.0 * (VS * VS) / 3.0);
        else if (q.name == "Mu") q.avg = RHO * (VS * VS);
        else if (q.name == "Density") q.avg = RHO;
      }
      props.push_back(q);
    }
  }
  std::vector<double> bmin(3 * (size_t)nMat, 0.0), bmax(3 * (size_t)nMat, 0.0);
  Deck dm((folder + "/domains.txt").c_str());
  if (!dm.ok()) return SCARL_EIO;
  std::string rec = dm.line();
  while (rec != "eof_gl") {
    std::vector<std::string> it = items(rec);
    int matNb;
    double b[6];
    if (it.size() < 7 || !to_int(it[0], &matNb)) return SCARL_EIO;
    for (int k = 0; k < 6; ++k)
      if (!to_double(it[1 + k], &b[k])) return SCARL_EIO;
    rec = dm.line();
    for (int i = 0; i < nMat; ++i)
      if (nb_Mat[i] == matNb) {
        for (int d = 0; d < 3; ++d) { bmin[3 * i + d] = b[d]; bmax[3 * i + d] = b[3 + d]; }
        break;
      }
  }
  copy_str(out_folder, flen, "./mat/h5");
  size_t pc = 0;
  for (int m = 0; m < nMat; ++m)
    for (int j = 0; j < nProp[m]; ++j, ++pc) {
      const Prop& p = props[pc];
      scarl_sample& q = out[pc];
      std::memset(&q, 0, sizeof q);
      std::string name = "Mat_" + std::to_string(p.mat) + "_" + p.name;
      copy_str(q.name, sizeof q.name, name);
      for (int d = 0; d < 3; ++d) {
        q.xMinGlob[d] = bmin[3 * m + d];
        q.xMaxGlob[d] = bmax[3 * m + d];
        q.corrL[d] = p.corrL[d];
        q.overlap[d] = 5.0;
        q.pointsPerCorrL[d] = 5;
      }
      q.corrMod = p.corrMod;
      q.margiFirst = p.margiF;
      q.avg = p.avg;
      q.std_dev = p.CV * p.avg;
      q.seedBase = p.seed;
      q.nu = 0.5;
    }
  return SCARL_OK;
}

// ---------------------------------------------------------------------------
// Ensemble draws (no counterpart in the reference).  Philox4x32-10 (Salmon et
// al., SC11) on the host: realisation r reads the block at counter
// {r, r >> 32, 0, 2}, key {seed, seed >> 32}.
// ---------------------------------------------------------------------------
static void philox_host(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

int ensemble_draw(uint64_t seed, long long first, int n, const int* choices, int nchoices,
                  double lmin, double lmax, int* Np, double* corrL) {
  if (n < 0 || nchoices < 1 || !choices || !Np || !corrL || first < 0) return SCARL_EINVAL;
  for (int i = 0; i < n; ++i) {
    const uint64_t r = (uint64_t)first + (uint64_t)i;
    const uint32_t ctr[4] = {(uint32_t)r, (uint32_t)(r >> 32), 0u, 2u};
    uint32_t w[4];
    philox_host(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), w);
    for (int d = 0; d < 3; ++d)
      Np[3 * i + d] = choices[(int)(((uint64_t)w[d] * (uint64_t)nchoices) >> 32)];
    const double u = (double)w[3] * 0x1p-32 + 0x1p-33;
    corrL[3 * i] = corrL[3 * i + 1] = corrL[3 * i + 2] = lmin + (lmax - lmin) * u;
  }
  return SCARL_OK;
}

}  // namespace scarl
