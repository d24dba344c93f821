// host_maps.h -- host-side restatements shared by the C-ABI layer.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "../../include/scarl.h"

namespace scarl {

int verify_inputs(const scarl_sample* s, int gen_meth, char* msg, size_t len);
void decide_topo_shape(int nb_procs, const int L[3], const int ovlp[3], long long ppbi,
                       int topo[3]);
void get_topo_pos(int rank, const int shape[3], int pos[3]);
int get_topo_rank(const int shape[3], const int pos[3]);
int sample_layout(const scarl_sample* s, int gen_meth, int nb_procs, const int* topo_in,
                  scarl_layout* o);
void tile_geometry(const scarl_layout* lay, const double xMin[3], int rank, scarl_tile* t);
std::vector<double> pou_pattern(int Np_ovlp, int side, int topo_pos, int topo_shape,
                                int partitionType);
void pou_axis_tables(int Np, int Np_ovlp, int topo_pos, int topo_shape, int partitionType,
                     double* lo, double* hi);
void blend_axis_flags(int Np, int Np_ovlp, int topo_pos, int topo_shape, uint8_t* flags);
void unity_partition_weights(const int Np[3], const int No[3], int partitionType,
                             const int pos[3], const int shape[3], double* w);
int shino_sizes(const int Np[3], const double xRange[3], const double corrL[3], int sz_c[3],
                int sz_Sk[3], double delta_k[3]);
double axis_correlation(int corrMod, double nu, double l, double r);
// Padded lengths the generator runs: 8..2048, a power of two or m 2^a with
// m = 3, 5, 7 and 2^a >= 16.
bool fft_length_supported(int n);
int pad_size(int policy, int corrMod, double nu, const double corrL[3], const double xStep[3],
             const int Np[3], double tol, int P[3]);
int ensemble_draw(uint64_t seed, long long first, int n, const int* choices, int nchoices,
                  double lmin, double lmax, int* Np, double* corrL);
int read_config(const char* path, int* gen_meth, int* c_info, int* d_sample, int* one_file,
                int* one_hdf_ds, char* input_file, size_t len);
int read_extra_config(const char* path, int* found, int topo[3]);
int read_input(const char* path, char* folder, size_t flen, int* nSamples, scarl_sample* out,
               int max_samples);
int read_input_sem(const char* folder, char* out_folder, size_t flen, int* nSamples,
                   scarl_sample* out, int max_samples);

}  // namespace scarl
