// smd_launch.h -- host-side declarations of the kernel launchers.
#pragma once

#include <cuda.h>

#include "smd_device.cuh"

namespace smd {

size_t rk_smem_bytes(int N, int precision);
int rk_threads(int N, int precision);
int rk_max_sites(int precision);
cudaError_t launch_rk(const LatticeDev &L, const RKJob &J, int precision, bool gen,
                      cudaStream_t st);

// local-field histograms of S samples ([S][3][N] FP64 state; imp [S][N] or
// null): hist [nh][3] counts are added to (rk_kernels.cu)
cudaError_t launch_field_hist(const LatticeDev &L, const double *state, const uint8_t *imp, int S, double r0,
                              double fc, int nh, unsigned long long *hist, bool gen, cudaStream_t st);
// static structure factor of S samples' grid transforms, series
// [3][nqb][S] FP64, added to out [3][Q] in sample order (prepass.cu)
cudaError_t launch_static_sf(const void *series, int Q, int nqb, int S, double cap, double *out,
                             cudaStream_t st);

// components per block of the grid transform (3 or 1); 0 when the grid
// does not fit one block
int grid_proj_ng(int G, int precision, const FFTPlan &p);
size_t grid_proj_smem(int G, int precision, const FFTPlan &p);
// two-pass transform of grids too large for one block (G even, <= 512)
bool grid_large_ok(int G, int precision, const FFTPlan &p);
size_t grid_large_scratch(int G, int R, int precision);   // bytes per sample
cudaError_t launch_grid_proj_large(const void *snap, int precision, int N, int W, int R,
                                   int nrec_chunk, int rec_begin, int n_rec_total,
                                   const int *grid_map, const FFTPlan &plan, const void *tw,
                                   double scale, const double *win, void *series, int nqb,
                                   void *Zg, cudaStream_t st);
cudaError_t launch_grid_proj(const void *snap, int precision, int N, int W, int R, int nrec_chunk,
                             int rec_begin, int n_rec_total, const int *grid_map,
                             const FFTPlan &plan, const void *tw, double scale, const double *win,
                             void *series, int nqb, cudaStream_t st);
// FP64 list projection on the FP64 tensor cores (proj_f64.cu)
cudaError_t launch_list_proj_f64(const double *snap, int W, int R, int nrec_chunk, int N, int rec_begin,
                                 int n_rec_total, const double *P, int Lq, const double *win, void *series,
                                 int nqb, int qoff, cudaStream_t st);
// q values per block of the series layout (series_qb) of a precision
int series_qblock(int precision);
int time_fft_qt(int n, int precision);
size_t time_fft_smem(int n, int qt, int precision, const FFTPlan &p);
// whether the shared-memory time transform takes length n
bool time_fft_fits(int n, int precision, const FFTPlan &p);
// ncomp: spin components transformed (3; 1 with series and acc offset to
// one component's rows)
cudaError_t launch_time_fft(const void *series, int precision, int W, int Q, int nqb,
                            const FFTPlan &plan, const void *tw, double *acc, int *status,
                            cudaStream_t st, int ncomp = 3);
cudaError_t launch_aos_to_soa(const double *in, double *out, int W, int N, cudaStream_t st);
cudaError_t launch_soa_to_aos(const double *in, double *out, int W, int N, cudaStream_t st);
cudaError_t launch_sum_rows(const double *rows, int W, int n, double *out, cudaStream_t st);
cudaError_t launch_scale(double *p, size_t n, double f, cudaStream_t st);

// tensor-core list projection (proj_tc.cu)
bool make_bf16_map(CUtensorMap *map, const void *base, int rows, int kp, int box_rows);
int tc_kpitch(int N);
int tc_bn();
int tc_bm();
cudaError_t launch_split_bf16(const float *x, int rows, int N, int kp, void *hi, void *lo,
                              cudaStream_t st);
cudaError_t launch_list_proj_tc(const CUtensorMap &Ah, const CUtensorMap &Al, const CUtensorMap &Bh,
                                const CUtensorMap &Bl, int M, int kp, int R, int nrec_chunk,
                                int rec_begin, int n_rec_total, int Lq, const double *win,
                                void *series, int nqb, int qoff, int *status, cudaStream_t st);

}  // namespace smd
