// rk_rows.cuh -- RK4 + energy-correction kernel for Bravais lattices with
// one site per cell (square, triangular) stored as a padded 2D grid of rows
// (declarations shared by host and device code).
//
// Site g = x + L y.  Every neighbour of shell s sits at a fixed cell offset
// (dx, dy) with |dx|, |dy| <= 2 (the tables of make_nborsTable,
// Codes_Folder/subrouts.cpp:2983-3316, are translation invariant; the host
// checks that before choosing this kernel).  A sample is cut into CS bands
// of rows, one per CTA of a cluster.  A CTA keeps its rows plus two ghost
// rows above and below and two ghost columns on each side in shared memory
// so every neighbour of a site is at a constant offset from the site's own
// record: the field of a thread's SPT consecutive sites of a row is
// gathered from five row windows, each value loaded once and used by every
// site that needs it.  Within a row, one pad record follows every SPT
// records (column x at rows_col(x)), so the windows of consecutive threads
// start SPT + 1 records apart and a quarter-warp's 16-byte loads fall in
// distinct banks.  Ghost columns are
// written by the owners of the wrapped columns; ghost rows by the owners in
// the neighbouring bands (distributed shared memory stores); one split
// cluster barrier per stage, as in the cluster kernel.
#pragma once

#include "rk_cluster.cuh"

namespace smd {

enum { kStencilSquare = 0, kStencilTriang = 1 };

struct RowsParams {
    int N, L, CS;
    int ny_max;                       // rows of the largest band
    int row0[kMaxClusterCTAs + 1];    // first row of each band, row0[CS] = L
    int geom;                         // kStencilSquare or kStencilTriang
    int shells;                       // active shells, bit s = shell s
    double h;
    double coef64[3][3];              // J_s * lambda_s per shell and component
    float coef32[3][3];
};

// Cell offsets of the shells, in a fixed order per geometry.
__host__ __device__ constexpr int stencil_z(int geom, int s)
{
    return geom == kStencilSquare ? 4 : 6;
}

__host__ __device__ constexpr int stencil_off(int geom, int s, int e, int xy)
{
    // square: (0,-1) (1,0) (0,1) (-1,0) | (1,-1) (1,1) (-1,1) (-1,-1) | (0,-2) (2,0) (0,2) (-2,0)
    // triang: (0,-1) (1,-1) (1,0) (0,1) (-1,1) (-1,0) | (1,-2) (2,-1) (1,1) (-1,2) (-2,1) (-1,-1)
    //         | (0,-2) (2,-2) (2,0) (0,2) (-2,2) (-2,0)
    constexpr int sq[3][4][2] = {{{0, -1}, {1, 0}, {0, 1}, {-1, 0}},
                                 {{1, -1}, {1, 1}, {-1, 1}, {-1, -1}},
                                 {{0, -2}, {2, 0}, {0, 2}, {-2, 0}}};
    constexpr int tr[3][6][2] = {{{0, -1}, {1, -1}, {1, 0}, {0, 1}, {-1, 1}, {-1, 0}},
                                 {{1, -2}, {2, -1}, {1, 1}, {-1, 2}, {-2, 1}, {-1, -1}},
                                 {{0, -2}, {2, -2}, {2, 0}, {0, 2}, {-2, 2}, {-2, 0}}};
    return geom == kStencilSquare ? sq[s][e][xy] : tr[s][e][xy];
}

// sites per thread, and the block-size limit of a precision: FP32 blocks
// of up to 576 threads (96 registers each), FP64 up to 384 (168)
constexpr int rows_spt(int precision) { return precision == 0 ? 2 : 2; }
constexpr int rows_max_threads(int precision) { return precision == 0 ? 384 : 576; }

// floor(x / spt) for x >= -spt
__host__ __device__ constexpr int rows_fdiv(int x, int spt) { return (x + spt) / spt - 1; }
// record of column x (-2 <= x < L + 2) within a row
__host__ __device__ constexpr int rows_col(int x, int spt) { return x + 3 + rows_fdiv(x, spt); }
// records per row
__host__ __device__ constexpr int rows_pitch(int L, int spt) { return rows_col(L + 1, spt) + 1; }

size_t rk_rows_smem(const RowsParams &P, int precision);
int rk_rows_threads(const RowsParams &P, int precision);
cudaError_t launch_rk_rows(const RowsParams &P, const RKJob &J, int precision, cudaStream_t st);

}  // namespace smd
