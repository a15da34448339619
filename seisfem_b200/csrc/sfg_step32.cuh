// sfg_step32.cuh -- the fused FP32 step in the two-class node numbering.
//
// Node classes (decided at set-up from the M-PML profiles and the union
// sparsity pattern):
//   Z  the split zone: rows inside the M-PML (any of dx, dy, dxx, dyy non-zero)
//      and every column those rows reference -- the nodes whose split fields
//      U1 U2 U3 / W1 W2 W3 somebody reads;
//   A  all other nodes.  Their rows multiply every split-field, K5 and K6
//      product by a zero damping coefficient, and nobody reads their split
//      fields, so they carry only the totals U = U1+U2+U3, W = W1+W2+W3 (the
//      Newmark update, elastic_wave.c:757-768, is linear: the totals follow
//      the same recursion with the summed accelerations).
// Numbering: rows [0, na) are class A, rows [na, n) class Z, na a multiple
// of 32 (the last few rows of A join Z); inside each class, windows of 2048
// rows are sorted by (M-PML flag, row length) so that 32-row SELL slices need
// no padding.  perm[r'] is the mesh node of row r'.
//
// State records (node-major, shot index innermost for batches of S shots):
//   Gc[n][12]   gathered by every row: U W Lx1 Lx2 | Lx3 Lx4 Ly1 Ly2 | Ly3 Ly4
//               lo_u lo_w   (the totals as FP32 pairs U + lo_u, W + lo_w: in
//               class A the compensated displacement itself, in class Z the
//               FP64 sum of the split pairs split into two floats; the
//               one-shot kernels form K U as sum_j K_ij (U_j - U_i) from both
//               parts, since every row of K1..K6 sums to zero)
//   Pa[na][4]   class A, private: Au Aw Vu Vw (total accelerations, velocities)
//   Gs[nz][12]  class Z, gathered by M-PML rows: U1 U2 U3 W1 W2 W3 (high FP32
//               part) | V1..V6
//   Ps[nz][12]  class Z, private: A1..A6 | lo1..lo6
// Compensated precision keeps every displacement as an FP32 pair hi + lo
// updated with a Kahan sum; the plain FP32 variant leaves lo at 0.
#pragma once

#include <cuda_runtime.h>

#include "sfg_step.cuh"

namespace sfg {

constexpr int GC = 12, PA = 4, GS = 12, PS = 12;

// One-shot layout (S = 1) of the 48-byte records Gc, Gs, Ps and the class-Z
// coefficients: rows in blocks of 32, block b holding float4 q of its rows
// 32 b .. 32 b + 31 contiguously (q = 0 .. nq - 1).  The 32 rows of a SELL
// slice gather neighbours that are mostly consecutive rows, so one float4
// load of the warp touches 4-5 128-byte lines instead of the 12 of records
// laid end to end.  Arrays in this layout hold whole blocks (rows rounded up
// to 32).  Batches (S > 1) keep [row][value][S].
__host__ __device__ __forceinline__ long long blk4(long long r, int q, int nq)
{
    return (((r >> 5) * nq + q) << 5) | (r & 31);
}
// rows rounded up to whole blocks of 32
__host__ __device__ __forceinline__ long long blk_rows(long long n) { return (n + 31) & ~31LL; }

struct State32 {
    const float *Gc, *Pa, *Gs, *Ps;
};
struct State32W {
    float *Gc, *Pa, *Gs, *Ps;
};

struct Step2 {
    StepCommon c;              // c.n = all rows; src / rec in the permuted numbering
    int na;                    // class-A rows [0, na); class Z [na, n)
    int S;                     // shots of the batch: the state's innermost stride
    const float *sellA;        // SELL-32 over rows [0, na): planes col, M, K1..K4
    const int *sliceA;
    const float *sellZ;        // SELL-32 over rows [na, n): planes col, M, K1..K6
    const int *sliceZ;
    // value dictionary (sfg_dict.cu; dict_n = 0 without one): the one-shot
    // kernels then read SELL-32 slots (q, d) from sellAd / sellZd (same
    // slices as sellA / sellZ): q = blk4(column, 0, 3), the float4 index of
    // the column's Gc record, and d = 2 id, the tuple (M / rho_row, K1..K6)
    // being dict[d], dict[d + 1]; the mass products are scaled by rowrho
    const int2 *sellAd;
    const int2 *sellZd;
    const float4 *dict;
    int dict_n;
    const float *rowrho;       // [n] row density, permuted numbering
    const float4 *h_dict;      // host copy of dict[0 .. 2 dict_n), or nullptr: the one-shot launches
                               // of at most kParamTuples tuples pass it in the kernel's parameters
    const int *up;             // row-major union records in the permuted numbering
    const float *rec;          //   [nnz][8]: col, M, K1..K6
    const float *recA;         // class-A rows, one model: [upp[na]][8] col, M and the
                               //   constants folded into K1..K4 (rec_fold_fill)
    const float4 *coefA;       // [na] c11 c13 c33 c44
    const float *imA;          // [na] 1/m_lump (0 on Dirichlet rows)
    const float *coefZ;        // [n-na][12] (sfg_step.cuh coefficient order)
    // one model per shot (batched, compensated): rec then carries the
    // geometric mass matrix M_geo (M = diag(rho) M_geo), cmm[n][6][S] the
    // shot's c11 c13 c33 c44, 1/m_lump (0 on Dirichlet rows) and rho, and
    // sig[S] its vp_max over the set-up model's (the M-PML profiles scale
    // linearly with vp_max); nullptr otherwise
    const float *cmm;
    const float *sig;
    State32 in;
    State32W out;
    // staged-gather tiles of the one-shot kernels (value dictionary only;
    // tileA_off == nullptr without them): each class is cut into windows of
    // kTileRows consecutive rows; tile t's halo is its own rows followed by
    // the rows tile?_ext[tile?_off[t] .. tile?_off[t + 1]) (sorted) that
    // its rows reference outside it; the SELL-32 slots (same slices as
    // sellAd / sellZd) hold (halo position << 16 | tuple id)
    const unsigned *sellAt, *sellZt;
    const int *tileA_off, *tileA_ext, *tileZ_off, *tileZ_ext;
    int haloA_max, haloZ_max;  // largest halo of a tile of each class (rows)
    int slotsA_max, slotsZ_max;  // most SELL slot rows (32 slots each) of a tile of each class
    int max_row_len;           // longest union row (slot rows of one slice at most)
};

// rows per staged-gather tile (one block of as many threads per tile)
constexpr int kTileRows = 256;
// largest halo a tile may have (own rows included); a mesh whose tiles reach
// further keeps the unstaged kernels
constexpr int kTileHaloMax = 2048;

// single shot (thread per row); variant = launch shape 0..step2_variants()-1
int step2_variants();
cudaError_t launch_stepA(const Step2 &a, bool comp, int variant, cudaStream_t st);
cudaError_t launch_stepZ(const Step2 &a, bool comp, int variant, cudaStream_t st);
// threads per block of one-shot launch shape `variant`
int step2_threads(int variant);
// several one-shot problems per launch: descs[m] the step descriptor of mesh
// m for this step's parity (it and the receiver row are set from `it`);
// map[b] = (mesh, block of that mesh) for each of the nblocks blocks, blocks
// of step2_threads(variant) rows; dict: every mesh has a value dictionary,
// dict_max its largest tuple count
cudaError_t launch_stepA_multi(const Step2 *descs, const int2 *map, int nblocks, bool dict, int dict_max, bool comp,
                               int variant, int it, cudaStream_t st);
cudaError_t launch_stepZ_multi(const Step2 *descs, const int2 *map, int nblocks, bool dict, int dict_max, bool comp,
                               int variant, int it, cudaStream_t st);
// staged-gather tiles (launch shape kTileShape of launch_stepA / launch_stepZ):
// the tile's own records and its halo are copied into shared memory with
// cp.async, and every gather of the step reads shared memory
constexpr int kTileShape = 6;
// one-shot kernels whose 128-row blocks copy their slot streams into shared
// memory before their rows start (value dictionary; gathers stay global)
constexpr int kSlotStageShape = 7;
cudaError_t launch_stepA_tile(const Step2 &a, bool comp, cudaStream_t st);
cudaError_t launch_stepZ_tile(const Step2 &a, bool comp, cudaStream_t st);
// S = a.S shots, a multiple of 32 * spl; a warp advances 32 * spl shots of
// one row (spl per lane); warps per block a multiple of S / (32 * spl)
cudaError_t launch_stepA_batched(const Step2 &a, bool comp, int spl, int warps, cudaStream_t st);
int stepA_batched_max_warps(int spl, bool models);
cudaError_t launch_stepZ_batched(const Step2 &a, bool comp, int spl, int warps, cudaStream_t st);
// class A with staged neighbour gathers (cp.async into per-warp shared-memory
// buffers), 64 shots, one persistent block of 8 warps per SM
cudaError_t launch_stepA_staged(const Step2 &a, bool comp, cudaStream_t st);
// receiver gather of a finished state; snapshots scattered back to mesh order
cudaError_t launch_gather2(const StepCommon &c, int na, const State32 &s, int S, cudaStream_t st);
cudaError_t launch_snapshot2(const State32 &s, int n, int na, int S, const int *perm, double *snap_u,
                             double *snap_w, long long shot_stride, cudaStream_t st);

// set-up builders
// SELL-32 over permuted rows [r0, r1) with `planes` planes (6: col M K1..K4; 8: + K5 K6)
cudaError_t build_sell_range(int r0, int r1, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                             const int *d_perm, const int *d_inv, int planes, float **d_sell, int **d_slice,
                             long long *slots, cudaStream_t st);
// row-major records in the permuted numbering (d_upp: permuted row pointers)
cudaError_t build_rec_perm(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                           const int *d_perm, const int *d_inv, const int *d_upp, float **d_rec, cudaStream_t st);
// the two-class numbering on the device: perm (class A, then class Z; windows
// of 2048 rows stably sorted by M-PML flag and decreasing length), its
// inverse and the permuted row pointers; na = class-A rows, npml = M-PML rows
// tile_rows > 0: windows of tile_rows rows (a power of two <= 2048) instead
// of 2048; d_x, d_y given: rows inside each class in Morton order of the node
// coordinates (over [x0, x1] x [y0, y1]) before the windows, else mesh order
cudaError_t build_classes(int n, const int *d_up, const int *d_uj, const double *d_mpml, int maxlen, int **d_perm,
                          int **d_inv, int **d_upp, int *na, int *npml, cudaStream_t st, int tile_rows = 0,
                          const double *d_x = nullptr, const double *d_y = nullptr, double x0 = 0, double x1 = 1,
                          double y0 = 0, double y1 = 1);
// staged-gather tiles of permuted rows [r0, r1) (windows of kTileRows): the
// external halo rows per tile (d_off [ntiles + 1], d_ext) and the packed
// SELL-32 slots over the slices of d_slice (build_sell_range_dict's);
// *halo_max = the largest halo (own rows included), or -1 when a tile's
// halo passes kTileHaloMax (no tile data is then kept); *slots_max = the most
// slot rows (32 slots each) of a tile
cudaError_t build_tiles(int r0, int r1, const int *d_up, const int *d_uj, const int *d_tid, int zero_id,
                        const int *d_perm, const int *d_inv, const int *d_slice, long long slots, int **d_off,
                        int **d_ext, unsigned **d_sell, int *halo_max, int *slots_max, cudaStream_t st);
// one model per shot: row records with M_geo = M / rho0(row) in plane 1
// (stream-ordered allocation), and the row sums of M_geo in mesh order
cudaError_t build_rec_geo(int n, const int *d_up, const double *d_ux, long long nnz, const int *d_perm,
                          const int *d_upp, const double *d_rho0, const float *d_recp, float **d_rec, cudaStream_t st);
cudaError_t mass_row_sums_geo(int n, const int *d_up, const double *d_ux, const double *d_rho0, double *d_out,
                              cudaStream_t st);
// class-A / class-Z coefficient arrays from the [n][12] FP32 record
// value dictionary of the one-shot kernels (sfg_dict.cu): at most kDictMax
// tuples of (M / rho_row, K1..K6), two float4 each in shared memory
constexpr int kDictMax = 512;
// tuples the one-shot launches pass in the kernel's parameters (2 float4
// each: 4 KB)
constexpr int kParamTuples = 128;
// tuples found (0: not applicable, the kernels keep full-value slots; -1 on a
// CUDA error); d_tid[nnz] the tuple id of every union entry, d_table[2 T]
int build_value_dict(int n, const int *d_up, const double *d_ux, long long nnz, const double *d_rho, int **d_tid,
                     float4 **d_table, int *zero_id, cudaStream_t st);
cudaError_t build_sell_range_dict(int r0, int r1, const int *d_up, const int *d_uj, const int *d_tid, int zero_id,
                                  const int *d_perm, const int *d_inv, int2 **d_sell, int **d_slice, long long *slots,
                                  cudaStream_t st);
cudaError_t build_row_density(int n, const double *d_rho, const int *d_perm, float **d_out, cudaStream_t st);
cudaError_t launch_range_slice_len(int r0, int r1, const int *d_up, const int *d_perm, int *d_len, cudaStream_t st);

// the folded class-A records of Step2::recA (c: [4][n] c11 c13 c33 c44, mesh order)
cudaError_t build_rec_fold(int n, int na, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                           const int *d_perm, const int *d_inv, const int *d_upp, const double *d_c, float **d_rec,
                           cudaStream_t st);
cudaError_t build_coef2(int n, int na, const float *d_coef32, const int *d_perm, float4 **d_coefA, float **d_imA,
                        float **d_coefZ, cudaStream_t st);

}  // namespace sfg
