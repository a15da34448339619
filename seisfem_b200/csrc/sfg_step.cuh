// sfg_step.cuh -- step-kernel argument blocks and launchers.
//
// State layout (per shot; node-major so that one node's record is
// contiguous).  FP32 paths:
//   G[n][24]  the record neighbours gather, ordered so that rows outside the
//             M-PML read only its first 10 values:
//               0 U, 1 W (totals U1+U2+U3, W1+W2+W3, formed by the owner in
//               FP64), 2..5 Lx1..Lx4, 6..9 Ly1..Ly4, 10..15 U1 U2 U3 W1 W2 W3
//               (high FP32 part), 16..21 V1..V6 (U1t U2t U3t W1t W2t W3t),
//               22..23 A1 A2 (U1tt U2tt)
//   P[n][10]  values only the owner reads: 0..3 A3..A6 (U3tt W1tt W2tt
//             W3tt), 4..9 low FP32 parts of U1..W3 (compensated precision;
//             the displacement is hi + lo)
// FP64 path: G[n][20] = U1..W3 | V1..V6 | Lx1..4 | Ly1..4, P[n][12] = A1..A6.
// Batched runs put the shot index innermost: G[n][24][S], P[n][10][S].
// G and P are double-buffered (ping-pong) so that a step never reads a value
// it has already overwritten.
#pragma once

#include <cuda_runtime.h>

namespace sfg {

constexpr int G32 = 24;    // FP32 gathered record
constexpr int P32 = 10;    // FP32 private record
constexpr int GREC = 20;   // FP64 gathered record
constexpr int PREC = 12;   // FP64 private record
constexpr int CREC = 12;   // coefficients per node

// Coefficient record per node (FP32 and FP64 variants share the order):
//   0 c11, 1 c13, 2 c33, 3 c44, 4 dx, 5 dy, 6 dxx, 7 dyy,
//   8 1/m_lump (0 on Dirichlet or zero-mass nodes), 9 dxx_pyx, 10 dyy_pxy,
//   11 m_lump (FP64 path divides like the reference) or 0

struct StepCommon {
    int n;                 // rows (nodes)
    int it;                // time index of this step
    double dt;
    const double *amp;     // [step] Ricker value at it (FP64, seismic_source.c)
    double sin_af, cos_af; // sin/cos(Angle_force * pi / 180), elastic_wave.c:585,651
    const int *src;        // [S] source node per shot
    int nshot;             // S
    // receiver gather of the step's INPUT state (the previous step's result)
    const int *rec;        // [R]
    int nrec;
    int seis_row;          // row to write, < 0: none
    int seis_rows;         // rows per shot
    double *seis_u, *seis_w;   // [S][seis_rows][R]
    double *energy;        // [S][step][2]
    int nsteps;
};

struct Step32 {
    StepCommon c;
    const float *sell;      // SELL-32 slots [slots][8][32]
    const int *slice_ptr;   // [n/32 + 1]
    const float *rec32;     // CSR union records [nnz][8] (batched kernel)
    const int *up;          // union row pointers (batched kernel)
    const float *coef;      // [n][12]
    const float *Gin; float *Gout;
    const float *Pin; float *Pout;
};

struct Step64 {
    StepCommon c;
    const int *up, *uj;
    const double *ux;       // [7][nnz]: M, K1..K6
    long long nnz;
    const double *coef;     // [n][12]
    const double *Gin; double *Gout;
    const double *Pin; double *Pout;
};

enum StepKind { STEP_FP32_KAHAN = 0, STEP_FP32 = 1, STEP_FP64 = 2 };

// single shot
cudaError_t launch_step32(const Step32 &a, bool kahan, int threads, cudaStream_t st);
cudaError_t launch_step64(const Step64 &a, int threads, cudaStream_t st);
// S = 32 * spl shots, one warp per row
cudaError_t launch_step32_batched(const Step32 &a, bool kahan, int spl, int warps, cudaStream_t st);

// receiver gather of a finished state (after the last step), snapshots
cudaError_t launch_gather32(const StepCommon &c, const float *G, const float *P, int S, cudaStream_t st);
cudaError_t launch_gather64(const StepCommon &c, const double *G, int S, cudaStream_t st);
cudaError_t launch_snapshot32(const float *G, const float *P, int n, int S, double *snap_u, double *snap_w,
                              long long shot_stride, cudaStream_t st);
cudaError_t launch_snapshot64(const double *G, int n, double *snap_u, double *snap_w, cudaStream_t st);

// unfused baseline (elastic_wave.c structure): FP32 CSR per matrix
struct PlainCsr32 { const int *p, *j; const float *x; };
struct Plain32 {
    StepCommon c;
    PlainCsr32 m[7];        // M, K1..K6
    const float *coef;      // [n][12]
    float *st;              // [36][n] U1..W3, V1..V6, A1..A6, Lx1..4, Ly1..4, U, W, (6 pad)
    float *eq;              // [18][n]
    float *rhs;             // [14][n]
    float *anew;            // [6][n]
};
cudaError_t launch_plain_step(const Plain32 &a, int threads, cudaStream_t st, int *launches);
cudaError_t launch_plain_gather(const Plain32 &a, cudaStream_t st);

// device step data from the FP64 union CSR
cudaError_t build_sell32(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                         float **d_sell, int **d_slice_ptr, long long *slots, cudaStream_t st);
cudaError_t build_rec32(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                        float **d_rec, cudaStream_t st);
cudaError_t build_coef(int n, const double *d_c, const double *d_mpml, const double *d_mass,
                       const unsigned char *d_dir, float **d_coef32, double **d_coef64, cudaStream_t st);

}  // namespace sfg
