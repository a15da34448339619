// sfg_step.cuh -- step-kernel argument blocks and launchers.
//
// FP64 path state (original node numbering, node-major):
//   G[n][20] = U1..W3 | V1..V6 (U1t..W3t) | Lx1..4 | Ly1..4, P[n][12] = A1..A6
// The FP32 fused paths use the two-class layout of sfg_step32.cuh.
#pragma once

#include <cuda_runtime.h>

namespace sfg {

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

cudaError_t launch_step64(const Step64 &a, int threads, cudaStream_t st);

// Consistent-mass solves (elastic_wave.c:664-680, 730-746: solver "pardiso" /
// "mgmres"): the 14 right-hand sides of a step are solved with M itself by a
// Jacobi-preconditioned conjugate gradient over all 14 columns at once.
constexpr int CM_COLS = 14;
constexpr int CM_MAXIT = 64;          // iterations queued per step (later ones return at once)
constexpr double CM_TOL = 1e-12;      // |r| <= CM_TOL |b| per column
struct Cm64 {
    int n;
    const int *up, *uj;
    const double *mx;                 // M on the union pattern (value stream 0)
    double *dinv;                     // [n] 1 / M_ii
    double *B, *X, *R, *Z, *P, *Q;    // [n][14]; X holds the previous step's solution
    double *sc;                       // [CM_MAXIT + 1][4][14]: r.z, b.b, p.q, r.r
    int *done;                        // all columns converged
    int *fails;                       // steps whose solve did not converge (accumulated)
    int *iters;                       // iterations run (accumulated)
};
size_t cm_scalar_count();
cudaError_t launch_cm_diag(const Cm64 &g, cudaStream_t st);
// the products and right-hand sides of step64_kernel into g.B (and the
// receiver gather of the step's input state)
cudaError_t launch_cm_rhs(const Step64 &a, const Cm64 &g, cudaStream_t st);
// M X = B; returns the number of kernels queued, or -1
int queue_cm_solve(const Cm64 &g, cudaStream_t st);
// Newmark update from the solved accelerations and memory variables
cudaError_t launch_cm_newmark(const Step64 &a, const Cm64 &g, cudaStream_t st);
// receiver gather of a finished state (after the last step), snapshots
cudaError_t launch_gather64(const StepCommon &c, const double *G, int S, cudaStream_t st);
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
cudaError_t permute_rows(int n, int width, const float *d_src, const int *d_perm, float **d_dst, cudaStream_t st);
cudaError_t build_coef(int n, const double *d_c, const double *d_mpml, const double *d_mass,
                       const unsigned char *d_dir, float **d_coef32, double **d_coef64, cudaStream_t st);

}  // namespace sfg
