// sfg_step.cu -- the time-step kernels of the elastic M-PML path
// (time_evolution/elastic_wave.c:519-809), one fused launch per step.
//
// Each step of the reference makes 44 csr_matvec calls (32 distinct
// products: K1..K6 times U and W, and the consistent mass M times the 20
// split / memory fields), forms 14 right-hand sides, divides by the lumped
// mass, and applies the Newmark update.  Here one kernel streams the union
// sparsity pattern of the seven matrices once, gathers each neighbour's
// 20-value record once, accumulates all 32 products in registers and
// finishes the node in the same thread: no intermediate vector ever reaches
// memory.  The loop is memory-bound (no tensor-core work); the per-step
// traffic is the matrix stream plus one read and one write of the state.
#include <cuda_runtime.h>

#include <algorithm>

#include "sfg_internal.h"
#include "sfg_dev.cuh"
#include "sfg_step.cuh"

namespace sfg {

namespace {


// ------------------------------------------------------- FP64 kernel

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// FP64, thread per row, the reference's operation order throughout and no
// multiply-add contraction: per-product row sums from 0.0 in column order
// (csr_matvec.c:10-16), right-hand sides as written at elastic_wave.c:585-591
// and 651-657, division by the lumped mass (:709-722), Newmark (:757-776).

// receiver gather of the step's input state (elastic_wave.c:787-795)
__device__ __forceinline__ void gather_in64(const Step64 &a, int i)
{
    const StepCommon &c = a.c;
    if (c.seis_row >= 0 && i < c.nrec) {
        long long node = c.rec[i];
        const double *g = a.Gin + node * GREC;
        size_t o = (size_t)c.seis_row * c.nrec + i;
        c.seis_u[o] = add(add(g[0], g[1]), g[2]);
        c.seis_w[o] = add(add(g[3], g[4]), g[5]);
    }
}

// the 32 distinct products of row i and its 14 right-hand sides
// (elastic_wave.c:533-592, 599-658), source included
__device__ __forceinline__ void rhs64(const Step64 &a, int i, double r[14])
{
    const StepCommon &c = a.c;
    double kU[6], kW[6], m[20];
    for (int k = 0; k < 6; k++) { kU[k] = 0.0; kW[k] = 0.0; }
    for (int k = 0; k < 20; k++) m[k] = 0.0;
    const long long nz = a.nnz;
    for (int e = a.up[i]; e < a.up[i + 1]; e++) {
        const int j = a.uj[e];
        const double *g = a.Gin + (long long)j * GREC;
        const double u = add(add(g[0], g[1]), g[2]);
        const double w = add(add(g[3], g[4]), g[5]);
        const double vm = a.ux[e];
        for (int k = 0; k < 6; k++) {
            const double kv = a.ux[(k + 1) * nz + e];
            kU[k] = add(kU[k], mul(kv, u));
            kW[k] = add(kW[k], mul(kv, w));
        }
        for (int v = 0; v < 20; v++) m[v] = add(m[v], mul(vm, g[v]));
    }
    const double *cf = a.coef + (size_t)i * CREC;
    const double c0 = cf[0], c1 = cf[1], c2 = cf[2], c3 = cf[3];
    const double dx = cf[4], dy = cf[5], dxx = cf[6], dyy = cf[7];
    const double dxxp = cf[9], dyyp = cf[10];
    const double dt = c.dt;
    // m: 0..5 = M*U1..W3, 6..11 = M*V1..V6, 12..15 = M*Lx1..4, 16..19 = M*Ly1..4
    r[0] = sub(sub(mul(-c0, kU[0]), mul(mul(2.0, dx), m[6])), mul(mul(dx, dx), m[0]));
    r[0] = add(add(r[0], m[12]), m[13]);
    r[1] = sub(sub(sub(sub(mul(-c1, kW[2]), mul(c3, kW[3])), mul(dx, m[7])), mul(dy, m[7])), mul(mul(dx, dy), m[1]));
    r[2] = sub(sub(mul(-c3, kU[1]), mul(mul(2.0, dy), m[8])), mul(mul(dy, dy), m[2]));
    r[2] = add(add(r[2], m[14]), m[15]);
    r[3] = add(sub(mul(mul(mul(-dt, c0), dxx), kU[4]), mul(mul(dt, dx), m[12])), m[12]);
    r[4] = add(sub(mul(mul(mul(-dt, c3), dyyp), kW[4]), mul(mul(dt, dy), m[13])), m[13]);
    r[5] = add(sub(mul(mul(mul(-dt, c1), dxxp), kW[5]), mul(mul(dt, dx), m[14])), m[14]);
    r[6] = add(sub(mul(mul(mul(-dt, c3), dyy), kU[5]), mul(mul(dt, dy), m[15])), m[15]);
    r[7] = sub(sub(mul(-c3, kW[0]), mul(mul(2.0, dx), m[9])), mul(mul(dx, dx), m[3]));
    r[7] = add(add(r[7], m[16]), m[17]);
    r[8] = sub(sub(sub(sub(mul(-c3, kU[2]), mul(c1, kU[3])), mul(dx, m[10])), mul(dy, m[10])), mul(mul(dx, dy), m[4]));
    r[9] = sub(sub(mul(-c2, kW[1]), mul(mul(2.0, dy), m[11])), mul(mul(dy, dy), m[5]));
    r[9] = add(add(r[9], m[18]), m[19]);
    r[10] = add(sub(mul(mul(mul(-dt, c3), dxx), kW[4]), mul(mul(dt, dx), m[16])), m[16]);
    r[11] = add(sub(mul(mul(mul(-dt, c1), dyyp), kU[4]), mul(mul(dt, dy), m[17])), m[17]);
    r[12] = add(sub(mul(mul(mul(-dt, c3), dxxp), kU[5]), mul(mul(dt, dx), m[18])), m[18]);
    r[13] = add(sub(mul(mul(mul(-dt, c2), dyy), kW[5]), mul(mul(dt, dy), m[19])), m[19]);
    if (i == c.src[0]) {
        const double ps = c.amp[c.it];
        r[0] = add(r[0], mul(ps, c.sin_af));
        r[7] = add(r[7], mul(ps, c.cos_af));
    }
}

// Newmark update of row i (elastic_wave.c:754-786) from the new
// accelerations an (U1..W3) and memory variables L (Lx1..4, Ly1..4)
__device__ __forceinline__ void newmark64(const Step64 &a, int i, const double an[6], const double L[8], double &eu,
                                          double &ew)
{
    const double dt = a.c.dt;
    const double *g = a.Gin + (size_t)i * GREC;
    const double *pi = a.Pin + (size_t)i * PREC;
    double *go = a.Gout + (size_t)i * GREC;
    double *po = a.Pout + (size_t)i * PREC;
    double U[6];
    for (int k = 0; k < 6; k++) {
        const double Uk = g[k], Vk = g[6 + k], Ak = pi[k];
        const double X = add(mul(-0.5, Ak), an[k]);
        U[k] = add(add(Uk, mul(Vk, dt)), mul(mul(X, dt), dt));
        go[k] = U[k];
        go[6 + k] = add(Vk, mul(add(mul(-0.5, Ak), mul(1.5, an[k])), dt));
        po[k] = an[k];
    }
    for (int k = 0; k < 8; k++) go[12 + k] = L[k];
    const double uu = add(add(U[0], U[1]), U[2]), ww = add(add(U[3], U[4]), U[5]);
    eu = uu * uu;
    ew = ww * ww;
}

// right-hand side k of each solved field: accelerations U1..W3, then Lx1..4, Ly1..4
__constant__ int kAccRhs[6] = {0, 1, 2, 7, 8, 9};

__global__ void __launch_bounds__(128) step64_kernel(const Step64 a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    gather_in64(a, i);
    double eu = 0.0, ew = 0.0;
    if (i < a.c.n) {
        double r[14];
        rhs64(a, i, r);
        const double *cf = a.coef + (size_t)i * CREC;
        const double dirichlet_or_zero = cf[8], mlump = cf[11];
        const bool zero = dirichlet_or_zero == 0.0;
        double an[6], L[8];
        for (int k = 0; k < 6; k++) an[k] = zero ? 0.0 : __ddiv_rn(r[kAccRhs[k]], mlump);
        for (int k = 0; k < 4; k++) {
            L[k] = zero ? 0.0 : __ddiv_rn(r[3 + k], mlump);
            L[4 + k] = zero ? 0.0 : __ddiv_rn(r[10 + k], mlump);
        }
        newmark64(a, i, an, L, eu, ew);
    }
    block_energy(a.c.energy ? a.c.energy + ((size_t)a.c.it) * 2 : nullptr, eu, ew);
}

// ------------------------------------------------ consistent-mass solves
//
// The reference solves M x = rhs for the 14 fields with PARDISO or with
// restarted GMRES + ILU (tolerance 1e-8, the previous values as the first
// guess; elastic_wave.c:664-680, 730-746).  Here: conjugate gradients with
// the Jacobi preconditioner (M is symmetric positive definite), the 14
// columns together so that M is streamed once per iteration for all of
// them, started from the previous solution and stopped per column when
// |r| <= 1e-12 |b|.  Each iteration is three kernels (q = M p with p.q;
// x, r, z updates with r.z and r.r; the new directions); the block sums of
// the dot products are added atomically into per-iteration slots.  CM_MAXIT
// iterations are queued per step; once every column has converged the
// remaining ones return at once.  Scalars sc[t]: [0] r.z, [1] b.b (t = 0),
// [2] p.q, [3] r.r, each CM_COLS wide.

constexpr int kCmThreads = 256;

__device__ __forceinline__ void block_add_cols(double v[CM_COLS], double *out)
{
    __shared__ double sh[CM_COLS][kCmThreads / 32];
#pragma unroll
    for (int k = 0; k < CM_COLS; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < CM_COLS; k++) sh[k][threadIdx.x >> 5] = v[k];
    __syncthreads();
    if (threadIdx.x < CM_COLS) {
        double s = 0.0;
        for (int w = 0; w < kCmThreads / 32; w++) s += sh[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, s);
    }
    __syncthreads();
}

__device__ __forceinline__ void spmm_row(const Cm64 &g, int i, const double *__restrict__ V, double q[CM_COLS])
{
    for (int k = 0; k < CM_COLS; k++) q[k] = 0.0;
    for (int e = g.up[i]; e < g.up[i + 1]; e++) {
        const double m = g.mx[e];
        const double *v = V + (size_t)g.uj[e] * CM_COLS;
#pragma unroll
        for (int k = 0; k < CM_COLS; k++) q[k] += m * v[k];
    }
}

__device__ __forceinline__ const double *cm_sc(const Cm64 &g, int t, int which) { return g.sc + ((size_t)t * 4 + which) * CM_COLS; }

__device__ __forceinline__ bool cm_conv(const Cm64 &g, int t, int k)
{
    const double rr = cm_sc(g, t, 3)[k], bb = cm_sc(g, 0, 1)[k];
    return rr <= CM_TOL * CM_TOL * bb || rr <= 1e-200;
}

__global__ void cm_diag_kernel(const Cm64 g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    double d = 0.0;
    for (int e = g.up[i]; e < g.up[i + 1]; e++)
        if (g.uj[e] == i) d = g.mx[e];
    g.dinv[i] = d != 0.0 ? 1.0 / d : 0.0;
}

__global__ void __launch_bounds__(128) cm_rhs_kernel(const Step64 a, const Cm64 g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    gather_in64(a, i);
    if (i < a.c.n) {
        double r[14];
        rhs64(a, i, r);
        for (int k = 0; k < CM_COLS; k++) g.B[(size_t)i * CM_COLS + k] = r[k];
    }
}

// r = b - M x, z = D^-1 r, p = z; sums r.z, b.b, r.r
__global__ void __launch_bounds__(kCmThreads) cm_init_kernel(const Cm64 g)
{
    const int i = blockIdx.x * kCmThreads + threadIdx.x;
    double rz[CM_COLS], bb[CM_COLS], rr[CM_COLS];
    for (int k = 0; k < CM_COLS; k++) { rz[k] = 0.0; bb[k] = 0.0; rr[k] = 0.0; }
    if (i < g.n) {
        double q[CM_COLS];
        spmm_row(g, i, g.X, q);
        const double di = g.dinv[i];
        for (int k = 0; k < CM_COLS; k++) {
            const size_t o = (size_t)i * CM_COLS + k;
            const double b = g.B[o], r = b - q[k], z = r * di;
            g.R[o] = r; g.Z[o] = z; g.P[o] = z;
            rz[k] = r * z; bb[k] = b * b; rr[k] = r * r;
        }
    }
    block_add_cols(rz, g.sc + 0 * CM_COLS);
    block_add_cols(bb, g.sc + 1 * CM_COLS);
    block_add_cols(rr, g.sc + 3 * CM_COLS);
}

// q = M p; sum p.q into iteration t
__global__ void __launch_bounds__(kCmThreads) cm_spmm_kernel(const Cm64 g, int t)
{
    if (*g.done) return;
    const int i = blockIdx.x * kCmThreads + threadIdx.x;
    double pq[CM_COLS];
    for (int k = 0; k < CM_COLS; k++) pq[k] = 0.0;
    if (i < g.n) {
        double q[CM_COLS];
        spmm_row(g, i, g.P, q);
        for (int k = 0; k < CM_COLS; k++) {
            const size_t o = (size_t)i * CM_COLS + k;
            g.Q[o] = q[k];
            pq[k] = g.P[o] * q[k];
        }
    }
    block_add_cols(pq, g.sc + ((size_t)t * 4 + 2) * CM_COLS);
}

// x += alpha p, r -= alpha q, z = D^-1 r; sums r.z and r.r into iteration t + 1
__global__ void __launch_bounds__(kCmThreads) cm_update_kernel(const Cm64 g, int t)
{
    if (*g.done) return;
    const int i = blockIdx.x * kCmThreads + threadIdx.x;
    double rz[CM_COLS], rr[CM_COLS];
    for (int k = 0; k < CM_COLS; k++) { rz[k] = 0.0; rr[k] = 0.0; }
    if (i < g.n) {
        const double di = g.dinv[i];
        for (int k = 0; k < CM_COLS; k++) {
            const size_t o = (size_t)i * CM_COLS + k;
            double r = g.R[o];
            if (!cm_conv(g, t, k)) {
                const double alpha = cm_sc(g, t, 0)[k] / cm_sc(g, t, 2)[k];
                g.X[o] += alpha * g.P[o];
                r -= alpha * g.Q[o];
                g.R[o] = r;
                g.Z[o] = r * di;
            }
            rz[k] = r * g.Z[o];
            rr[k] = r * r;
        }
    }
    block_add_cols(rz, g.sc + ((size_t)(t + 1) * 4 + 0) * CM_COLS);
    block_add_cols(rr, g.sc + ((size_t)(t + 1) * 4 + 3) * CM_COLS);
}

// p = z + beta p for the columns still running; the flag when none is
__global__ void __launch_bounds__(kCmThreads) cm_direction_kernel(const Cm64 g, int t)
{
    if (*g.done) return;
    const int i = blockIdx.x * kCmThreads + threadIdx.x;
    bool all = true;
    for (int k = 0; k < CM_COLS; k++) {
        const bool c = cm_conv(g, t + 1, k);
        all = all && c;
        if (!c && i < g.n) {
            const size_t o = (size_t)i * CM_COLS + k;
            const double beta = cm_sc(g, t + 1, 0)[k] / cm_sc(g, t, 0)[k];
            g.P[o] = g.Z[o] + beta * g.P[o];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *g.iters += 1;
        if (all) *g.done = 1;
    }
}

// a solve that used every queued iteration without converging
__global__ void cm_check_kernel(const Cm64 g)
{
    if (*g.done) return;
    bool all = true;
    for (int k = 0; k < CM_COLS; k++) all = all && cm_conv(g, CM_MAXIT, k);
    if (!all) atomicAdd(g.fails, 1);
}

__global__ void __launch_bounds__(128) cm_newmark_kernel(const Step64 a, const Cm64 g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double eu = 0.0, ew = 0.0;
    if (i < a.c.n) {
        const double *x = g.X + (size_t)i * CM_COLS;
        double an[6], L[8];
        for (int k = 0; k < 6; k++) an[k] = x[kAccRhs[k]];
        for (int k = 0; k < 4; k++) { L[k] = x[3 + k]; L[4 + k] = x[10 + k]; }
        newmark64(a, i, an, L, eu, ew);
    }
    block_energy(a.c.energy ? a.c.energy + ((size_t)a.c.it) * 2 : nullptr, eu, ew);
}

// ------------------------------------------------ gathers, snapshots

__global__ void gather64_kernel(const StepCommon c, const double *G)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (c.seis_row < 0 || i >= c.nrec) return;
    long long node = c.rec[i];
    const double *g = G + node * GREC;
    size_t o = (size_t)c.seis_row * c.nrec + i;
    c.seis_u[o] = __dadd_rn(__dadd_rn(g[0], g[1]), g[2]);
    c.seis_w[o] = __dadd_rn(__dadd_rn(g[3], g[4]), g[5]);
}

__global__ void snapshot64_kernel(const double *G, int n, double *su, double *sw)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *g = G + (size_t)i * GREC;
    su[i] = __dadd_rn(__dadd_rn(g[0], g[1]), g[2]);
    sw[i] = __dadd_rn(__dadd_rn(g[3], g[4]), g[5]);
}

// --------------------------------------------------- unfused baseline

__global__ void spmv32_kernel(int n, const int *__restrict__ p, const int *__restrict__ j,
                              const float *__restrict__ x, const float *__restrict__ v, float *__restrict__ y)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float t = 0.f;
    for (int k = p[i]; k < p[i + 1]; k++) t += x[k] * v[j[k]];
    y[i] = t;
}

// state planes of the unfused path
enum { PU = 0, PV = 6, PA = 12, PLX = 18, PLY = 22, PUN = 26, PWN = 27, PLANES = 36 };

__global__ void plain_rhs_kernel(const Plain32 a, int half)
{
    const int n = a.c.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *e = a.eq;
    auto E = [&](int k) { return e[(size_t)k * n + i]; };
    const float4 *cf = reinterpret_cast<const float4 *>(a.coef) + (size_t)i * 3;
    const float4 c0 = cf[0], c1 = cf[1], c2 = cf[2];
    const float c11 = c0.x, c13 = c0.y, c33 = c0.z, c44 = c0.w;
    const float dx = c1.x, dy = c1.y, dxx = c1.z, dyy = c1.w, dxxp = c2.y, dyyp = c2.z;
    const float dt = (float)a.c.dt;
    float src = 0.f;
    if (i == a.c.src[0]) src = (float)(a.c.amp[a.c.it] * (half == 0 ? a.c.sin_af : a.c.cos_af));
    float *r = a.rhs + (size_t)(half * 7) * n + i;
    // equ index: 0 e11, 1 e12, 2 e13, 3 e14, 4 e15, 5 e21, 6 e22, 7 e23, 8 e24, 9 e31, 10 e32,
    // 11 e33, 12 e34, 13 e35, 14 e41, 15 e42, 16 e51, 17 e52, 18 e61, 19 e62, 20 e71, 21 e72
    float ca = half == 0 ? c11 : c44, cb1 = half == 0 ? c13 : c44, cb2 = half == 0 ? c44 : c13;
    float cc = half == 0 ? c44 : c33, c4 = half == 0 ? c11 : c44, c5 = half == 0 ? c44 : c13;
    float c6 = half == 0 ? c13 : c44, c7 = half == 0 ? c44 : c33;
    r[0] = -ca * E(0) - 2.0f * dx * E(1) - dx * dx * E(2) + E(3) + E(4) + src;
    r[(size_t)n] = -cb1 * E(5) - cb2 * E(6) - dx * E(7) - dy * E(7) - dx * dy * E(8);
    r[2 * (size_t)n] = -cc * E(9) - 2.0f * dy * E(10) - dy * dy * E(11) + E(12) + E(13);
    r[3 * (size_t)n] = -dt * c4 * dxx * E(14) - dt * dx * E(15) + E(15);
    r[4 * (size_t)n] = -dt * c5 * dyyp * E(16) - dt * dy * E(17) + E(17);
    r[5 * (size_t)n] = -dt * c6 * dxxp * E(18) - dt * dx * E(19) + E(19);
    r[6 * (size_t)n] = -dt * c7 * dyy * E(20) - dt * dy * E(21) + E(21);
}

__global__ void plain_solve_kernel(const Plain32 a)
{
    const int n = a.c.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float im = a.coef[(size_t)i * CREC + 8];
    const float *r = a.rhs;
    float *st = a.st;
    // tt_new of U1 U2 U3 W1 W2 W3 and the memory variables (elastic_wave.c:681-729)
    const int racc[6] = {0, 1, 2, 7, 8, 9};
    for (int k = 0; k < 6; k++) a.anew[(size_t)k * n + i] = r[(size_t)racc[k] * n + i] * im;
    for (int k = 0; k < 4; k++) {
        st[(size_t)(PLX + k) * n + i] = r[(size_t)(3 + k) * n + i] * im;
        st[(size_t)(PLY + k) * n + i] = r[(size_t)(10 + k) * n + i] * im;
    }
}

__global__ void plain_newmark_kernel(const Plain32 a)
{
    const int n = a.c.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double eu = 0.0, ew = 0.0;
    if (i < n) {
        float *st = a.st;
        const float dt = (float)a.c.dt;
        float u = 0.f, w = 0.f;
        for (int k = 0; k < 6; k++) {
            float U = st[(size_t)(PU + k) * n + i], V = st[(size_t)(PV + k) * n + i];
            float A = st[(size_t)(PA + k) * n + i], an = a.anew[(size_t)k * n + i];
            U = U + V * dt + (-0.5f * A + an) * dt * dt;
            V = V + (-0.5f * A + 1.5f * an) * dt;
            st[(size_t)(PU + k) * n + i] = U;
            st[(size_t)(PV + k) * n + i] = V;
            st[(size_t)(PA + k) * n + i] = an;
            if (k < 3) u += U; else w += U;
        }
        st[(size_t)PUN * n + i] = u;
        st[(size_t)PWN * n + i] = w;
        eu = (double)u * u;
        ew = (double)w * w;
    }
    block_energy(a.c.energy ? a.c.energy + ((size_t)a.c.it) * 2 : nullptr, eu, ew);
}

__global__ void plain_gather_kernel(const Plain32 a)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    const StepCommon &c = a.c;
    if (c.seis_row < 0 || r >= c.nrec) return;
    int node = c.rec[r];
    size_t o = (size_t)c.seis_row * c.nrec + r;
    c.seis_u[o] = a.st[(size_t)PUN * c.n + node];
    c.seis_w[o] = a.st[(size_t)PWN * c.n + node];
}

// ------------------------------------------------ step data builders

__global__ void permute_rows_kernel(int n, int width, const float *__restrict__ src, const int *__restrict__ perm,
                                    float *__restrict__ dst)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * width) return;
    long long r = t / width;
    int k = (int)(t - r * width);
    dst[t] = src[(long long)perm[r] * width + k];
}

__global__ void coef_kernel(int n, const double *__restrict__ c, const double *__restrict__ mp,
                            const double *__restrict__ mass, const unsigned char *__restrict__ dir,
                            float *__restrict__ c32, double *__restrict__ c64)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool zero = dir[i] || mass[i] == 0.0;
    double v[12];
    for (int k = 0; k < 4; k++) v[k] = c[(size_t)k * n + i];
    for (int k = 0; k < 4; k++) v[4 + k] = mp[(size_t)k * n + i];
    v[8] = zero ? 0.0 : 1.0 / mass[i];
    v[9] = mp[4 * (size_t)n + i];
    v[10] = mp[5 * (size_t)n + i];
    v[11] = mass[i];
    for (int k = 0; k < 12; k++) {
        c32[(size_t)i * CREC + k] = (float)v[k];
        c64[(size_t)i * CREC + k] = v[k];
    }
}

}  // namespace

// ---------------------------------------------------------- launchers

cudaError_t launch_step64(const Step64 &a, int threads, cudaStream_t st)
{
    int blocks = (a.c.n + threads - 1) / threads;
    step64_kernel<<<blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

size_t cm_scalar_count() { return (size_t)(CM_MAXIT + 1) * 4 * CM_COLS; }

cudaError_t launch_cm_diag(const Cm64 &g, cudaStream_t st)
{
    if (g.n > 0) cm_diag_kernel<<<(g.n + 255) / 256, 256, 0, st>>>(g);
    return cudaGetLastError();
}

cudaError_t launch_cm_rhs(const Step64 &a, const Cm64 &g, cudaStream_t st)
{
    const int n = std::max(a.c.n, a.c.seis_row >= 0 ? a.c.nrec : 0);
    if (n > 0) cm_rhs_kernel<<<(n + 127) / 128, 128, 0, st>>>(a, g);
    return cudaGetLastError();
}

int queue_cm_solve(const Cm64 &g, cudaStream_t st)
{
    if (cudaMemsetAsync(g.sc, 0, sizeof(double) * cm_scalar_count(), st) != cudaSuccess) return -1;
    if (cudaMemsetAsync(g.done, 0, sizeof(int), st) != cudaSuccess) return -1;
    const unsigned blocks = (unsigned)((g.n + kCmThreads - 1) / kCmThreads);
    int launches = 0;
    if (blocks) {
        cm_init_kernel<<<blocks, kCmThreads, 0, st>>>(g);
        launches++;
        for (int t = 0; t < CM_MAXIT; t++) {
            cm_spmm_kernel<<<blocks, kCmThreads, 0, st>>>(g, t);
            cm_update_kernel<<<blocks, kCmThreads, 0, st>>>(g, t);
            cm_direction_kernel<<<blocks, kCmThreads, 0, st>>>(g, t);
            launches += 3;
        }
        cm_check_kernel<<<1, 1, 0, st>>>(g);
        launches++;
    }
    return cudaGetLastError() == cudaSuccess ? launches : -1;
}

cudaError_t launch_cm_newmark(const Step64 &a, const Cm64 &g, cudaStream_t st)
{
    if (a.c.n > 0) cm_newmark_kernel<<<(a.c.n + 127) / 128, 128, 0, st>>>(a, g);
    return cudaGetLastError();
}

cudaError_t launch_gather64(const StepCommon &c, const double *G, int S, cudaStream_t st)
{
    (void)S;
    if (c.nrec > 0 && c.seis_row >= 0) gather64_kernel<<<(c.nrec + 127) / 128, 128, 0, st>>>(c, G);
    return cudaGetLastError();
}

cudaError_t launch_snapshot64(const double *G, int n, double *su, double *sw, cudaStream_t st)
{
    snapshot64_kernel<<<(n + 255) / 256, 256, 0, st>>>(G, n, su, sw);
    return cudaGetLastError();
}

cudaError_t launch_plain_step(const Plain32 &a, int threads, cudaStream_t st, int *launches)
{
    const int n = a.c.n;
    const int b = (n + threads - 1) / threads;
    float *S_ = a.st, *E_ = a.eq;
    auto P = [&](int k) { return S_ + (size_t)k * n; };
    auto Q = [&](int k) { return E_ + (size_t)k * n; };
    auto spmv = [&](int mat, const float *v, float *y) {
        spmv32_kernel<<<b, threads, 0, st>>>(n, a.m[mat].p, a.m[mat].j, a.m[mat].x, v, y);
    };
    int cnt = 0;
    for (int half = 0; half < 2; half++) {
        const float *Ux = half == 0 ? P(PUN) : P(PWN);   // the field of this half
        const float *Wx = half == 0 ? P(PWN) : P(PUN);   // the other field
        int o = half * 3;                                // U1.. or W1..
        const float *Lf = half == 0 ? P(PLX) : P(PLY);
        // elastic_wave.c:533-580 (u half) and :599-646 (w half), in order
        spmv(1, Ux, Q(0));
        spmv(0, P(PV + o), Q(1));
        spmv(0, P(PU + o), Q(2));
        spmv(0, Lf, Q(3));
        spmv(0, Lf + n, Q(4));
        spmv(3, Wx, Q(5));
        spmv(4, Wx, Q(6));
        spmv(0, P(PV + o + 1), Q(7));
        spmv(0, P(PU + o + 1), Q(8));
        spmv(2, Ux, Q(9));
        spmv(0, P(PV + o + 2), Q(10));
        spmv(0, P(PU + o + 2), Q(11));
        spmv(0, Lf + 2 * (size_t)n, Q(12));
        spmv(0, Lf + 3 * (size_t)n, Q(13));
        spmv(5, Ux, Q(14));
        spmv(0, Lf, Q(15));
        spmv(5, Wx, Q(16));
        spmv(0, Lf + n, Q(17));
        spmv(6, Wx, Q(18));
        spmv(0, Lf + 2 * (size_t)n, Q(19));
        spmv(6, Ux, Q(20));
        spmv(0, Lf + 3 * (size_t)n, Q(21));
        cnt += 22;
        plain_rhs_kernel<<<b, threads, 0, st>>>(a, half);
        cnt += 1;
    }
    plain_solve_kernel<<<b, threads, 0, st>>>(a);
    plain_newmark_kernel<<<b, threads, 0, st>>>(a);
    cnt += 2;
    if (a.c.seis_row >= 0 && a.c.nrec > 0) {
        plain_gather_kernel<<<(a.c.nrec + 127) / 128, 128, 0, st>>>(a);
        cnt += 1;
    }
    if (launches) *launches += cnt;
    return cudaGetLastError();
}

cudaError_t launch_plain_gather(const Plain32 &a, cudaStream_t st)
{
    if (a.c.seis_row >= 0 && a.c.nrec > 0) plain_gather_kernel<<<(a.c.nrec + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t permute_rows(int n, int width, const float *d_src, const int *d_perm, float **d_dst, cudaStream_t st)
{
    cudaError_t e = keep_alloc(d_dst, sizeof(float) * width * std::max(n, 1), st);
    if (e != cudaSuccess) return e;
    long long tot = (long long)n * width;
    if (tot) permute_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, width, d_src, d_perm, *d_dst);
    return cudaGetLastError();
}

cudaError_t build_coef(int n, const double *d_c, const double *d_mpml, const double *d_mass,
                       const unsigned char *d_dir, float **d_coef32, double **d_coef64, cudaStream_t st)
{
    cudaError_t e;
    if ((e = keep_alloc(d_coef32, sizeof(float) * CREC * std::max(n, 1), st)) != cudaSuccess) return e;
    if ((e = keep_alloc(d_coef64, sizeof(double) * CREC * std::max(n, 1), st)) != cudaSuccess) return e;
    coef_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, d_c, d_mpml, d_mass, d_dir, *d_coef32, *d_coef64);
    return cudaGetLastError();
}

}  // namespace sfg
