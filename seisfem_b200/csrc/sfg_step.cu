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
#include "sfg_step.cuh"

namespace sfg {

namespace {

__device__ __forceinline__ float ldgf(const float *p) { return __ldg(p); }

// Block-wide sum of (a, b) into dst[0], dst[1] (one atomic pair per block).
__device__ __forceinline__ void block_energy(double *dst, double a, double b)
{
    __shared__ double sa[32], sb[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = l < nw ? sa[l] : 0.0;
        b = l < nw ? sb[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (l == 0 && dst) { atomicAdd(dst, a); atomicAdd(dst + 1, b); }
    }
}

// Receiver gather of a finished FP32 state into seismogram row `row`
// (elastic_wave.c:787-795): displacement = sum over the three split fields
// of (high + low FP32 part), formed in FP64.
__device__ __forceinline__ void gather_one32(const StepCommon &c, const float *G, const float *P, int S,
                                             int t, int row)
{
    if (row < 0 || t >= c.nrec * S) return;
    int s = t / c.nrec, r = t - s * c.nrec;
    long long node = c.rec[r];
    double u = 0.0, w = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        u += (double)G[(node * G32 + 10 + k) * S + s] + (double)P[(node * P32 + 4 + k) * S + s];
        w += (double)G[(node * G32 + 13 + k) * S + s] + (double)P[(node * P32 + 7 + k) * S + s];
    }
    size_t o = ((size_t)s * c.seis_rows + row) * c.nrec + r;
    c.seis_u[o] = u;
    c.seis_w[o] = w;
}

// ------------------------------------------------ FP32 single-shot kernel

template <typename T>
struct RhsT {
    T a[6];          // accelerations of U1 U2 U3 W1 W2 W3
    T lx[4], ly[4];  // new memory variables
};

// Right-hand sides (elastic_wave.c:585-591, 651-657) times 1/m_lump
// (:709-722), evaluated in T (FP64 for the compensated path) from the FP32
// products: kU[k], kW[k] = K_{k+1} times U, W; m[0..19] = M times U1..W3,
// V1..V6, Lx1..4, Ly1..4.
template <typename T>
__device__ __forceinline__ void rhs_eval(const float *kU, const float *kW, const float *m, float4 c0, float4 c1,
                                         float4 c2, T dt, T src_u, T src_w, RhsT<T> &o)
{
    const T c11 = c0.x, c13 = c0.y, c33 = c0.z, c44 = c0.w;
    const T dx = c1.x, dy = c1.y, dxx = c1.z, dyy = c1.w;
    const T im = c2.x, dxxp = c2.y, dyyp = c2.z;
    const T kx = T(1) - dt * dx, ky = T(1) - dt * dy;
    auto K = [&](const float *v, int k) { return T(v[k]); };
    auto Mv = [&](int k) { return T(m[k]); };
    o.a[0] = im * (-c11 * K(kU, 0) - T(2) * dx * Mv(6) - dx * dx * Mv(0) + Mv(12) + Mv(13) + src_u);
    o.a[1] = im * (-c13 * K(kW, 2) - c44 * K(kW, 3) - (dx + dy) * Mv(7) - dx * dy * Mv(1));
    o.a[2] = im * (-c44 * K(kU, 1) - T(2) * dy * Mv(8) - dy * dy * Mv(2) + Mv(14) + Mv(15));
    o.lx[0] = im * (-dt * c11 * dxx * K(kU, 4) + kx * Mv(12));
    o.lx[1] = im * (-dt * c44 * dyyp * K(kW, 4) + ky * Mv(13));
    o.lx[2] = im * (-dt * c13 * dxxp * K(kW, 5) + kx * Mv(14));
    o.lx[3] = im * (-dt * c44 * dyy * K(kU, 5) + ky * Mv(15));
    o.a[3] = im * (-c44 * K(kW, 0) - T(2) * dx * Mv(9) - dx * dx * Mv(3) + Mv(16) + Mv(17) + src_w);
    o.a[4] = im * (-c44 * K(kU, 2) - c13 * K(kU, 3) - (dx + dy) * Mv(10) - dx * dy * Mv(4));
    o.a[5] = im * (-c33 * K(kW, 1) - T(2) * dy * Mv(11) - dy * dy * Mv(5) + Mv(18) + Mv(19));
    o.ly[0] = im * (-dt * c44 * dxx * K(kW, 4) + kx * Mv(16));
    o.ly[1] = im * (-dt * c13 * dyyp * K(kU, 4) + ky * Mv(17));
    o.ly[2] = im * (-dt * c44 * dxxp * K(kU, 5) + kx * Mv(18));
    o.ly[3] = im * (-dt * c33 * dyy * K(kW, 5) + ky * Mv(19));
}

// Newmark, alpha = 1, delta = 1.5 (elastic_wave.c:97, 757-768), for one split
// field.  Compensated: the displacement is carried as an FP32 pair hi + lo,
// updated in FP64 and split again, so the running sum keeps ~48 bits.
__device__ __forceinline__ double newmark_comp(float &hi, float &lo, float &V, float &A, double an, double dt)
{
    const double Ad = A, Vd = V;
    const double U = ((double)hi + (double)lo) + Vd * dt + (an - 0.5 * Ad) * (dt * dt);
    hi = (float)U;
    lo = (float)(U - (double)hi);
    V = (float)(Vd + (1.5 * an - 0.5 * Ad) * dt);
    A = (float)an;
    return U;
}

__device__ __forceinline__ float newmark_plain(float &U, float &V, float &A, float an, float dt)
{
    U = U + V * dt + (an - 0.5f * A) * (dt * dt);
    V = V + (1.5f * an - 0.5f * A) * dt;
    A = an;
    return U;
}

// Finish one node: right-hand sides, lumped solve, Newmark, new records.
// g[24] / p[10] are the node's own records (layout in sfg_step.cuh).
template <bool COMP>
__device__ __forceinline__ void finish_node(const float *kU, const float *kW, const float *m, float4 c0, float4 c1,
                                            float4 c2, double dt, double src_u, double src_w, const float *g,
                                            const float *p, float *go, float *po, double &uu, double &ww)
{
    float hi[6] = {g[10], g[11], g[12], g[13], g[14], g[15]};
    float V[6] = {g[16], g[17], g[18], g[19], g[20], g[21]};
    float A[6] = {g[22], g[23], p[0], p[1], p[2], p[3]};
    float lo[6] = {p[4], p[5], p[6], p[7], p[8], p[9]};
    float Lx[4], Ly[4];
    double Ut[6];
    if (COMP) {
        RhsT<double> r;
        rhs_eval<double>(kU, kW, m, c0, c1, c2, dt, src_u, src_w, r);
#pragma unroll
        for (int k = 0; k < 6; k++) Ut[k] = newmark_comp(hi[k], lo[k], V[k], A[k], r.a[k], dt);
#pragma unroll
        for (int k = 0; k < 4; k++) { Lx[k] = (float)r.lx[k]; Ly[k] = (float)r.ly[k]; }
    } else {
        RhsT<float> r;
        rhs_eval<float>(kU, kW, m, c0, c1, c2, (float)dt, (float)src_u, (float)src_w, r);
#pragma unroll
        for (int k = 0; k < 6; k++) Ut[k] = newmark_plain(hi[k], V[k], A[k], r.a[k], (float)dt);
#pragma unroll
        for (int k = 0; k < 4; k++) { Lx[k] = r.lx[k]; Ly[k] = r.ly[k]; }
    }
    uu = (Ut[0] + Ut[1]) + Ut[2];
    ww = (Ut[3] + Ut[4]) + Ut[5];
    go[0] = (float)uu; go[1] = (float)ww;
#pragma unroll
    for (int k = 0; k < 4; k++) { go[2 + k] = Lx[k]; go[6 + k] = Ly[k]; }
#pragma unroll
    for (int k = 0; k < 6; k++) { go[10 + k] = hi[k]; go[16 + k] = V[k]; }
    go[22] = A[0]; go[23] = A[1];
    po[0] = A[2]; po[1] = A[3]; po[2] = A[4]; po[3] = A[5];
#pragma unroll
    for (int k = 0; k < 6; k++) po[4 + k] = COMP ? lo[k] : 0.f;
}

__device__ __forceinline__ bool is_pml_row(float4 c1)
{
    return c1.x != 0.f || c1.y != 0.f || c1.z != 0.f || c1.w != 0.f;
}

// One thread per row over SELL-32 slices.  Rows outside the M-PML (their
// dx, dy, dxx, dyy are 0) multiply every M*V, M*U_k, K5 and K6 product by 0,
// so a warp whose rows are all interior streams only the column, M and
// K1..K4 planes and gathers only U, W, Lx, Ly (the first 10 record values).
template <bool COMP>
__global__ void __launch_bounds__(256) step32_kernel(const Step32 a)
{
    const StepCommon &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    gather_one32(c, a.Gin, a.Pin, 1, i, c.seis_row);
    float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0, c2 = c0;
    if (i < c.n) {
        const float4 *cf = reinterpret_cast<const float4 *>(a.coef) + (size_t)i * 3;
        c0 = __ldg(cf); c1 = __ldg(cf + 1); c2 = __ldg(cf + 2);
    }
    const bool full = __any_sync(0xffffffffu, i < c.n && is_pml_row(c1));
    double eu = 0.0, ew = 0.0;
    if (i < c.n) {
        const int lane = i & 31, slice = i >> 5;
        float kU[6], kW[6], m[20];
#pragma unroll
        for (int k = 0; k < 6; k++) { kU[k] = 0.f; kW[k] = 0.f; }
#pragma unroll
        for (int k = 0; k < 20; k++) m[k] = 0.f;
        const int s0 = __ldg(a.slice_ptr + slice), s1 = __ldg(a.slice_ptr + slice + 1);
        const float *sd = a.sell + (size_t)s0 * 256 + lane;
        if (full) {
#pragma unroll 2
            for (int g = s0; g < s1; ++g, sd += 256) {
                const int j = __float_as_int(ldgf(sd));
                const float vm = ldgf(sd + 32);
                float kv[6];
#pragma unroll
                for (int k = 0; k < 6; k++) kv[k] = ldgf(sd + 64 + 32 * k);
                const float4 *gj = reinterpret_cast<const float4 *>(a.Gin + (size_t)j * G32);
                const float4 q0 = __ldg(gj), q1 = __ldg(gj + 1), q2 = __ldg(gj + 2), q3 = __ldg(gj + 3),
                             q4 = __ldg(gj + 4);
                const float2 q5 = __ldg(reinterpret_cast<const float2 *>(gj + 5));
#pragma unroll
                for (int k = 0; k < 6; k++) { kU[k] += kv[k] * q0.x; kW[k] += kv[k] * q0.y; }
                m[0] += vm * q2.z;  m[1] += vm * q2.w;  m[2] += vm * q3.x;  m[3] += vm * q3.y;
                m[4] += vm * q3.z;  m[5] += vm * q3.w;  m[6] += vm * q4.x;  m[7] += vm * q4.y;
                m[8] += vm * q4.z;  m[9] += vm * q4.w;  m[10] += vm * q5.x; m[11] += vm * q5.y;
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        } else {
#pragma unroll 2
            for (int g = s0; g < s1; ++g, sd += 256) {
                const int j = __float_as_int(ldgf(sd));
                const float vm = ldgf(sd + 32);
                float kv[4];
#pragma unroll
                for (int k = 0; k < 4; k++) kv[k] = ldgf(sd + 64 + 32 * k);
                const float4 *gj = reinterpret_cast<const float4 *>(a.Gin + (size_t)j * G32);
                const float4 q0 = __ldg(gj), q1 = __ldg(gj + 1);
                const float2 q2 = __ldg(reinterpret_cast<const float2 *>(gj + 2));
#pragma unroll
                for (int k = 0; k < 4; k++) { kU[k] += kv[k] * q0.x; kW[k] += kv[k] * q0.y; }
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        }
        double src_u = 0.0, src_w = 0.0;
        if (i == c.src[0]) {
            const double ps = c.amp[c.it];
            src_u = ps * c.sin_af;
            src_w = ps * c.cos_af;
        }
        float g[G32], p[P32], go[G32], po[P32];
        const float4 *gi = reinterpret_cast<const float4 *>(a.Gin + (size_t)i * G32);
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const float4 v = __ldg(gi + k);
            g[4 * k] = v.x; g[4 * k + 1] = v.y; g[4 * k + 2] = v.z; g[4 * k + 3] = v.w;
        }
        const float2 *pi = reinterpret_cast<const float2 *>(a.Pin + (size_t)i * P32);
#pragma unroll
        for (int k = 0; k < 5; k++) { const float2 v = __ldg(pi + k); p[2 * k] = v.x; p[2 * k + 1] = v.y; }
        double uu, ww;
        finish_node<COMP>(kU, kW, m, c0, c1, c2, c.dt, src_u, src_w, g, p, go, po, uu, ww);
        float4 *gout = reinterpret_cast<float4 *>(a.Gout + (size_t)i * G32);
#pragma unroll
        for (int k = 0; k < 6; k++) gout[k] = make_float4(go[4 * k], go[4 * k + 1], go[4 * k + 2], go[4 * k + 3]);
        float2 *pout = reinterpret_cast<float2 *>(a.Pout + (size_t)i * P32);
#pragma unroll
        for (int k = 0; k < 5; k++) pout[k] = make_float2(po[2 * k], po[2 * k + 1]);
        eu = uu * uu;
        ew = ww * ww;
    }
    block_energy(c.energy ? c.energy + ((size_t)c.it) * 2 : nullptr, eu, ew);
}

// ------------------------------------------------ FP32 batched kernel

template <int SPL>
struct VecF;
template <> struct VecF<1> {
    float v[1];
    __device__ __forceinline__ void load(const float *p) { v[0] = __ldg(p); }
    __device__ __forceinline__ void store(float *p) const { p[0] = v[0]; }
};
template <> struct VecF<2> {
    float v[2];
    __device__ __forceinline__ void load(const float *p) { float2 t = __ldg(reinterpret_cast<const float2 *>(p)); v[0] = t.x; v[1] = t.y; }
    __device__ __forceinline__ void store(float *p) const { *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]); }
};
template <> struct VecF<4> {
    float v[4];
    __device__ __forceinline__ void load(const float *p) { float4 t = __ldg(reinterpret_cast<const float4 *>(p)); v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w; }
    __device__ __forceinline__ void store(float *p) const { *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]); }
};

// One warp per row, S = 32*SPL shots with the shot index innermost: each
// matrix entry is read once (a warp-uniform 32-byte record) and applied to
// all S shots; each lane gathers SPL consecutive shots of a neighbour's
// record with one vector load per value.  Interior rows (row-uniform
// decision) gather only U, W, Lx, Ly.
template <bool COMP, int SPL>
__global__ void __launch_bounds__(256) step32_batched_kernel(const Step32 a)
{
    constexpr int S = 32 * SPL;
    const StepCommon &c = a.c;
    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = gtid; t < c.nrec * S; t += gridDim.x * blockDim.x) gather_one32(c, a.Gin, a.Pin, S, t, c.seis_row);
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    const int s_base = lane * SPL;
    int src[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) src[q] = s_base + q < c.nshot ? c.src[s_base + q] : -1;
    const double ps = c.amp[c.it];
    const double src_u = ps * c.sin_af, src_w = ps * c.cos_af;
    float eu[SPL], ew[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) { eu[q] = 0.f; ew[q] = 0.f; }
    for (int i = gtid >> 5; i < c.n; i += warps_total) {
        const float4 *cf = reinterpret_cast<const float4 *>(a.coef) + (size_t)i * 3;
        const float4 c0 = __ldg(cf), c1 = __ldg(cf + 1), c2 = __ldg(cf + 2);
        const bool full = is_pml_row(c1);
        float kU[6][SPL], kW[6][SPL], m[20][SPL];
#pragma unroll
        for (int k = 0; k < 6; k++)
#pragma unroll
            for (int q = 0; q < SPL; q++) { kU[k][q] = 0.f; kW[k][q] = 0.f; }
#pragma unroll
        for (int k = 0; k < 20; k++)
#pragma unroll
            for (int q = 0; q < SPL; q++) m[k][q] = 0.f;
        const int e0 = __ldg(a.up + i), e1 = __ldg(a.up + i + 1);
        const float4 *rec = reinterpret_cast<const float4 *>(a.rec32);
        if (full) {
            for (int e = e0; e < e1; e++) {
                const float4 r0 = __ldg(rec + 2 * (size_t)e), r1 = __ldg(rec + 2 * (size_t)e + 1);
                const int j = __float_as_int(r0.x);
                const float vm = r0.y;
                const float kv[6] = {r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
                const float *gj = a.Gin + (size_t)j * G32 * S + s_base;
                VecF<SPL> x[22];
#pragma unroll
                for (int v = 0; v < 22; v++) x[v].load(gj + v * S);
#pragma unroll
                for (int q = 0; q < SPL; q++) {
#pragma unroll
                    for (int k = 0; k < 6; k++) { kU[k][q] += kv[k] * x[0].v[q]; kW[k][q] += kv[k] * x[1].v[q]; }
#pragma unroll
                    for (int v = 0; v < 8; v++) m[12 + v][q] += vm * x[2 + v].v[q];
#pragma unroll
                    for (int v = 0; v < 12; v++) m[v][q] += vm * x[10 + v].v[q];
                }
            }
        } else {
            for (int e = e0; e < e1; e++) {
                const float4 r0 = __ldg(rec + 2 * (size_t)e), r1 = __ldg(rec + 2 * (size_t)e + 1);
                const int j = __float_as_int(r0.x);
                const float vm = r0.y;
                const float kv[4] = {r0.z, r0.w, r1.x, r1.y};
                const float *gj = a.Gin + (size_t)j * G32 * S + s_base;
                VecF<SPL> x[10];
#pragma unroll
                for (int v = 0; v < 10; v++) x[v].load(gj + v * S);
#pragma unroll
                for (int q = 0; q < SPL; q++) {
#pragma unroll
                    for (int k = 0; k < 4; k++) { kU[k][q] += kv[k] * x[0].v[q]; kW[k][q] += kv[k] * x[1].v[q]; }
#pragma unroll
                    for (int v = 0; v < 8; v++) m[12 + v][q] += vm * x[2 + v].v[q];
                }
            }
        }
        const float *gi = a.Gin + (size_t)i * G32 * S + s_base;
        const float *pi = a.Pin + (size_t)i * P32 * S + s_base;
        float *gop = a.Gout + (size_t)i * G32 * S + s_base;
        float *pop = a.Pout + (size_t)i * P32 * S + s_base;
        VecF<SPL> gv[G32], pv[P32];
#pragma unroll
        for (int v = 0; v < G32; v++) gv[v].load(gi + v * S);
#pragma unroll
        for (int v = 0; v < P32; v++) pv[v].load(pi + v * S);
#pragma unroll
        for (int q = 0; q < SPL; q++) {
            float kUq[6], kWq[6], mq[20], g[G32], p[P32], go[G32], po[P32];
#pragma unroll
            for (int k = 0; k < 6; k++) { kUq[k] = kU[k][q]; kWq[k] = kW[k][q]; }
#pragma unroll
            for (int v = 0; v < 20; v++) mq[v] = m[v][q];
#pragma unroll
            for (int v = 0; v < G32; v++) g[v] = gv[v].v[q];
#pragma unroll
            for (int v = 0; v < P32; v++) p[v] = pv[v].v[q];
            const bool is_src = (i == src[q]);
            double uu, ww;
            finish_node<COMP>(kUq, kWq, mq, c0, c1, c2, c.dt, is_src ? src_u : 0.0, is_src ? src_w : 0.0, g, p, go,
                              po, uu, ww);
#pragma unroll
            for (int v = 0; v < G32; v++) gv[v].v[q] = go[v];
#pragma unroll
            for (int v = 0; v < P32; v++) pv[v].v[q] = po[v];
            eu[q] += (float)(uu * uu);
            ew[q] += (float)(ww * ww);
        }
#pragma unroll
        for (int v = 0; v < G32; v++) gv[v].store(gop + v * S);
#pragma unroll
        for (int v = 0; v < P32; v++) pv[v].store(pop + v * S);
    }
    // energy per shot: block reduction over warps, one atomic pair per shot
    if (c.energy) {
        __shared__ float se[8][2][32 * SPL];
        const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < SPL; q++) { se[w][0][s_base + q] = eu[q]; se[w][1][s_base + q] = ew[q]; }
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * S; t += blockDim.x) {
            int comp = t / S, s = t - comp * S;
            double acc = 0.0;
            for (int k = 0; k < nw; k++) acc += se[k][comp][s];
            if (s < c.nshot) atomicAdd(c.energy + ((size_t)s * c.nsteps + c.it) * 2 + comp, acc);
        }
    }
}

// ------------------------------------------------------- FP64 kernel

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// FP64, thread per row, the reference's operation order throughout and no
// multiply-add contraction: per-product row sums from 0.0 in column order
// (csr_matvec.c:10-16), right-hand sides as written at elastic_wave.c:585-591
// and 651-657, division by the lumped mass (:709-722), Newmark (:757-776).
__global__ void __launch_bounds__(128) step64_kernel(const Step64 a)
{
    const StepCommon &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (c.seis_row >= 0 && i < c.nrec) {
        long long node = c.rec[i];
        const double *g = a.Gin + node * GREC;
        size_t o = (size_t)c.seis_row * c.nrec + i;
        c.seis_u[o] = add(add(g[0], g[1]), g[2]);
        c.seis_w[o] = add(add(g[3], g[4]), g[5]);
    }
    double eu = 0.0, ew = 0.0;
    if (i < c.n) {
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
        const double dirichlet_or_zero = cf[8], dxxp = cf[9], dyyp = cf[10], mlump = cf[11];
        const double dt = c.dt;
        // m: 0..5 = M*U1..W3, 6..11 = M*V1..V6, 12..15 = M*Lx1..4, 16..19 = M*Ly1..4
        double r[14];
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
        const bool zero = dirichlet_or_zero == 0.0;
        double an[6], L[8];
        const int ia[6] = {0, 1, 2, 7, 8, 9};
        for (int k = 0; k < 6; k++) an[k] = zero ? 0.0 : __ddiv_rn(r[ia[k]], mlump);
        for (int k = 0; k < 4; k++) {
            L[k] = zero ? 0.0 : __ddiv_rn(r[3 + k], mlump);
            L[4 + k] = zero ? 0.0 : __ddiv_rn(r[10 + k], mlump);
        }
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
    block_energy(c.energy ? c.energy + ((size_t)c.it) * 2 : nullptr, eu, ew);
}

// ------------------------------------------------ gathers, snapshots

__global__ void gather32_kernel(const StepCommon c, const float *G, const float *P, int S)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    gather_one32(c, G, P, S, t, c.seis_row);
}

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

__global__ void snapshot32_kernel(const float *G, const float *P, int n, int S, double *su, double *sw,
                                  long long shot_stride)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * S) return;
    int s = (int)(t % S);
    long long node = t / S;
    double u = 0.0, w = 0.0;
    for (int k = 0; k < 3; k++) {
        u += (double)G[(node * G32 + 10 + k) * S + s] + (double)P[(node * P32 + 4 + k) * S + s];
        w += (double)G[(node * G32 + 13 + k) * S + s] + (double)P[(node * P32 + 7 + k) * S + s];
    }
    su[s * shot_stride + node] = u;
    sw[s * shot_stride + node] = w;
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

__global__ void slice_len_kernel(int n, const int *__restrict__ up, int *len)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int nsl = (n + 31) / 32;
    if (s >= nsl) return;
    int m = 0;
    for (int l = 0; l < 32; l++) {
        int r = s * 32 + l;
        if (r < n) m = max(m, up[r + 1] - up[r]);
    }
    len[s] = m;
}

__global__ void sell_fill_kernel(int n, const int *__restrict__ up, const int *__restrict__ uj,
                                 const double *__restrict__ ux, long long nnz, const int *__restrict__ sp,
                                 float *__restrict__ sell)
{
    int s = blockIdx.x;
    int lane = threadIdx.x;
    int r = s * 32 + lane;
    int s0 = sp[s], s1 = sp[s + 1];
    int a0 = r < n ? up[r] : 0, len = r < n ? up[r + 1] - a0 : 0;
    for (int k = 0; k < s1 - s0; k++) {
        float *slot = sell + (size_t)(s0 + k) * 256;
        if (k < len) {
            long long e = a0 + k;
            slot[lane] = __int_as_float(uj[e]);
            for (int m = 0; m < 7; m++) slot[32 * (m + 1) + lane] = (float)ux[m * nnz + e];
        } else {
            // padding: the row itself with zero weights (a valid, cached address)
            slot[lane] = __int_as_float(r < n ? r : 0);
            for (int m = 0; m < 7; m++) slot[32 * (m + 1) + lane] = 0.f;
        }
    }
}

__global__ void rec_fill_kernel(long long nnz, const int *__restrict__ uj, const double *__restrict__ ux,
                                float *__restrict__ rec)
{
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    rec[e * 8] = __int_as_float(uj[e]);
    for (int m = 0; m < 7; m++) rec[e * 8 + 1 + m] = (float)ux[m * nnz + e];
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

cudaError_t launch_step32(const Step32 &a, bool kahan, int threads, cudaStream_t st)
{
    int blocks = (a.c.n + threads - 1) / threads;
    if (kahan) step32_kernel<true><<<blocks, threads, 0, st>>>(a);
    else step32_kernel<false><<<blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_step64(const Step64 &a, int threads, cudaStream_t st)
{
    int blocks = (a.c.n + threads - 1) / threads;
    step64_kernel<<<blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_step32_batched(const Step32 &a, bool kahan, int spl, int warps, cudaStream_t st)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int threads = 32 * warps;
    int per_sm = 0;
    if (kahan) {
        if (spl == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<true, 1>, threads, 0);
        else if (spl == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<true, 2>, threads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<true, 4>, threads, 0);
    } else {
        if (spl == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<false, 1>, threads, 0);
        else if (spl == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<false, 2>, threads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step32_batched_kernel<false, 4>, threads, 0);
    }
    if (per_sm < 1) per_sm = 1;
    long long need = ((long long)a.c.n + warps - 1) / warps;
    long long blocks = std::min<long long>((long long)sms * per_sm, need);
    if (blocks < 1) blocks = 1;
#define SFG_BATCH(K, P) step32_batched_kernel<K, P><<<(unsigned)blocks, threads, 0, st>>>(a)
    if (kahan) { if (spl == 1) SFG_BATCH(true, 1); else if (spl == 2) SFG_BATCH(true, 2); else SFG_BATCH(true, 4); }
    else { if (spl == 1) SFG_BATCH(false, 1); else if (spl == 2) SFG_BATCH(false, 2); else SFG_BATCH(false, 4); }
#undef SFG_BATCH
    return cudaGetLastError();
}

cudaError_t launch_gather32(const StepCommon &c, const float *G, const float *P, int S, cudaStream_t st)
{
    int tot = c.nrec * S;
    if (tot > 0 && c.seis_row >= 0) gather32_kernel<<<(tot + 127) / 128, 128, 0, st>>>(c, G, P, S);
    return cudaGetLastError();
}

cudaError_t launch_gather64(const StepCommon &c, const double *G, int S, cudaStream_t st)
{
    (void)S;
    if (c.nrec > 0 && c.seis_row >= 0) gather64_kernel<<<(c.nrec + 127) / 128, 128, 0, st>>>(c, G);
    return cudaGetLastError();
}

cudaError_t launch_snapshot32(const float *G, const float *P, int n, int S, double *su, double *sw,
                              long long shot_stride, cudaStream_t st)
{
    long long tot = (long long)n * S;
    snapshot32_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(G, P, n, S, su, sw, shot_stride);
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

cudaError_t build_sell32(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                         float **d_sell, int **d_slice_ptr, long long *slots, cudaStream_t st)
{
    int nsl = (n + 31) / 32;
    int *len = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&len, sizeof(int) * ((size_t)nsl + 1))) != cudaSuccess) return e;
    if ((e = cudaMalloc(d_slice_ptr, sizeof(int) * ((size_t)nsl + 1))) != cudaSuccess) return e;
    slice_len_kernel<<<(nsl + 127) / 128, 128, 0, st>>>(n, d_up, len);
    if ((e = exclusive_scan_int(len, *d_slice_ptr, nsl, st)) != cudaSuccess) return e;
    int tot = 0;
    cudaMemcpyAsync(&tot, *d_slice_ptr + nsl, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *slots = tot;
    if ((e = cudaMalloc(d_sell, sizeof(float) * 256 * std::max<size_t>(tot, 1))) != cudaSuccess) return e;
    if (nsl) sell_fill_kernel<<<nsl, 32, 0, st>>>(n, d_up, d_uj, d_ux, nnz, *d_slice_ptr, *d_sell);
    e = cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaFree(len);
    return e;
}

cudaError_t build_rec32(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                        float **d_rec, cudaStream_t st)
{
    (void)n; (void)d_up;
    cudaError_t e = cudaMalloc(d_rec, sizeof(float) * 8 * std::max<long long>(nnz, 1));
    if (e != cudaSuccess) return e;
    if (nnz) rec_fill_kernel<<<(unsigned)((nnz + 255) / 256), 256, 0, st>>>(nnz, d_uj, d_ux, *d_rec);
    return cudaGetLastError();
}

cudaError_t build_coef(int n, const double *d_c, const double *d_mpml, const double *d_mass,
                       const unsigned char *d_dir, float **d_coef32, double **d_coef64, cudaStream_t st)
{
    cudaError_t e;
    if ((e = cudaMalloc(d_coef32, sizeof(float) * CREC * std::max(n, 1))) != cudaSuccess) return e;
    if ((e = cudaMalloc(d_coef64, sizeof(double) * CREC * std::max(n, 1))) != cudaSuccess) return e;
    coef_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, d_c, d_mpml, d_mass, d_dir, *d_coef32, *d_coef64);
    return cudaGetLastError();
}

}  // namespace sfg
