// sfg_step32.cu -- fused FP32 time step (time_evolution/elastic_wave.c:519-809)
// in the two-class layout described in sfg_step32.cuh.
//
// One launch per class and step: the class-A kernel (interior rows: totals
// only, 16 products per row: K1..K4 times U and W, M times Lx1..4, Ly1..4)
// and the class-Z kernel (split zone: all 32 products on M-PML rows) read the
// step's input records and write the output records of their own rows, so
// the two run concurrently.  Each streams its rows' SELL-32 slices once,
// gathers each neighbour record once, keeps every product in registers and
// finishes the node (right-hand sides elastic_wave.c:585-591 / 651-657,
// lumped solve :709-722, Newmark :757-776) in the same thread.  The SpMV
// products and the per-node epilogue run in FP32; the compensated precision
// keeps every displacement as an FP32 hi + lo pair updated with a Kahan sum,
// and forms the class-Z totals U1+U2+U3, W1+W2+W3 from those pairs in FP64.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "sfg_dev.cuh"
#include "sfg_internal.h"
#include "sfg_step32.cuh"

namespace sfg {

namespace {

__device__ __forceinline__ float ldgf(const float *p) { return __ldg(p); }

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

// --------------------------------------------------------------- epilogues

// Newmark, alpha = 1, delta = 1.5 (elastic_wave.c:97, 757-768) for one
// displacement carried as hi + lo: the step's increment is added with a
// compensated (Kahan) sum in FP32, so the rounding error of the running
// displacement does not build up over the steps.  Returns hi + lo.
__device__ __forceinline__ float newmark_kahan(float &hi, float &lo, float &V, float &A, float an, float dt)
{
    const float d = V * dt + (an - 0.5f * A) * (dt * dt);
    const float y = d + lo;
    const float t = hi + y;
    lo = y - (t - hi);
    hi = t;
    V = V + (1.5f * an - 0.5f * A) * dt;
    A = an;
    return t + lo;
}

__device__ __forceinline__ float newmark_plain(float &U, float &V, float &A, float an, float dt)
{
    U = U + V * dt + (an - 0.5f * A) * (dt * dt);
    V = V + (1.5f * an - 0.5f * A) * dt;
    A = an;
    return U;
}

// Stiffness part of the class-A right-hand sides from the products kU, kW
// (K1..K4 times U, W) and the row's c11 c13 c33 c44 (elastic_wave.c:585-591,
// 651-657 with the damping terms zero).
__device__ __forceinline__ void stiff_sums(const float *kU, const float *kW, float4 c, float &su, float &sw)
{
    su = -c.x * kU[0] - c.w * kU[1] - c.y * kW[2] - c.w * kW[3];
    sw = -c.w * kW[0] - c.z * kW[1] - c.w * kU[2] - c.y * kU[3];
}

// Class A: the summed right-hand sides of the three split fields with
// dx = dy = dxx = dyy = 0:  a_u = (rhs_u1 + rhs_u2 + rhs_u3) / m,
// a_w = (rhs_w1 + rhs_w2 + rhs_w3) / m, and L_k = (M L_k) / m.
// su, sw: the stiffness sums (stiff_sums, or accumulated from folded
// records); mL: M times Lx1..4, Ly1..4.
// g[12]: own Gc record, p[4]: own Pa record, replaced by the new records.
template <bool COMP>
__device__ __forceinline__ void finish_A(float su, float sw, const float *mL, float im, double dt, double src_u,
                                         double src_w, float *g, float *p, float &uu, float &ww)
{
    float Uh = g[0], Wh = g[1], lou = g[10], low = g[11];
    float Au = p[0], Aw = p[1], Vu = p[2], Vw = p[3];
    const float au = im * (su + ((mL[0] + mL[1]) + (mL[2] + mL[3])) + (float)src_u);
    const float aw = im * (sw + ((mL[4] + mL[5]) + (mL[6] + mL[7])) + (float)src_w);
    if (COMP) {
        uu = newmark_kahan(Uh, lou, Vu, Au, au, (float)dt);
        ww = newmark_kahan(Wh, low, Vw, Aw, aw, (float)dt);
    } else {
        uu = newmark_plain(Uh, Vu, Au, au, (float)dt);
        ww = newmark_plain(Wh, Vw, Aw, aw, (float)dt);
        lou = 0.f;
        low = 0.f;
    }
    g[0] = Uh;
    g[1] = Wh;
#pragma unroll
    for (int k = 0; k < 8; k++) g[2 + k] = im * mL[k];
    g[10] = lou;
    g[11] = low;
    p[0] = Au; p[1] = Aw; p[2] = Vu; p[3] = Vw;
}

template <typename T>
struct RhsT {
    T a[6];          // accelerations of U1 U2 U3 W1 W2 W3
    T lx[4], ly[4];  // new memory variables
};

// Split right-hand sides (elastic_wave.c:585-591, 651-657) times 1/m_lump,
// from the FP32 products: kU[k], kW[k] = K_{k+1} times U, W; m[0..19] = M
// times U1..W3, V1..V6, Lx1..4, Ly1..4.
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

// Class Z: split fields.  gs[12] / ps[12]: own Gs / Ps records (replaced);
// gc[12] receives the new Gc record (totals, memory variables).
template <bool COMP>
__device__ __forceinline__ void finish_Z(const float *kU, const float *kW, const float *m, float4 c0, float4 c1,
                                         float4 c2, double dt, double src_u, double src_w, float *gs, float *ps,
                                         float *gc, float &uu, float &ww)
{
    float L[8];
    RhsT<float> r;
    rhs_eval<float>(kU, kW, m, c0, c1, c2, (float)dt, (float)src_u, (float)src_w, r);
    float su, sw;
    if (COMP) {
#pragma unroll
        for (int k = 0; k < 6; k++) newmark_kahan(gs[k], ps[6 + k], gs[6 + k], ps[k], r.a[k], (float)dt);
        // the totals from the compensated split fields (each hi + lo) in FP64:
        // inside the M-PML the split fields are far larger than their sum
        const double su64 = (((double)gs[0] + ps[6]) + ((double)gs[1] + ps[7])) + ((double)gs[2] + ps[8]);
        const double sw64 = (((double)gs[3] + ps[9]) + ((double)gs[4] + ps[10])) + ((double)gs[5] + ps[11]);
        su = (float)su64;
        sw = (float)sw64;
        gc[10] = (float)(su64 - (double)su);
        gc[11] = (float)(sw64 - (double)sw);
    } else {
        float Ut[6];
#pragma unroll
        for (int k = 0; k < 6; k++) { Ut[k] = newmark_plain(gs[k], gs[6 + k], ps[k], r.a[k], (float)dt); ps[6 + k] = 0.f; }
        su = (Ut[0] + Ut[1]) + Ut[2];
        sw = (Ut[3] + Ut[4]) + Ut[5];
        gc[10] = 0.f;
        gc[11] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) { L[k] = r.lx[k]; L[4 + k] = r.ly[k]; }
    uu = su;
    ww = sw;
    gc[0] = su;
    gc[1] = sw;
#pragma unroll
    for (int k = 0; k < 8; k++) gc[2 + k] = L[k];
}

__device__ __forceinline__ bool is_pml_row(float4 c1)
{
    return c1.x != 0.f || c1.y != 0.f || c1.z != 0.f || c1.w != 0.f;
}

// Displacement of permuted row `node` of shot `s` in a finished state:
// class A: hi + lo of the totals; class Z: sum of the split pairs (FP64).
// Value k of row r's 12-float record in a state array: the one-shot block
// layout (blk4) when S = 1, else [row][value][S].
__device__ __forceinline__ double rec_val(const float *base, long long r, int k, int S, int s)
{
    return (double)(S == 1 ? base[4 * blk4(r, k >> 2, 3) + (k & 3)] : base[(r * 12 + k) * S + s]);
}

__device__ __forceinline__ void total_uw(const State32 &st, int na, int S, long long node, int s, double &u, double &w)
{
    if (node < na) {
        u = rec_val(st.Gc, node, 0, S, s) + rec_val(st.Gc, node, 10, S, s);
        w = rec_val(st.Gc, node, 1, S, s) + rec_val(st.Gc, node, 11, S, s);
    } else {
        const long long z = node - na;
        u = 0.0;
        w = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            u += rec_val(st.Gs, z, k, S, s) + rec_val(st.Ps, z, 6 + k, S, s);
            w += rec_val(st.Gs, z, 3 + k, S, s) + rec_val(st.Ps, z, 9 + k, S, s);
        }
    }
}

// Receiver gather (elastic_wave.c:787-795) of the step's input state.
__device__ __forceinline__ void gather2_one(const StepCommon &c, int na, const State32 &st, int S, int t,
                                            int seis_row)
{
    if (seis_row < 0 || t >= c.nrec * S) return;
    const int s = t / c.nrec, r = t - s * c.nrec;
    double u, w;
    total_uw(st, na, S, c.rec[r], s, u, w);
    const size_t o = ((size_t)s * c.seis_rows + seis_row) * c.nrec + r;
    c.seis_u[o] = u;
    c.seis_w[o] = w;
}

// ------------------------------------------------- single-shot kernels

// The (column, tuple id) slots of one row in a SELL-32 slice, read two slots
// ahead of use: their stream latency then overlaps the gathers of the slots
// in hand instead of preceding them.  Streams that no other row reads (slots,
// coefficients, private state) load with the evict-first hint (ld.global.cs),
// leaving L1 to the neighbour gathers.
struct DictSlots {
    const int2 *p;
    int left;
    int2 s0, s1;
    __device__ __forceinline__ void init(const int2 *base, int n)
    {
        p = base;
        left = n;
        s0 = n > 0 ? __ldcs(p) : make_int2(0, 0);
        s1 = n > 1 ? __ldcs(p + 32) : make_int2(0, 0);
        p += 64;
    }
    __device__ __forceinline__ int2 next()
    {
        const int2 r = s0;
        s0 = s1;
        s1 = left > 2 ? __ldcs(p) : make_int2(0, 0);
        p += 32;
        left--;
        return r;
    }
};

// The same with three slot rows in flight: the class-A loop (unrolled by
// three) keeps one more slot load outstanding per thread, which its
// register budget allows and class Z's does not.
struct DictSlots3 {
    const int2 *p;
    int left;
    int2 s0, s1, s2;
    __device__ __forceinline__ void init(const int2 *base, int n)
    {
        p = base;
        left = n;
        s0 = n > 0 ? __ldcs(p) : make_int2(0, 0);
        s1 = n > 1 ? __ldcs(p + 32) : make_int2(0, 0);
        s2 = n > 2 ? __ldcs(p + 64) : make_int2(0, 0);
        p += 96;
    }
    __device__ __forceinline__ int2 next()
    {
        const int2 r = s0;
        s0 = s1;
        s1 = s2;
        s2 = left > 3 ? __ldcs(p) : make_int2(0, 0);
        p += 32;
        left--;
        return r;
    }
};

// the dictionary's tuples into shared memory (2 float4 each)
template <int THREADS>
__device__ __forceinline__ void load_dict(const Step2 &a, float4 *stab)
{
    for (int t = threadIdx.x; t < 2 * a.dict_n; t += THREADS) stab[t] = __ldg(a.dict + t);
    __syncthreads();
}

// Class-A rows of block `bid` of one mesh (the tuples already in stab).
template <bool COMP, int THREADS, bool DICT, bool STG = false>
__device__ __forceinline__ void stepA_body(const Step2 &a, int bid, const float4 *stab, int it, int seis_row,
                                           const int2 *stg = nullptr, int slb = 0)
{
    const StepCommon &c = a.c;
    const int i = bid * THREADS + threadIdx.x;
    gather2_one(c, a.na, a.in, 1, i, seis_row);
    float eu = 0.f, ew = 0.f;
    if (i < a.na) {
        const int lane = i & 31, slice = i >> 5;
        float kU[4], kW[4], mL[8];
#pragma unroll
        for (int k = 0; k < 4; k++) { kU[k] = 0.f; kW[k] = 0.f; }
#pragma unroll
        for (int k = 0; k < 8; k++) mL[k] = 0.f;
        const int s0 = __ldg(a.sliceA + slice), s1 = __ldg(a.sliceA + slice + 1);
        if (DICT && !STG && lane == 0) {
            // the slice's slot rows and the private streams of its rows (read
            // once, after the gathers) into L2 ahead of use: the whole slice
            // is in flight at once instead of the two slot rows the registers
            // hold
            const int r0 = slice * 32, nr = min(32, a.na - r0);
            prefetch_l2(a.sellAd + (size_t)s0 * 32, (unsigned)(s1 - s0) * 256u);
            prefetch_l2(reinterpret_cast<const float4 *>(a.in.Pa) + r0, 16u * nr);
            prefetch_l2(a.coefA + r0, 16u * nr);
            prefetch_l2(a.imA + r0, (4u * nr) & ~15u);
            prefetch_l2(a.rowrho + r0, (4u * nr) & ~15u);
        }
        // own displacements (hi, lo): every row of K1..K6 sums to zero, so
        // K U = sum_j K_ij (U_j - U_i), and the differences of the hi and lo
        // parts keep the products free of the cancellation that FP32 sums
        // of K_ij U_j suffer on smooth fields
        const float4 *G4 = reinterpret_cast<const float4 *>(a.in.Gc);
        const float4 own0 = __ldg(G4 + blk4(i, 0, 3)), own2 = __ldg(G4 + blk4(i, 2, 3));
        // the values the row's update reads after the slot loop, into L1
        prefetch_l1(G4 + blk4(i, 1, 3));
        prefetch_l1(reinterpret_cast<const float4 *>(a.in.Pa) + i);
        prefetch_l1(a.coefA + i);
        prefetch_l1(a.imA + i);
        if (DICT) prefetch_l1(a.rowrho + i);
        // jq: the float4 index blk4(j, 0, 3) of neighbour j's record
        auto acc = [&](int jq, float vm, const float *kv) {
            const float4 *gj = G4 + jq;
            const float4 q0 = __ldg(gj), q1 = __ldg(gj + 32), q2 = __ldg(gj + 64);
            const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
#pragma unroll
            for (int k = 0; k < 4; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
            mL[0] += vm * q0.z; mL[1] += vm * q0.w; mL[2] += vm * q1.x; mL[3] += vm * q1.y;
            mL[4] += vm * q1.z; mL[5] += vm * q1.w; mL[6] += vm * q2.x; mL[7] += vm * q2.y;
        };
        if (DICT) {
            DictSlots3 ss;
            if (!STG) ss.init(a.sellAd + (size_t)s0 * 32 + lane, s1 - s0);
#pragma unroll 3
            for (int g = s0; g < s1; ++g) {
                const int2 cv = STG ? stg[(g - slb) * 32 + lane] : ss.next();
                const float4 t0 = stab[cv.y], t1 = stab[cv.y + 1];
                const float kv[4] = {t0.y, t0.z, t0.w, t1.x};
                acc(cv.x, t0.x, kv);
            }
            const float rho = __ldcs(a.rowrho + i);
#pragma unroll
            for (int k = 0; k < 8; k++) mL[k] *= rho;
        } else {
            const float *sd = a.sellA + (size_t)s0 * 192 + lane;
#pragma unroll 3
            for (int g = s0; g < s1; ++g, sd += 192) {
                float kv[4];
#pragma unroll
                for (int k = 0; k < 4; k++) kv[k] = ldgf(sd + 64 + 32 * k);
                acc((int)blk4(__float_as_int(ldgf(sd)), 0, 3), ldgf(sd + 32), kv);
            }
        }
        const float4 cf = __ldcs(a.coefA + i);
        const float im = __ldcs(a.imA + i);
        double src_u = 0.0, src_w = 0.0;
        if (i == c.src[0]) {
            const double ps = c.amp[it];
            src_u = ps * c.sin_af;
            src_w = ps * c.cos_af;
        }
        float g[GC], p[PA];
        const float4 own1 = __ldg(G4 + blk4(i, 1, 3));
        g[0] = own0.x; g[1] = own0.y; g[2] = own0.z; g[3] = own0.w;
        g[4] = own1.x; g[5] = own1.y; g[6] = own1.z; g[7] = own1.w;
        g[8] = own2.x; g[9] = own2.y; g[10] = own2.z; g[11] = own2.w;
        const float4 pv = __ldcs(reinterpret_cast<const float4 *>(a.in.Pa) + i);
        p[0] = pv.x; p[1] = pv.y; p[2] = pv.z; p[3] = pv.w;
        float uu, ww, su, sw;
        stiff_sums(kU, kW, cf, su, sw);
        finish_A<COMP>(su, sw, mL, im, c.dt, src_u, src_w, g, p, uu, ww);
        float4 *go = reinterpret_cast<float4 *>(a.out.Gc) + blk4(i, 0, 3);
#pragma unroll
        for (int k = 0; k < 3; k++) go[32 * k] = make_float4(g[4 * k], g[4 * k + 1], g[4 * k + 2], g[4 * k + 3]);
        reinterpret_cast<float4 *>(a.out.Pa)[i] = make_float4(p[0], p[1], p[2], p[3]);
        eu = uu * uu;
        ew = ww * ww;
    }
    block_energy(c.energy ? c.energy + ((size_t)it) * 2 : nullptr, eu, ew);
}

template <bool COMP, int THREADS, int MINB, bool DICT>
__global__ void __launch_bounds__(THREADS, MINB) stepA_kernel(const Step2 a)
{
    extern __shared__ float4 stab[];
    if (DICT) load_dict<THREADS>(a, stab);
    stepA_body<COMP, THREADS, DICT>(a, blockIdx.x, stab, a.c.it, a.c.seis_row);
}

// Class-Z rows of block `bid` of one mesh (the tuples already in stab).
template <bool COMP, int THREADS, bool DICT, bool STG = false>
__device__ __forceinline__ void stepZ_body(const Step2 &a, int bid, const float4 *stab, int it,
                                           const int2 *stg = nullptr, int slb = 0)
{
    const StepCommon &c = a.c;
    const int nz = c.n - a.na;
    const int local = bid * THREADS + threadIdx.x;
    const int i = a.na + local;
    float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0, c2 = c0;
    if (local < nz) {
        const float4 *cf = reinterpret_cast<const float4 *>(a.coefZ) + blk4(local, 0, 3);
        c0 = __ldcs(cf); c1 = __ldcs(cf + 32); c2 = __ldcs(cf + 64);
    }
    const bool full = __any_sync(0xffffffffu, local < nz && is_pml_row(c1));
    float eu = 0.f, ew = 0.f;
    if (local < nz) {
        const int lane = local & 31, slice = local >> 5;
        float kU[6], kW[6], m[20];
#pragma unroll
        for (int k = 0; k < 6; k++) { kU[k] = 0.f; kW[k] = 0.f; }
#pragma unroll
        for (int k = 0; k < 20; k++) m[k] = 0.f;
        const int s0 = __ldg(a.sliceZ + slice), s1 = __ldg(a.sliceZ + slice + 1);
        if (DICT && !STG && lane == 0) {
            // the slice's slot rows and its rows' private records into L2
            const int r0 = slice * 32;
            prefetch_l2(a.sellZd + (size_t)s0 * 32, (unsigned)(s1 - s0) * 256u);
            prefetch_l2(reinterpret_cast<const float4 *>(a.in.Ps) + blk4(r0, 0, 3), 1536u);
            prefetch_l2(reinterpret_cast<const float4 *>(a.in.Gs) + blk4(r0, 0, 3), 1536u);
        }
        // own totals (hi, lo) for the stiffness products in difference form
        const float4 *G4 = reinterpret_cast<const float4 *>(a.in.Gc);
        const float4 *S4 = reinterpret_cast<const float4 *>(a.in.Gs);
        const float4 own0 = __ldg(G4 + blk4(i, 0, 3)), own2 = __ldg(G4 + blk4(i, 2, 3));
        const float *sd = DICT ? nullptr : a.sellZ + (size_t)s0 * 256 + lane;
        DictSlots ss;
        if (DICT && !STG) ss.init(a.sellZd + (size_t)s0 * 32 + lane, s1 - s0);
        int gs_next = s0 - slb;   // staged slots: the next slot row in shared memory
        // slot g's record index jq = blk4(column, 0, 3), M and K1..K(NK): from
        // the dictionary or the full-value planes.  With na a multiple of 32,
        // a class-Z column's split-field record is Gs float4 jq - 3 na.
        const int zq = 3 * a.na;
        auto slot = [&](int &j, float &vm, float *kv, int nk) {
            if (DICT) {
                const int2 cv = STG ? stg[(gs_next++) * 32 + lane] : ss.next();
                const float4 t0 = stab[cv.y], t1 = stab[cv.y + 1];
                j = cv.x;
                vm = t0.x;
                kv[0] = t0.y; kv[1] = t0.z; kv[2] = t0.w; kv[3] = t1.x;
                if (nk == 6) { kv[4] = t1.y; kv[5] = t1.z; }
            } else {
                j = (int)blk4(__float_as_int(ldgf(sd)), 0, 3);
                vm = ldgf(sd + 32);
                for (int k = 0; k < nk; k++) kv[k] = ldgf(sd + 64 + 32 * k);
                sd += 256;
            }
        };
        if (full) {
#pragma unroll 1
            for (int g = s0; g < s1; ++g) {
                int j;
                float vm, kv[6];
                slot(j, vm, kv, 6);
                const float4 *gj = G4 + j;
                const float4 q0 = __ldg(gj), q1 = __ldg(gj + 32), q2 = __ldg(gj + 64);
                const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
                // split fields exist for class-Z columns; rows outside the
                // M-PML that share the warp see zeros for class-A columns (their
                // damping coefficients are zero, so those products are unused)
                float4 z0 = make_float4(0.f, 0.f, 0.f, 0.f), z1 = z0, z2 = z0;
                if (j >= zq) {
                    const float4 *sj = S4 + (j - zq);
                    z0 = __ldg(sj); z1 = __ldg(sj + 32); z2 = __ldg(sj + 64);
                }
#pragma unroll
                for (int k = 0; k < 6; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
                m[0] += vm * z0.x;  m[1] += vm * z0.y;  m[2] += vm * z0.z;  m[3] += vm * z0.w;
                m[4] += vm * z1.x;  m[5] += vm * z1.y;  m[6] += vm * z1.z;  m[7] += vm * z1.w;
                m[8] += vm * z2.x;  m[9] += vm * z2.y;  m[10] += vm * z2.z; m[11] += vm * z2.w;
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        } else {
#pragma unroll 1
            for (int g = s0; g < s1; ++g) {
                int j;
                float vm, kv[4];
                slot(j, vm, kv, 4);
                const float4 *gj = G4 + j;
                const float4 q0 = __ldg(gj), q1 = __ldg(gj + 32), q2 = __ldg(gj + 64);
                const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
#pragma unroll
                for (int k = 0; k < 4; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        }
        if (DICT) {
            const float rho = __ldcs(a.rowrho + i);
#pragma unroll
            for (int k = 0; k < 20; k++) m[k] *= rho;
        }
        double src_u = 0.0, src_w = 0.0;
        if (i == c.src[0]) {
            const double ps = c.amp[it];
            src_u = ps * c.sin_af;
            src_w = ps * c.cos_af;
        }
        float gs[GS], ps_[PS], gc[GC];
        const float4 *si = S4 + blk4(local, 0, 3);
        const float4 *pi = reinterpret_cast<const float4 *>(a.in.Ps) + blk4(local, 0, 3);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float4 v = __ldg(si + 32 * k), w = __ldcs(pi + 32 * k);
            gs[4 * k] = v.x; gs[4 * k + 1] = v.y; gs[4 * k + 2] = v.z; gs[4 * k + 3] = v.w;
            ps_[4 * k] = w.x; ps_[4 * k + 1] = w.y; ps_[4 * k + 2] = w.z; ps_[4 * k + 3] = w.w;
        }
        float uu, ww;
        finish_Z<COMP>(kU, kW, m, c0, c1, c2, c.dt, src_u, src_w, gs, ps_, gc, uu, ww);
        float4 *gco = reinterpret_cast<float4 *>(a.out.Gc) + blk4(i, 0, 3);
        float4 *so = reinterpret_cast<float4 *>(a.out.Gs) + blk4(local, 0, 3);
        float4 *po = reinterpret_cast<float4 *>(a.out.Ps) + blk4(local, 0, 3);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            gco[32 * k] = make_float4(gc[4 * k], gc[4 * k + 1], gc[4 * k + 2], gc[4 * k + 3]);
            so[32 * k] = make_float4(gs[4 * k], gs[4 * k + 1], gs[4 * k + 2], gs[4 * k + 3]);
            po[32 * k] = make_float4(ps_[4 * k], ps_[4 * k + 1], ps_[4 * k + 2], ps_[4 * k + 3]);
        }
        eu = uu * uu;
        ew = ww * ww;
    }
    block_energy(c.energy ? c.energy + ((size_t)it) * 2 : nullptr, eu, ew);
}

template <bool COMP, int THREADS, int MINB, bool DICT>
__global__ void __launch_bounds__(THREADS, MINB) stepZ_kernel(const Step2 a)
{
    extern __shared__ float4 stab[];
    if (DICT) load_dict<THREADS>(a, stab);
    stepZ_body<COMP, THREADS, DICT>(a, blockIdx.x, stab, a.c.it);
}

// The one-shot kernels with the tuple table in their parameters, which live
// in the constant bank (__grid_constant__: read in place, never copied): a
// warp whose lanes read one tuple -- most slot rows of a structured mesh --
// is served by one constant-cache broadcast instead of shared-memory
// wavefronts on the L1 data pipe, which the neighbour gathers keep busy
// (config 2: 59.1 -> 57.2 us per step).  Meshes with more tuples keep the
// table in shared memory.
struct Step2T {
    Step2 a;
    float4 tab[2 * kParamTuples];
};

template <bool COMP, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) stepA_kernel_ct(const __grid_constant__ Step2T p)
{
    stepA_body<COMP, THREADS, true>(p.a, blockIdx.x, p.tab, p.a.c.it, p.a.c.seis_row);
}

template <bool COMP, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) stepZ_kernel_ct(const __grid_constant__ Step2T p)
{
    stepZ_body<COMP, THREADS, true>(p.a, blockIdx.x, p.tab, p.a.c.it);
}

// ------------------------------------------------ several meshes per launch
//
// One launch per class and time step for a group of independent one-shot
// problems (meshes of different sizes): block b works on block map[b].y of
// mesh map[b].x and reads that mesh's step descriptor (the in/out state of
// this step's parity) in place; `it` gives the time index and receiver row,
// which the per-mesh launches carry in their descriptors.

template <bool COMP, int THREADS, int MINB, bool DICT>
__global__ void __launch_bounds__(THREADS, MINB) stepA_multi(const Step2 *__restrict__ descs,
                                                             const int2 *__restrict__ map, int it)
{
    extern __shared__ float4 stab[];
    const int2 mb = __ldg(map + blockIdx.x);
    const Step2 &a = descs[mb.x];
    if (DICT) load_dict<THREADS>(a, stab);
    stepA_body<COMP, THREADS, DICT>(a, mb.y, stab, it, it >= 3 ? it - 3 : -1);
}

template <bool COMP, int THREADS, int MINB, bool DICT>
__global__ void __launch_bounds__(THREADS, MINB) stepZ_multi(const Step2 *__restrict__ descs,
                                                             const int2 *__restrict__ map, int it)
{
    extern __shared__ float4 stab[];
    const int2 mb = __ldg(map + blockIdx.x);
    const Step2 &a = descs[mb.x];
    if (DICT) load_dict<THREADS>(a, stab);
    stepZ_body<COMP, THREADS, DICT>(a, mb.y, stab, it);
}

// --------------------------------------------------------- batched kernels

// Per-shot energies: each block sums its rows in shared memory, then adds
// one pair per shot to the step's global sums.
__device__ __forceinline__ void energy_zero(float *se, int S)
{
    for (int t = threadIdx.x; t < 2 * S; t += blockDim.x) se[t] = 0.f;
    __syncthreads();
}

template <int SPL>
__device__ __forceinline__ void energy_flush(const StepCommon &c, float *se, int S, int s_base, const float *eu,
                                             const float *ew)
{
#pragma unroll
    for (int q = 0; q < SPL; q++) {
        if (eu[q] != 0.f) atomicAdd(se + s_base + q, eu[q]);
        if (ew[q] != 0.f) atomicAdd(se + S + s_base + q, ew[q]);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * S; t += blockDim.x) {
        const int comp = t / S, s = t - comp * S;
        const float v = se[t];
        if (s < c.nshot && v != 0.f) atomicAdd(c.energy + ((size_t)s * c.nsteps + c.it) * 2 + comp, (double)v);
    }
}

// Batched kernels: S shots with the shot index innermost ([node][value][S]).
// A warp advances one row for a chunk of 32*SPL shots (SPL per lane); the
// S/(32*SPL) chunks of a row go to neighbouring warps of the same block, so
// the row's matrix records and its neighbours' state are shared through L1.
// The grid is persistent and its warp count a multiple of the chunk count,
// so every warp keeps one chunk.  The row's records (column + matrix values,
// 32 B) are loaded once per warp, one per lane, and broadcast with shuffles;
// neighbour records of two entries are loaded before either is applied.
struct Entry {
    int j;
    float vm, k[6];
};

template <int NK>
__device__ __forceinline__ Entry entry_at(const float4 &r0, const float4 &r1, int k)
{
    Entry e;
    e.j = __shfl_sync(0xffffffffu, __float_as_int(r0.x), k);
    e.vm = __shfl_sync(0xffffffffu, r0.y, k);
    e.k[0] = __shfl_sync(0xffffffffu, r0.z, k);
    e.k[1] = __shfl_sync(0xffffffffu, r0.w, k);
    e.k[2] = __shfl_sync(0xffffffffu, r1.x, k);
    e.k[3] = __shfl_sync(0xffffffffu, r1.y, k);
    if (NK == 6) {
        e.k[4] = __shfl_sync(0xffffffffu, r1.z, k);
        e.k[5] = __shfl_sync(0xffffffffu, r1.w, k);
    }
    return e;
}

// acc[q] += a * x[q] for the lane's shots; pairs of shots use the packed
// FP32x2 FMA of sm_100 (one instruction per two shots, same rounding as two
// fused multiply-adds).
template <int SPL>
__device__ __forceinline__ void axpy(float *acc, float a, const VecF<SPL> &x)
{
    if constexpr (SPL == 1) {
        acc[0] = fmaf(a, x.v[0], acc[0]);
    } else {
        const float2 aa = make_float2(a, a);
        const unsigned long long av = *reinterpret_cast<const unsigned long long *>(&aa);
#pragma unroll
        for (int q = 0; q < SPL; q += 2) {
            float2 c = make_float2(acc[q], acc[q + 1]);
            const float2 b = make_float2(x.v[q], x.v[q + 1]);
            unsigned long long cv = *reinterpret_cast<unsigned long long *>(&c);
            const unsigned long long bv = *reinterpret_cast<const unsigned long long *>(&b);
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(cv) : "l"(av), "l"(bv));
            c = *reinterpret_cast<float2 *>(&cv);
            acc[q] = c.x;
            acc[q + 1] = c.y;
        }
    }
}

// K1..K4 times U, W and M times Lx1..4, Ly1..4 of one neighbour record x[10].
template <int SPL>
__device__ __forceinline__ void acc_totals(const Entry &e, const VecF<SPL> *x, float (*kU)[SPL], float (*kW)[SPL],
                                           float (*mL)[SPL])
{
#pragma unroll
    for (int t = 0; t < 4; t++) { axpy<SPL>(kU[t], e.k[t], x[0]); axpy<SPL>(kW[t], e.k[t], x[1]); }
#pragma unroll
    for (int t = 0; t < 8; t++) axpy<SPL>(mL[t], e.vm, x[2 + t]);
}

// Folded records (Step2::recA): the stiffness sums directly, two products
// into each, plus M times Lx1..4, Ly1..4.
template <int SPL>
__device__ __forceinline__ void acc_folded(const Entry &e, const VecF<SPL> *x, float *su, float *sw,
                                           float (*mL)[SPL])
{
    axpy<SPL>(su, e.k[0], x[0]);
    axpy<SPL>(sw, e.k[2], x[1]);
    axpy<SPL>(su, e.k[1], x[1]);
    axpy<SPL>(sw, e.k[3], x[0]);
#pragma unroll
    for (int t = 0; t < 8; t++) axpy<SPL>(mL[t], e.vm, x[2 + t]);
}

// The products of one entry: folded records (one model for every shot) or
// K1..K4 (each shot with its own constants, MM).
template <bool MM, int SPL>
__device__ __forceinline__ void acc_entry(const Entry &e, const VecF<SPL> *x, float (*kU)[SPL], float (*kW)[SPL],
                                          float (*mL)[SPL])
{
    if constexpr (MM) acc_totals<SPL>(e, x, kU, kW, mL);
    else acc_folded<SPL>(e, x, kU[0], kW[0], mL);
}

// MM: every shot has its own model (a.cmm, a.sig; see Step2) and the kernel
// reads the raw records a.rec; otherwise the folded records a.recA.  Two
// shots per lane with folded records run in blocks of at most 4 warps, 5 per
// SM (at most 102 registers): 20 resident warps measured 4-5 % faster than
// 16 at 110 registers, and 24 at 80 registers slower again.
template <bool COMP, int SPL, int S, bool MM>
__global__ void __launch_bounds__(SPL == 2 && !MM ? 128 : 256, SPL == 1 ? 3 : (SPL == 2 ? (MM ? 2 : 5) : 1))
    stepA_batched(const Step2 a)
{
    __shared__ float se[2 * S];
    const StepCommon &c = a.c;
    constexpr int nch = S / (32 * SPL);
    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = gtid; t < c.nrec * S; t += gridDim.x * blockDim.x) gather2_one(c, a.na, a.in, S, t, c.seis_row);
    if (c.energy) energy_zero(se, S);
    const int warp = gtid >> 5, warps_total = (gridDim.x * blockDim.x) >> 5;
    const int s_base = (warp % nch) * 32 * SPL + lane * SPL;
    int src[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) src[q] = s_base + q < c.nshot ? c.src[s_base + q] : -1;
    const double ps = c.amp[c.it];
    const double src_u = ps * c.sin_af, src_w = ps * c.cos_af;
    float eu[SPL], ew[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) { eu[q] = 0.f; ew[q] = 0.f; }
    const float4 *rec = reinterpret_cast<const float4 *>(MM ? a.rec : a.recA);
    constexpr int NK = MM ? 4 : 1;    // accumulators per component: K1..K4 products, or the folded sum
    const long long tasks = (long long)a.na * nch;
    for (long long task = warp; task < tasks; task += warps_total) {
        const int i = (int)(task / nch);
        if (lane == 0 && task % nch == 0) {
            // into L2 while the row's gathers run: the row's own values that
            // its update reads afterwards (U, W and their lo parts, Pa), and
            // the next task's row records
            prefetch_l2(a.in.Gc + (size_t)i * GC * S, 2u * S * 4u);
            prefetch_l2(a.in.Gc + ((size_t)i * GC + 10) * S, 2u * S * 4u);
            prefetch_l2(a.in.Pa + (size_t)i * PA * S, (unsigned)PA * S * 4u);
            if (MM) prefetch_l2(a.cmm + (size_t)i * 6 * S, 6u * S * 4u);
            const long long nt = task + warps_total;
            if (nt < tasks) {
                const int i2 = (int)(nt / nch);
                const int f0 = __ldg(a.up + i2), f1 = __ldg(a.up + i2 + 1);
                prefetch_l2(rec + 2 * (size_t)f0, 32u * (unsigned)(f1 - f0));
            }
        }
        float kU[NK][SPL], kW[NK][SPL], mL[8][SPL];
#pragma unroll
        for (int q = 0; q < SPL; q++) {
#pragma unroll
            for (int k = 0; k < NK; k++) { kU[k][q] = 0.f; kW[k][q] = 0.f; }
#pragma unroll
            for (int k = 0; k < 8; k++) mL[k][q] = 0.f;
        }
        const int e0 = __ldg(a.up + i), e1 = __ldg(a.up + i + 1);
        for (int base = e0; base < e1; base += 32) {
            const int cnt = min(32, e1 - base);
            float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
            if (lane < cnt) { r0 = __ldg(rec + 2 * (size_t)(base + lane)); r1 = __ldg(rec + 2 * (size_t)(base + lane) + 1); }
            int k = 0;
            for (; k + 1 < cnt; k += 2) {
                const Entry ea = entry_at<4>(r0, r1, k), eb = entry_at<4>(r0, r1, k + 1);
                const float *ga = a.in.Gc + (size_t)ea.j * GC * S + s_base;
                const float *gb = a.in.Gc + (size_t)eb.j * GC * S + s_base;
                VecF<SPL> xa[10], xb[10];
#pragma unroll
                for (int v = 0; v < 10; v++) { xa[v].load(ga + v * S); xb[v].load(gb + v * S); }
                acc_entry<MM, SPL>(ea, xa, kU, kW, mL);
                acc_entry<MM, SPL>(eb, xb, kU, kW, mL);
            }
            if (k < cnt) {
                const Entry ea = entry_at<4>(r0, r1, k);
                const float *ga = a.in.Gc + (size_t)ea.j * GC * S + s_base;
                VecF<SPL> xa[10];
#pragma unroll
                for (int v = 0; v < 10; v++) xa[v].load(ga + v * S);
                acc_entry<MM, SPL>(ea, xa, kU, kW, mL);
            }
        }
        const float im = MM ? 0.f : __ldg(a.imA + i);
        VecF<SPL> cm[MM ? 6 : 1];
        if (MM) {
            const float *cp = a.cmm + (size_t)i * 6 * S + s_base;
#pragma unroll
            for (int v = 0; v < (MM ? 6 : 1); v++) cm[v].load(cp + v * S);
        }
        const float *gi = a.in.Gc + (size_t)i * GC * S + s_base;
        const float *pi = a.in.Pa + (size_t)i * PA * S + s_base;
        float *go = a.out.Gc + (size_t)i * GC * S + s_base;
        float *po = a.out.Pa + (size_t)i * PA * S + s_base;
        VecF<SPL> gv[GC], pv[PA];
        gv[0].load(gi);
        gv[1].load(gi + S);
        gv[10].load(gi + 10 * S);
        gv[11].load(gi + 11 * S);
#pragma unroll
        for (int v = 0; v < PA; v++) pv[v].load(pi + v * S);
#pragma unroll
        for (int q = 0; q < SPL; q++) {
            float mq[8], g[GC], p[PA];
#pragma unroll
            for (int t = 0; t < 8; t++) mq[t] = mL[t][q];
            g[0] = gv[0].v[q]; g[1] = gv[1].v[q]; g[10] = gv[10].v[q]; g[11] = gv[11].v[q];
#pragma unroll
            for (int v = 0; v < PA; v++) p[v] = pv[v].v[q];
            float imq = im, su, sw;
            if constexpr (MM) {   // the shot's constants, lumped mass and density (M = diag(rho) M_geo)
                float kUq[4], kWq[4];
#pragma unroll
                for (int t = 0; t < 4; t++) { kUq[t] = kU[t][q]; kWq[t] = kW[t][q]; }
                stiff_sums(kUq, kWq, make_float4(cm[0].v[q], cm[1].v[q], cm[2].v[q], cm[3].v[q]), su, sw);
                imq = cm[4].v[q];
#pragma unroll
                for (int t = 0; t < 8; t++) mq[t] *= cm[5].v[q];
            } else {
                su = kU[0][q];
                sw = kW[0][q];
            }
            const bool is_src = (i == src[q]);
            float uu, ww;
            finish_A<COMP>(su, sw, mq, imq, c.dt, is_src ? src_u : 0.0, is_src ? src_w : 0.0, g, p, uu, ww);
#pragma unroll
            for (int v = 0; v < GC; v++) gv[v].v[q] = g[v];
#pragma unroll
            for (int v = 0; v < PA; v++) pv[v].v[q] = p[v];
            eu[q] += uu * uu;
            ew[q] += ww * ww;
        }
#pragma unroll
        for (int v = 0; v < GC; v++) gv[v].store(go + v * S);
#pragma unroll
        for (int v = 0; v < PA; v++) pv[v].store(po + v * S);
    }
    if (c.energy) energy_flush<SPL>(c, se, S, s_base, eu, ew);
}

// ------------------------------------- class A, staged neighbour gathers
//
// 64 shots, one warp per row (two shots per lane).  The neighbour records a
// row needs (values 0..9 of Gc: 2560 contiguous bytes per neighbour) are
// copied into the warp's own shared-memory buffer with cp.async, up to
// SME entries per item, two buffers per warp: while the warp computes one
// item from shared memory the copies of the next are in flight, so each SM
// keeps many kilobytes of gathers outstanding without spending registers.

constexpr int SME = 5;                       // entries per staged item
constexpr int SREC = 10 * 64 * 4;            // bytes of one neighbour's values 0..9 (64 shots)

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

struct StageItem {
    int row, base, cnt, last;                // row, first entry, entries, last item of the row
};

template <bool COMP>
__global__ void __launch_bounds__(256, 1) stepA_staged(const Step2 a)
{
    constexpr int S = 64, SPL = 2;
    extern __shared__ __align__(16) unsigned char stage[];   // [warp][2][SME * SREC]
    __shared__ float se[2 * S];
    const StepCommon &c = a.c;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int t = gtid; t < c.nrec * S; t += gridDim.x * blockDim.x) gather2_one(c, a.na, a.in, S, t, c.seis_row);
    if (c.energy) energy_zero(se, S);
    const int warp = gtid >> 5, warps_total = (gridDim.x * blockDim.x) >> 5;
    const int s_base = lane * SPL;
    int src[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) src[q] = s_base + q < c.nshot ? c.src[s_base + q] : -1;
    const double ps = c.amp[c.it];
    const double src_u = ps * c.sin_af, src_w = ps * c.cos_af;
    float eu[SPL], ew[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) { eu[q] = 0.f; ew[q] = 0.f; }
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    unsigned char *buf0 = stage + (size_t)wib * 2 * SME * SREC;
    const uint32_t sbuf0 = (uint32_t)__cvta_generic_to_shared(buf0);

    // the item after `it` in this warp's sequence (rows warp, warp + warps_total, ...)
    auto first_of = [&](int row) {
        StageItem s;
        s.row = row;
        s.base = row < a.na ? __ldg(a.up + row) : 0;
        const int e1 = row < a.na ? __ldg(a.up + row + 1) : 0;
        s.cnt = min(SME, e1 - s.base);
        s.last = s.base + s.cnt >= e1;
        return s;
    };
    auto next_of = [&](const StageItem &it) {
        if (!it.last) {
            StageItem s = it;
            const int e1 = __ldg(a.up + it.row + 1);
            s.base = it.base + it.cnt;
            s.cnt = min(SME, e1 - s.base);
            s.last = s.base + s.cnt >= e1;
            return s;
        }
        return first_of(it.row + warps_total);
    };
    // row records of an item (lanes < cnt) and the copies of its neighbours
    auto issue = [&](const StageItem &it, int b, float4 &r0, float4 &r1) {
        r0 = make_float4(0.f, 0.f, 0.f, 0.f);
        r1 = r0;
        if (it.row < a.na && lane < it.cnt) {
            r0 = __ldg(rec + 2 * (size_t)(it.base + lane));
            r1 = __ldg(rec + 2 * (size_t)(it.base + lane) + 1);
        }
        if (it.row < a.na) {
            const uint32_t dst = sbuf0 + (uint32_t)(b * SME * SREC);
            for (int t = 0; t < it.cnt; t++) {
                const int j = __shfl_sync(0xffffffffu, __float_as_int(r0.x), t);
                const unsigned char *g = reinterpret_cast<const unsigned char *>(a.in.Gc + (size_t)j * GC * S);
#pragma unroll
                for (int u = 0; u < SREC / 16 / 32; u++) {
                    const int ch = lane + 32 * u;
                    cp_async16(dst + t * SREC + ch * 16, g + ch * 16);
                }
            }
        }
        cp_async_commit();
    };

    StageItem cur = first_of(warp);
    float4 r0, r1, n0, n1;
    int b = 0;
    issue(cur, 0, r0, r1);
    float kU[4][SPL], kW[4][SPL], mL[8][SPL];
    while (cur.row < a.na) {
        const StageItem nxt = next_of(cur);
        issue(nxt, b ^ 1, n0, n1);
        if (cur.base == __ldg(a.up + cur.row)) {
#pragma unroll
            for (int q = 0; q < SPL; q++) {
#pragma unroll
                for (int k = 0; k < 4; k++) { kU[k][q] = 0.f; kW[k][q] = 0.f; }
#pragma unroll
                for (int k = 0; k < 8; k++) mL[k][q] = 0.f;
            }
        }
        cp_async_wait1();
        __syncwarp();
        const unsigned char *sb = buf0 + b * SME * SREC + lane * 8;
        for (int t = 0; t < cur.cnt; t++) {
            const Entry e = entry_at<4>(r0, r1, t);
            VecF<SPL> x[10];
#pragma unroll
            for (int v = 0; v < 10; v++) {
                const float2 f = *reinterpret_cast<const float2 *>(sb + t * SREC + v * 256);
                x[v].v[0] = f.x;
                x[v].v[1] = f.y;
            }
            acc_totals<SPL>(e, x, kU, kW, mL);
        }
        __syncwarp();
        if (cur.last) {
            const int i = cur.row;
            const float4 cf = __ldg(a.coefA + i);
            const float im = __ldg(a.imA + i);
            const float *gi = a.in.Gc + (size_t)i * GC * S + s_base;
            const float *pi = a.in.Pa + (size_t)i * PA * S + s_base;
            float *go = a.out.Gc + (size_t)i * GC * S + s_base;
            float *po = a.out.Pa + (size_t)i * PA * S + s_base;
            VecF<SPL> gv[GC], pv[PA];
            gv[0].load(gi);
            gv[1].load(gi + S);
            gv[10].load(gi + 10 * S);
            gv[11].load(gi + 11 * S);
#pragma unroll
            for (int v = 0; v < PA; v++) pv[v].load(pi + v * S);
#pragma unroll
            for (int q = 0; q < SPL; q++) {
                float kUq[4], kWq[4], mq[8], g[GC], p[PA];
#pragma unroll
                for (int t = 0; t < 4; t++) { kUq[t] = kU[t][q]; kWq[t] = kW[t][q]; }
#pragma unroll
                for (int t = 0; t < 8; t++) mq[t] = mL[t][q];
                g[0] = gv[0].v[q]; g[1] = gv[1].v[q]; g[10] = gv[10].v[q]; g[11] = gv[11].v[q];
#pragma unroll
                for (int v = 0; v < PA; v++) p[v] = pv[v].v[q];
                const bool is_src = (i == src[q]);
                float uu, ww, su, sw;
                stiff_sums(kUq, kWq, cf, su, sw);
                finish_A<COMP>(su, sw, mq, im, c.dt, is_src ? src_u : 0.0, is_src ? src_w : 0.0, g, p, uu, ww);
#pragma unroll
                for (int v = 0; v < GC; v++) gv[v].v[q] = g[v];
#pragma unroll
                for (int v = 0; v < PA; v++) pv[v].v[q] = p[v];
                eu[q] += uu * uu;
                ew[q] += ww * ww;
            }
#pragma unroll
            for (int v = 0; v < GC; v++) gv[v].store(go + v * S);
#pragma unroll
            for (int v = 0; v < PA; v++) pv[v].store(po + v * S);
        }
        cur = nxt;
        r0 = n0;
        r1 = n1;
        b ^= 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (c.energy) energy_flush<SPL>(c, se, S, s_base, eu, ew);
}

// Split-zone products of one entry: K1..K6 times U, W (K5, K6 only on M-PML
// rows), M times the split fields y[12] (M-PML rows) and M times Lx, Ly.
template <int SPL>
__device__ __forceinline__ void acc_split(const Entry &e, const VecF<SPL> *x, const VecF<SPL> *y, bool full,
                                          bool has_y, float (*kU)[SPL], float (*kW)[SPL], float (*m)[SPL])
{
#pragma unroll
    for (int t = 0; t < 4; t++) { axpy<SPL>(kU[t], e.k[t], x[0]); axpy<SPL>(kW[t], e.k[t], x[1]); }
#pragma unroll
    for (int t = 0; t < 8; t++) axpy<SPL>(m[12 + t], e.vm, x[2 + t]);
    if (full) {
#pragma unroll
        for (int t = 4; t < 6; t++) { axpy<SPL>(kU[t], e.k[t], x[0]); axpy<SPL>(kW[t], e.k[t], x[1]); }
        if (has_y) {
#pragma unroll
            for (int t = 0; t < 12; t++) axpy<SPL>(m[t], e.vm, y[t]);
        }
    }
}

// All entries of row-chunk: full = M-PML row (K5, K6 and the split fields of
// its class-Z columns; M-PML rows reference class-Z columns only).
template <int SPL, int S>
__device__ __forceinline__ void row_split(const Step2 &a, const float4 *rec, int e0, int e1, int lane, int s_base,
                                          bool full, float (*kU)[SPL], float (*kW)[SPL], float (*m)[SPL])
{
    for (int base = e0; base < e1; base += 32) {
        const int cnt = min(32, e1 - base);
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
        if (lane < cnt) { r0 = __ldg(rec + 2 * (size_t)(base + lane)); r1 = __ldg(rec + 2 * (size_t)(base + lane) + 1); }
        int k = 0;
        // two entries in flight with 64 shots per warp, one with 32
        for (; SPL > 1 && k + 1 < cnt; k += 2) {
            const Entry ea = entry_at<6>(r0, r1, k), eb = entry_at<6>(r0, r1, k + 1);
            const float *ga = a.in.Gc + (size_t)ea.j * GC * S + s_base;
            const float *gb = a.in.Gc + (size_t)eb.j * GC * S + s_base;
            VecF<SPL> xa[10], xb[10], ya[12], yb[12];
#pragma unroll
            for (int v = 0; v < 10; v++) { xa[v].load(ga + v * S); xb[v].load(gb + v * S); }
            const bool hya = full && ea.j >= a.na, hyb = full && eb.j >= a.na;
            if (hya) {
                const float *sa = a.in.Gs + (size_t)(ea.j - a.na) * GS * S + s_base;
#pragma unroll
                for (int v = 0; v < 12; v++) ya[v].load(sa + v * S);
            }
            if (hyb) {
                const float *sb = a.in.Gs + (size_t)(eb.j - a.na) * GS * S + s_base;
#pragma unroll
                for (int v = 0; v < 12; v++) yb[v].load(sb + v * S);
            }
            acc_split<SPL>(ea, xa, ya, full, hya, kU, kW, m);
            acc_split<SPL>(eb, xb, yb, full, hyb, kU, kW, m);
        }
#pragma unroll 1
        for (; k < cnt; k++) {
            const Entry ea = entry_at<6>(r0, r1, k);
            const float *ga = a.in.Gc + (size_t)ea.j * GC * S + s_base;
            VecF<SPL> xa[10], ya[12];
#pragma unroll
            for (int v = 0; v < 10; v++) xa[v].load(ga + v * S);
            const bool hya = full && ea.j >= a.na;
            if (hya) {
                const float *sa = a.in.Gs + (size_t)(ea.j - a.na) * GS * S + s_base;
#pragma unroll
                for (int v = 0; v < 12; v++) ya[v].load(sa + v * S);
            }
            acc_split<SPL>(ea, xa, ya, full, hya, kU, kW, m);
        }
    }
}

template <bool COMP, int SPL, int S, bool MM>
__global__ void __launch_bounds__(256, SPL == 1 ? 2 : 1) stepZ_batched(const Step2 a)
{
    __shared__ float se[2 * S];
    const StepCommon &c = a.c;
    constexpr int nch = S / (32 * SPL);
    const int lane = threadIdx.x & 31;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    if (c.energy) energy_zero(se, S);
    const int warp = gtid >> 5, warps_total = (gridDim.x * blockDim.x) >> 5;
    const int s_base = (warp % nch) * 32 * SPL + lane * SPL;
    int src[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) src[q] = s_base + q < c.nshot ? c.src[s_base + q] : -1;
    const double ps = c.amp[c.it];
    const double src_u = ps * c.sin_af, src_w = ps * c.cos_af;
    float eu[SPL], ew[SPL];
#pragma unroll
    for (int q = 0; q < SPL; q++) { eu[q] = 0.f; ew[q] = 0.f; }
    const float4 *rec = reinterpret_cast<const float4 *>(a.rec);
    const int nz = c.n - a.na;
    const long long tasks = (long long)nz * nch;
    for (long long task = warp; task < tasks; task += warps_total) {
        const int local = (int)(task / nch);
        const int i = a.na + local;
        if (lane == 0 && task % nch == 0) {
            // into L2 while the row's gathers run: its own split fields and
            // private values (read by its update afterwards), and the next
            // task's row records
            prefetch_l2(a.in.Gs + (size_t)local * GS * S, (unsigned)GS * S * 4u);
            prefetch_l2(a.in.Ps + (size_t)local * PS * S, (unsigned)PS * S * 4u);
            if (MM) prefetch_l2(a.cmm + (size_t)i * 6 * S, 6u * S * 4u);
            const long long nt = task + warps_total;
            if (nt < tasks) {
                const int i2 = a.na + (int)(nt / nch);
                const int f0 = __ldg(a.up + i2), f1 = __ldg(a.up + i2 + 1);
                prefetch_l2(rec + 2 * (size_t)f0, 32u * (unsigned)(f1 - f0));
            }
        }
        const float4 *cfp = reinterpret_cast<const float4 *>(a.coefZ) + blk4(local, 0, 3);
        const float4 c0 = __ldg(cfp), c1 = __ldg(cfp + 32), c2 = __ldg(cfp + 64);
        float kU[6][SPL], kW[6][SPL], m[20][SPL];
#pragma unroll
        for (int q = 0; q < SPL; q++) {
#pragma unroll
            for (int k = 0; k < 6; k++) { kU[k][q] = 0.f; kW[k][q] = 0.f; }
#pragma unroll
            for (int k = 0; k < 20; k++) m[k][q] = 0.f;
        }
        const int e0 = __ldg(a.up + i), e1 = __ldg(a.up + i + 1);
        row_split<SPL, S>(a, rec, e0, e1, lane, s_base, is_pml_row(c1), kU, kW, m);
        const float *si = a.in.Gs + (size_t)local * GS * S + s_base;
        const float *pi = a.in.Ps + (size_t)local * PS * S + s_base;
        float *gco = a.out.Gc + (size_t)i * GC * S + s_base;
        float *so = a.out.Gs + (size_t)local * GS * S + s_base;
        float *po = a.out.Ps + (size_t)local * PS * S + s_base;
        VecF<SPL> sv[GS], pv[PS], cv[GC], cm[MM ? 6 : 1];
#pragma unroll
        for (int v = 0; v < GS; v++) sv[v].load(si + v * S);
#pragma unroll
        for (int v = 0; v < PS; v++) pv[v].load(pi + v * S);
        if (MM) {
            const float *cp = a.cmm + (size_t)i * 6 * S + s_base;
#pragma unroll
            for (int v = 0; v < (MM ? 6 : 1); v++) cm[v].load(cp + v * S);
        }
#pragma unroll
        for (int q = 0; q < SPL; q++) {
            float kUq[6], kWq[6], mq[20], gs[GS], ps_[PS], gc[GC];
#pragma unroll
            for (int t = 0; t < 6; t++) { kUq[t] = kU[t][q]; kWq[t] = kW[t][q]; }
#pragma unroll
            for (int t = 0; t < 20; t++) mq[t] = m[t][q];
#pragma unroll
            for (int v = 0; v < GS; v++) { gs[v] = sv[v].v[q]; ps_[v] = pv[v].v[q]; }
            float4 c0q = c0, c1q = c1, c2q = c2;
            if (MM) {   // the shot's constants, lumped mass, density; M-PML profiles scale with its vp_max
                const float sg = a.sig[s_base + q];
                c0q = make_float4(cm[0].v[q], cm[1].v[q], cm[2].v[q], cm[3].v[q]);
                c1q = make_float4(c1.x * sg, c1.y * sg, c1.z * sg, c1.w * sg);
                c2q = make_float4(cm[4].v[q], c2.y * sg, c2.z * sg, c2.w);
#pragma unroll
                for (int t = 0; t < 20; t++) mq[t] *= cm[MM ? 5 : 0].v[q];
            }
            const bool is_src = (i == src[q]);
            float uu, ww;
            finish_Z<COMP>(kUq, kWq, mq, c0q, c1q, c2q, c.dt, is_src ? src_u : 0.0, is_src ? src_w : 0.0, gs, ps_,
                           gc, uu, ww);
#pragma unroll
            for (int v = 0; v < GS; v++) { sv[v].v[q] = gs[v]; pv[v].v[q] = ps_[v]; cv[v].v[q] = gc[v]; }
            eu[q] += uu * uu;
            ew[q] += ww * ww;
        }
#pragma unroll
        for (int v = 0; v < GC; v++) cv[v].store(gco + v * S);
#pragma unroll
        for (int v = 0; v < GS; v++) sv[v].store(so + v * S);
#pragma unroll
        for (int v = 0; v < PS; v++) pv[v].store(po + v * S);
    }
    if (c.energy) energy_flush<SPL>(c, se, S, s_base, eu, ew);
}

// ------------------------------------------ staged-gather tile kernels
//
// One block of kTileRows threads per tile: a window of kTileRows consecutive
// rows of one class, which the set-up's Morton order makes a compact patch
// of the mesh.  The block first copies every record its rows gather -- its
// own rows' and its halo's (the rows outside the tile that its rows
// reference) -- from global memory into shared memory with cp.async, all
// copies in flight at once, and then runs the arithmetic of stepA_kernel /
// stepZ_kernel (value dictionary) with every neighbour read served from
// shared memory.  Slots are 4 bytes: (halo position << 16 | tuple id).  The
// staged records are planes of float4 (plane k holds bytes 16k..16k+15 of
// each record), so a warp reading one plane touches distinct banks when its
// columns are distinct.

// Copies the 48-byte records rows[k] (k < nr: row w0 + k; else ext[k - nr])
// of `base` (one-shot block layout, blk4) into planes P, P + H, P + 2H of
// shared memory.
__device__ __forceinline__ void tile_stage(const float *__restrict__ base, int w0, int nr,
                                           const int *__restrict__ ext, int ne, float4 *P, int H)
{
    const uint32_t s0 = (uint32_t)__cvta_generic_to_shared(P);
    const float4 *b4 = reinterpret_cast<const float4 *>(base);
    for (int k = threadIdx.x; k < nr + ne; k += blockDim.x) {
        const int g = k < nr ? w0 + k : __ldg(ext + k - nr);
        const float4 *src = b4 + blk4(g, 0, 3);
        cp_async16(s0 + 16u * (uint32_t)k, src);
        cp_async16(s0 + 16u * (uint32_t)(H + k), src + 32);
        cp_async16(s0 + 16u * (uint32_t)(2 * H + k), src + 64);
    }
}

// Copies n float4 from global src to shared dst (all threads, 16-byte cp.async).
__device__ __forceinline__ void tile_copy(float4 *dst, const float4 *__restrict__ src, int n)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    for (int k = threadIdx.x; k < n; k += blockDim.x) cp_async16(d + 16u * (uint32_t)k, src + k);
}

template <bool COMP>
__global__ void __launch_bounds__(kTileRows, 3) stepAT_kernel(const Step2 a)
{
    // shared memory (float4 units): the halo's three planes [3H], the
    // dictionary [2D], the tile's slots [8 SM], Pa [kTileRows], c [kTileRows]
    extern __shared__ float4 tsm[];
    const int H = a.haloA_max, SM = a.slotsA_max;
    const float4 *P0 = tsm, *P1 = tsm + H, *P2 = tsm + 2 * H;
    float4 *stab = tsm + 3 * H;
    float4 *SL = stab + 2 * a.dict_n;
    float4 *PAs = SL + 8 * SM;
    float4 *CFs = PAs + kTileRows;
    const StepCommon &c = a.c;
    const int t = blockIdx.x, tx = threadIdx.x;
    const int i = t * kTileRows + tx;
    gather2_one(c, a.na, a.in, 1, i, c.seis_row);
    const int w0 = t * kTileRows;
    const int nr = max(0, min(a.na - w0, kTileRows));
    for (int k = tx; k < 2 * a.dict_n; k += kTileRows) stab[k] = __ldg(a.dict + k);
    int slb = 0;   // the tile's first slot row
    if (nr > 0) {
        const int e0 = __ldg(a.tileA_off + t), ne = __ldg(a.tileA_off + t + 1) - e0;
        slb = __ldg(a.sliceA + w0 / 32);
        const int sle = __ldg(a.sliceA + (w0 + nr + 31) / 32);
        tile_copy(SL, reinterpret_cast<const float4 *>(a.sellAt) + (size_t)slb * 8, (sle - slb) * 8);
        tile_copy(PAs, reinterpret_cast<const float4 *>(a.in.Pa) + w0, nr);
        tile_copy(CFs, a.coefA + w0, nr);
        tile_stage(a.in.Gc, w0, nr, a.tileA_ext + e0, ne, tsm, H);
    }
    const float im = tx < nr ? __ldcs(a.imA + i) : 0.f;
    const float rho = tx < nr ? __ldcs(a.rowrho + i) : 0.f;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    double eu = 0.0, ew = 0.0;
    if (tx < nr) {
        const int lane = i & 31, slice = i >> 5;
        float kU[4], kW[4], mL[8];
#pragma unroll
        for (int k = 0; k < 4; k++) { kU[k] = 0.f; kW[k] = 0.f; }
#pragma unroll
        for (int k = 0; k < 8; k++) mL[k] = 0.f;
        const int sl0 = __ldg(a.sliceA + slice), sl1 = __ldg(a.sliceA + slice + 1);
        // own (hi, lo) displacements: K U = sum_j K_ij (U_j - U_i)
        const float4 own0 = P0[tx], own2 = P2[tx];
        const unsigned *sv = reinterpret_cast<const unsigned *>(SL) + lane;
#pragma unroll 2
        for (int g = sl0; g < sl1; ++g) {
            const unsigned v = sv[(g - slb) * 32];
            const int loc = (int)(v >> 16), id = (int)(v & 0xFFFFu);
            const float4 t0 = stab[2 * id], t1 = stab[2 * id + 1];
            const float4 q0 = P0[loc], q1 = P1[loc], q2 = P2[loc];
            const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
            const float kv[4] = {t0.y, t0.z, t0.w, t1.x};
            const float vm = t0.x;
#pragma unroll
            for (int k = 0; k < 4; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
            mL[0] += vm * q0.z; mL[1] += vm * q0.w; mL[2] += vm * q1.x; mL[3] += vm * q1.y;
            mL[4] += vm * q1.z; mL[5] += vm * q1.w; mL[6] += vm * q2.x; mL[7] += vm * q2.y;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) mL[k] *= rho;
        const float4 cf = CFs[tx];
        double src_u = 0.0, src_w = 0.0;
        if (i == c.src[0]) {
            const double ps = c.amp[c.it];
            src_u = ps * c.sin_af;
            src_w = ps * c.cos_af;
        }
        float g[GC], p[PA];
        const float4 own1 = P1[tx];
        g[0] = own0.x; g[1] = own0.y; g[2] = own0.z; g[3] = own0.w;
        g[4] = own1.x; g[5] = own1.y; g[6] = own1.z; g[7] = own1.w;
        g[8] = own2.x; g[9] = own2.y; g[10] = own2.z; g[11] = own2.w;
        const float4 pv = PAs[tx];
        p[0] = pv.x; p[1] = pv.y; p[2] = pv.z; p[3] = pv.w;
        float uu, ww, su, sw;
        stiff_sums(kU, kW, cf, su, sw);
        finish_A<COMP>(su, sw, mL, im, c.dt, src_u, src_w, g, p, uu, ww);
        float4 *go = reinterpret_cast<float4 *>(a.out.Gc) + blk4(i, 0, 3);
#pragma unroll
        for (int k = 0; k < 3; k++) go[32 * k] = make_float4(g[4 * k], g[4 * k + 1], g[4 * k + 2], g[4 * k + 3]);
        reinterpret_cast<float4 *>(a.out.Pa)[i] = make_float4(p[0], p[1], p[2], p[3]);
        eu = (double)uu * uu;
        ew = (double)ww * ww;
    }
    block_energy(c.energy ? c.energy + ((size_t)c.it) * 2 : nullptr, eu, ew);
}

template <bool COMP>
__global__ void __launch_bounds__(kTileRows, 2) stepZT_kernel(const Step2 a)
{
    // shared memory (float4 units): the halo's Gc planes [3H] and Gs planes
    // [3H], the dictionary [2D], the tile's slots [8 SM], Ps [3 kTileRows],
    // coefficients [3 kTileRows]
    extern __shared__ float4 tsm[];
    const int H = a.haloZ_max, SM = a.slotsZ_max;
    const float4 *P0 = tsm, *P1 = tsm + H, *P2 = tsm + 2 * H;       // Gc records
    float4 *Q = tsm + 3 * H;                                       // Gs records
    const float4 *Q0 = Q, *Q1 = Q + H, *Q2 = Q + 2 * H;
    float4 *stab = tsm + 6 * H;
    float4 *SL = stab + 2 * a.dict_n;
    float4 *PSs = SL + 8 * SM;
    float4 *CFs = PSs + 3 * kTileRows;
    const StepCommon &c = a.c;
    const int nz = c.n - a.na;
    const int t = blockIdx.x, tx = threadIdx.x;
    const int local = t * kTileRows + tx;
    const int i = a.na + local;
    const int w0 = a.na + t * kTileRows;
    const int nr = max(0, min(nz - t * kTileRows, kTileRows));
    for (int k = tx; k < 2 * a.dict_n; k += kTileRows) stab[k] = __ldg(a.dict + k);
    const int e0 = __ldg(a.tileZ_off + t), ne = __ldg(a.tileZ_off + t + 1) - e0;
    const int *ext = a.tileZ_ext + e0;
    const int lb = t * kTileRows;                                  // the tile's first class-Z row
    const int slb = __ldg(a.sliceZ + lb / 32), sle = __ldg(a.sliceZ + (lb + nr + 31) / 32);
    tile_copy(SL, reinterpret_cast<const float4 *>(a.sellZt) + (size_t)slb * 8, (sle - slb) * 8);
    // the tile's Ps records and coefficients: whole blocks of the block
    // layout (lb is a multiple of 32), read back with blk4(tx, k, 3)
    tile_copy(PSs, reinterpret_cast<const float4 *>(a.in.Ps) + (size_t)lb * 3, 3 * (int)blk_rows(nr));
    tile_copy(CFs, reinterpret_cast<const float4 *>(a.coefZ) + (size_t)lb * 3, 3 * (int)blk_rows(nr));
    const float rho = tx < nr ? __ldcs(a.rowrho + i) : 0.f;
    tile_stage(a.in.Gc, w0, nr, ext, ne, tsm, H);
    {
        // split-field records of the staged rows (class Z only; zeros for
        // class-A columns, whose split fields no row uses)
        const uint32_t q0 = (uint32_t)__cvta_generic_to_shared(Q);
        for (int k = tx; k < nr + ne; k += kTileRows) {
            const int g = k < nr ? w0 + k : __ldg(ext + k - nr);
            if (g >= a.na) {
                const float4 *src = reinterpret_cast<const float4 *>(a.in.Gs) + blk4(g - a.na, 0, 3);
                cp_async16(q0 + 16u * (uint32_t)k, src);
                cp_async16(q0 + 16u * (uint32_t)(H + k), src + 32);
                cp_async16(q0 + 16u * (uint32_t)(2 * H + k), src + 64);
            } else {
                const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
                Q[k] = z;
                Q[H + k] = z;
                Q[2 * H + k] = z;
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0, c2 = c0;
    if (tx < nr) {
        c0 = CFs[blk4(tx, 0, 3)]; c1 = CFs[blk4(tx, 1, 3)]; c2 = CFs[blk4(tx, 2, 3)];
    }
    const bool full = __any_sync(0xffffffffu, tx < nr && is_pml_row(c1));
    double eu = 0.0, ew = 0.0;
    if (tx < nr) {
        const int lane = local & 31, slice = local >> 5;
        float kU[6], kW[6], m[20];
#pragma unroll
        for (int k = 0; k < 6; k++) { kU[k] = 0.f; kW[k] = 0.f; }
#pragma unroll
        for (int k = 0; k < 20; k++) m[k] = 0.f;
        const int sl0 = __ldg(a.sliceZ + slice), sl1 = __ldg(a.sliceZ + slice + 1);
        const float4 own0 = P0[tx], own2 = P2[tx];
        const unsigned *sv = reinterpret_cast<const unsigned *>(SL) + lane;
        if (full) {
#pragma unroll 2
            for (int g = sl0; g < sl1; ++g) {
                const unsigned v = sv[(g - slb) * 32];
                const int loc = (int)(v >> 16), id = (int)(v & 0xFFFFu);
                const float4 t0 = stab[2 * id], t1 = stab[2 * id + 1];
                const float kv[6] = {t0.y, t0.z, t0.w, t1.x, t1.y, t1.z};
                const float vm = t0.x;
                const float4 q0 = P0[loc], q1 = P1[loc], q2 = P2[loc];
                const float4 z0 = Q0[loc], z1 = Q1[loc], z2 = Q2[loc];
                const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
#pragma unroll
                for (int k = 0; k < 6; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
                m[0] += vm * z0.x;  m[1] += vm * z0.y;  m[2] += vm * z0.z;  m[3] += vm * z0.w;
                m[4] += vm * z1.x;  m[5] += vm * z1.y;  m[6] += vm * z1.z;  m[7] += vm * z1.w;
                m[8] += vm * z2.x;  m[9] += vm * z2.y;  m[10] += vm * z2.z; m[11] += vm * z2.w;
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        } else {
#pragma unroll 2
            for (int g = sl0; g < sl1; ++g) {
                const unsigned v = sv[(g - slb) * 32];
                const int loc = (int)(v >> 16), id = (int)(v & 0xFFFFu);
                const float4 t0 = stab[2 * id], t1 = stab[2 * id + 1];
                const float kv[4] = {t0.y, t0.z, t0.w, t1.x};
                const float vm = t0.x;
                const float4 q0 = P0[loc], q1 = P1[loc], q2 = P2[loc];
                const float du = (q0.x - own0.x) + (q2.z - own2.z), dw = (q0.y - own0.y) + (q2.w - own2.w);
#pragma unroll
                for (int k = 0; k < 4; k++) { kU[k] += kv[k] * du; kW[k] += kv[k] * dw; }
                m[12] += vm * q0.z; m[13] += vm * q0.w; m[14] += vm * q1.x; m[15] += vm * q1.y;
                m[16] += vm * q1.z; m[17] += vm * q1.w; m[18] += vm * q2.x; m[19] += vm * q2.y;
            }
        }
#pragma unroll
        for (int k = 0; k < 20; k++) m[k] *= rho;
        double src_u = 0.0, src_w = 0.0;
        if (i == c.src[0]) {
            const double ps = c.amp[c.it];
            src_u = ps * c.sin_af;
            src_w = ps * c.cos_af;
        }
        float gs[GS], ps_[PS], gc[GC];
        const float4 sq[3] = {Q0[tx], Q1[tx], Q2[tx]};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float4 w = PSs[blk4(tx, k, 3)];
            gs[4 * k] = sq[k].x; gs[4 * k + 1] = sq[k].y; gs[4 * k + 2] = sq[k].z; gs[4 * k + 3] = sq[k].w;
            ps_[4 * k] = w.x; ps_[4 * k + 1] = w.y; ps_[4 * k + 2] = w.z; ps_[4 * k + 3] = w.w;
        }
        float uu, ww;
        finish_Z<COMP>(kU, kW, m, c0, c1, c2, c.dt, src_u, src_w, gs, ps_, gc, uu, ww);
        float4 *gco = reinterpret_cast<float4 *>(a.out.Gc) + blk4(i, 0, 3);
        float4 *so = reinterpret_cast<float4 *>(a.out.Gs) + blk4(local, 0, 3);
        float4 *po = reinterpret_cast<float4 *>(a.out.Ps) + blk4(local, 0, 3);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            gco[32 * k] = make_float4(gc[4 * k], gc[4 * k + 1], gc[4 * k + 2], gc[4 * k + 3]);
            so[32 * k] = make_float4(gs[4 * k], gs[4 * k + 1], gs[4 * k + 2], gs[4 * k + 3]);
            po[32 * k] = make_float4(ps_[4 * k], ps_[4 * k + 1], ps_[4 * k + 2], ps_[4 * k + 3]);
        }
        eu = (double)uu * uu;
        ew = (double)ww * ww;
    }
    block_energy(c.energy ? c.energy + ((size_t)c.it) * 2 : nullptr, eu, ew);
}

// ------------------------------- one-shot kernels with staged slot streams
//
// Launch shape kSlotStageShape: blocks of 128 rows copy all the SELL slots of
// their 4 slices (value dictionary: 8-byte (column, tuple id) pairs) into
// shared memory with cp.async before their rows start, so that no row waits
// for its slot stream; the neighbour gathers stay global (L1/L2), in the
// mesh-order numbering where a slice's gathers are contiguous.
constexpr int kStgThreads = 128;

template <bool COMP>
__global__ void __launch_bounds__(kStgThreads, 4) stepA_kernel_stg(const Step2 a)
{
    extern __shared__ float4 stab[];            // dictionary [2D], then the slot rows
    int2 *slt = reinterpret_cast<int2 *>(stab + 2 * a.dict_n);
    const int nsl = (a.na + 31) / 32;
    const int sa = min(nsl, (int)blockIdx.x * (kStgThreads / 32)), sb = min(nsl, sa + kStgThreads / 32);
    const int slb = sa < nsl ? __ldg(a.sliceA + sa) : 0, sle = sa < nsl ? __ldg(a.sliceA + sb) : 0;
    tile_copy(reinterpret_cast<float4 *>(slt), reinterpret_cast<const float4 *>(a.sellAd + (size_t)slb * 32),
              (sle - slb) * 16);
    for (int t = threadIdx.x; t < 2 * a.dict_n; t += kStgThreads) stab[t] = __ldg(a.dict + t);
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    stepA_body<COMP, kStgThreads, true, true>(a, blockIdx.x, stab, a.c.it, a.c.seis_row, slt, slb);
}

template <bool COMP>
__global__ void __launch_bounds__(kStgThreads, 4) stepZ_kernel_stg(const Step2 a)
{
    extern __shared__ float4 stab[];
    int2 *slt = reinterpret_cast<int2 *>(stab + 2 * a.dict_n);
    const int nsl = (a.c.n - a.na + 31) / 32;
    const int sa = min(nsl, (int)blockIdx.x * (kStgThreads / 32)), sb = min(nsl, sa + kStgThreads / 32);
    const int slb = sa < nsl ? __ldg(a.sliceZ + sa) : 0, sle = sa < nsl ? __ldg(a.sliceZ + sb) : 0;
    tile_copy(reinterpret_cast<float4 *>(slt), reinterpret_cast<const float4 *>(a.sellZd + (size_t)slb * 32),
              (sle - slb) * 16);
    for (int t = threadIdx.x; t < 2 * a.dict_n; t += kStgThreads) stab[t] = __ldg(a.dict + t);
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    stepZ_body<COMP, kStgThreads, true, true>(a, blockIdx.x, stab, a.c.it, slt, slb);
}

// --------------------------------------------------- gathers, snapshots

__global__ void gather2_kernel(const StepCommon c, int na, const State32 st, int S)
{
    gather2_one(c, na, st, S, blockIdx.x * blockDim.x + threadIdx.x, c.seis_row);
}

__global__ void snapshot2_kernel(const State32 st, int n, int na, int S, const int *perm, double *su, double *sw,
                                 long long shot_stride)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * S) return;
    const int s = (int)(t % S);
    const long long node = t / S;
    double u, w;
    total_uw(st, na, S, node, s, u, w);
    const long long o = perm[node];
    su[s * shot_stride + o] = u;
    sw[s * shot_stride + o] = w;
}

// ------------------------------------------------------------ builders

__global__ void range_slice_len(int r0, int r1, const int *__restrict__ up, const int *__restrict__ perm, int *len)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = r1 - r0, nsl = (n + 31) / 32;
    if (s >= nsl) return;
    int m = 0;
    for (int l = 0; l < 32; l++) {
        const int r = s * 32 + l;
        if (r < n) {
            const int o = perm[r0 + r];
            m = max(m, up[o + 1] - up[o]);
        }
    }
    len[s] = m;
}

__global__ void range_sell_fill(int r0, int r1, const int *__restrict__ up, const int *__restrict__ uj,
                                const double *__restrict__ ux, long long nnz, const int *__restrict__ sp,
                                const int *__restrict__ perm, const int *__restrict__ inv, int planes,
                                float *__restrict__ sell)
{
    const int s = blockIdx.x, lane = threadIdx.x;
    const int n = r1 - r0, r = s * 32 + lane;
    const int s0 = sp[s], s1 = sp[s + 1];
    const int o = r < n ? perm[r0 + r] : 0;
    const int a0 = r < n ? up[o] : 0, len = r < n ? up[o + 1] - a0 : 0;
    for (int k = 0; k < s1 - s0; k++) {
        float *slot = sell + (size_t)(s0 + k) * planes * 32;
        if (k < len) {
            const long long e = a0 + k;
            slot[lane] = __int_as_float(inv[uj[e]]);
            for (int m = 0; m < planes - 1; m++) slot[32 * (m + 1) + lane] = (float)ux[m * nnz + e];
        } else {
            slot[lane] = __int_as_float(r < n ? r0 + r : r0);   // the row itself, zero weights
            for (int m = 0; m < planes - 1; m++) slot[32 * (m + 1) + lane] = 0.f;
        }
    }
}

// One warp per permuted row: its union entries as 8-float records (column
// in the permuted numbering, then M, K1..K6 rounded to FP32), two float4
// stores per entry, consecutive entries on consecutive lanes.
__global__ void rec_perm_fill(int n, const int *__restrict__ up, const int *__restrict__ uj,
                              const double *__restrict__ ux, long long nnz, const int *__restrict__ perm,
                              const int *__restrict__ inv, const int *__restrict__ upp, float *__restrict__ rec)
{
    const long long wr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wr >= n) return;
    const int r = (int)wr, lane = threadIdx.x & 31;
    const int o = perm[r];
    const int a0 = up[o], len = up[o + 1] - a0;
    const long long d0 = upp[r];
    for (int k = lane; k < len; k += 32) {
        const long long e = a0 + k;
        float4 *d = reinterpret_cast<float4 *>(rec + (d0 + k) * 8);
        d[0] = make_float4(__int_as_float(inv[uj[e]]), (float)ux[e], (float)ux[nnz + e], (float)ux[2 * nnz + e]);
        d[1] = make_float4((float)ux[3 * nnz + e], (float)ux[4 * nnz + e], (float)ux[5 * nnz + e],
                           (float)ux[6 * nnz + e]);
    }
}

// Class-A rows with one model for every shot: the row's elastic constants
// folded into its stiffness entries, formed in FP64 from the union values and
// rounded once.  Planes: column, M (as rec_perm_fill), then
//   -(c11 K1 + c44 K2) (times U) and -(c13 K3 + c44 K4) (times W), summed into
//   the u right-hand side;
//   -(c44 K1 + c33 K2) (times W) and -(c44 K3 + c13 K4) (times U), into the w
//   right-hand side;
// planes 6, 7 zero.  c: [4][n] c11, c13, c33, c44 in mesh order.
__global__ void rec_fold_fill(int na, int n, const int *__restrict__ up, const int *__restrict__ uj,
                              const double *__restrict__ ux, long long nnz, const int *__restrict__ perm,
                              const int *__restrict__ inv, const int *__restrict__ upp, const double *__restrict__ c,
                              float *__restrict__ rec)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= na) return;
    const int o = perm[r];
    const double c11 = c[o], c13 = c[(size_t)n + o], c33 = c[2 * (size_t)n + o], c44 = c[3 * (size_t)n + o];
    const int a0 = up[o], len = up[o + 1] - a0;
    const long long d0 = upp[r];
    for (int k = 0; k < len; k++) {
        const long long e = a0 + k, d = d0 + k;
        const double K1 = ux[nnz + e], K2 = ux[2 * nnz + e], K3 = ux[3 * nnz + e], K4 = ux[4 * nnz + e];
        float *q = rec + d * 8;
        q[0] = __int_as_float(inv[uj[e]]);
        q[1] = (float)ux[e];
        q[2] = (float)(-(c11 * K1 + c44 * K2));
        q[3] = (float)(-(c13 * K3 + c44 * K4));
        q[4] = (float)(-(c44 * K1 + c33 * K2));
        q[5] = (float)(-(c44 * K3 + c13 * K4));
        q[6] = 0.f;
        q[7] = 0.f;
    }
}

__global__ void coef2_kernel(int n, int na, const float *__restrict__ coef, const int *__restrict__ perm,
                             float4 *__restrict__ coefA, float *__restrict__ imA, float *__restrict__ coefZ)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float *src = coef + (size_t)perm[r] * CREC;
    if (r < na) {
        coefA[r] = make_float4(src[0], src[1], src[2], src[3]);
        imA[r] = src[8];
    } else {
        // the block layout of the one-shot records (blk4), 12 floats per row
        for (int k = 0; k < CREC; k++) coefZ[4 * blk4(r - na, k >> 2, 3) + (k & 3)] = src[k];
    }
}

// ------------------------------------------------- two-class numbering

// pml[r]: any of dx, dy, dxx, dyy non-zero in FP32 (the step's test)
__global__ void class_flags(int n, const double *__restrict__ mpml, unsigned char *__restrict__ pml,
                            unsigned char *__restrict__ zone, int *npml)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    bool f = false;
#pragma unroll
    for (int k = 0; k < 4; k++) f = f || ((float)mpml[(size_t)k * n + r] != 0.f);
    pml[r] = f ? 1 : 0;
    zone[r] = 0;
    if (f) atomicAdd(npml, 1);
}

// zone: M-PML rows and every column they reference (idempotent writes)
__global__ void class_zone(int n, const int *__restrict__ up, const int *__restrict__ uj,
                           const unsigned char *__restrict__ pml, unsigned char *__restrict__ zone)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || !pml[r]) return;
    zone[r] = 1;
    for (int e = up[r]; e < up[r + 1]; e++) zone[uj[e]] = 1;
}

__global__ void class_split(int n, const unsigned char *__restrict__ zone, int *__restrict__ isA,
                            int *__restrict__ isZ)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    isA[r] = zone[r] ? 0 : 1;
    isZ[r] = zone[r] ? 1 : 0;
}

// the last `k` class-A rows (mesh order) join class Z, so that the class-A
// row count is a multiple of 32 (posA: exclusive scan of the class-A flags)
__global__ void class_align(int n, int k, const int *__restrict__ posA, unsigned char *__restrict__ zone)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || zone[r]) return;
    if (posA[r] >= posA[n] - k) zone[r] = 1;
}

// class A rows first, then class Z, each in mesh order
__global__ void class_scatter(int n, const unsigned char *__restrict__ zone, const int *__restrict__ posA,
                              const int *__restrict__ posZ, int *__restrict__ perm0)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int na = posA[n];
    perm0[zone[r] ? na + posZ[r] : posA[r]] = r;
}

// Morton key (bits of the two quantised coordinates interleaved) of the
// mesh node of every entry of perm0, for the spatial order inside a class.
__device__ __forceinline__ unsigned spread16(unsigned v)
{
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__global__ void class_morton(int n, const int *__restrict__ perm0, const double *__restrict__ x,
                             const double *__restrict__ y, double x0, double sx, double y0, double sy,
                             unsigned *__restrict__ key)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = perm0[i];
    const double qx = fmin(fmax((x[r] - x0) * sx, 0.0), 65535.0);
    const double qy = fmin(fmax((y[r] - y0) * sy, 0.0), 65535.0);
    key[i] = (spread16((unsigned)qy) << 1) | spread16((unsigned)qx);
}

// One block per window of W rows (a power of two <= 2048; windows restart at
// the class boundary): a stable sort by (M-PML flag, decreasing row length)
// -- a bitonic sort of keys that carry the position in the window as their
// low 11 bits.
__global__ void __launch_bounds__(1024) class_windows(int n, int na, int maxlen, const int *__restrict__ up,
                                                      const unsigned char *__restrict__ pml,
                                                      const int *__restrict__ perm0, int *__restrict__ perm, int W)
{
    __shared__ unsigned key[2048];
    const int wa = (na + W - 1) / W;
    const int w = blockIdx.x;
    // (W is uniform across the block)
    const int w0 = w < wa ? w * W : na + (w - wa) * W;
    const int w1 = w < wa ? min(na, w0 + W) : min(n, w0 + W);
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        unsigned k = 0xFFFFFFFFu;
        if (w0 + i < w1) {
            const int r = perm0[w0 + i];
            const int len = up[r + 1] - up[r];
            k = ((unsigned)(pml[r] * (maxlen + 1) + (maxlen - len)) << 11) | (unsigned)i;
        }
        key[i] = k;
    }
    __syncthreads();
    for (int k = 2; k <= W; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < W; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool asc = (i & k) == 0;
                    const unsigned a = key[i], b = key[ixj];
                    if ((a > b) == asc) { key[i] = b; key[ixj] = a; }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < w1 - w0; i += blockDim.x) perm[w0 + i] = perm0[w0 + (int)(key[i] & 2047u)];
}

__global__ void class_inverse(int n, const int *__restrict__ perm, const int *__restrict__ up, int *__restrict__ inv,
                              int *__restrict__ lenp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = perm[i];
    inv[r] = i;
    lenp[i] = up[r + 1] - up[r];
}

// one model per shot: the geometric mass matrix M_geo = M / rho0(row) in
// plane 1 of the row records, and the row sums of M_geo
__global__ void rec_geo_fill(int n, const int *__restrict__ up, const double *__restrict__ ux,
                             const int *__restrict__ perm, const int *__restrict__ upp,
                             const double *__restrict__ rho0, float *__restrict__ rec)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int o = perm[r];
    const int a0 = up[o], len = up[o + 1] - a0;
    const long long d0 = upp[r];
    for (int k = 0; k < len; k++) rec[(d0 + k) * 8 + 1] = (float)(ux[a0 + k] / rho0[o]);
}

__global__ void row_sums_geo(int n, const int *__restrict__ up, const double *__restrict__ ux,
                             const double *__restrict__ rho0, double *__restrict__ out)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    double s = 0.0;
    for (int e = up[o]; e < up[o + 1]; e++) s += ux[e];
    out[o] = s / rho0[o];
}

}  // namespace

// ---------------------------------------------------------- launchers

// Launch shapes of the single-shot kernels (rows = threads per block,
// minimum resident blocks for the register allocation):
//   0: 128 x 4   1: 128 x 6   2: 256 x 3   3: 256 x 4   4: 64 x 16   5: 512 x 2
int step2_variants() { return 6; }

cudaError_t launch_range_slice_len(int r0, int r1, const int *d_up, const int *d_perm, int *d_len, cudaStream_t st)
{
    const int nsl = (r1 - r0 + 31) / 32;
    if (nsl) range_slice_len<<<(nsl + 127) / 128, 128, 0, st>>>(r0, r1, d_up, d_perm, d_len);
    return cudaGetLastError();
}

// (threads per block, minimum resident blocks) of the one-shot launch
// shapes; shape 0 of the class-A kernel asks for 7 resident blocks of 128
// threads (72 registers, 28 warps per SM), of the class-Z kernel for 4
// (128 registers: its 32 products per M-PML slot stay in registers)
#define SFG_SHAPES(KERNEL, COUNT, MINB0)                                                       \
    do {                                                                                       \
        if ((COUNT) <= 0) return cudaSuccess;                                                  \
        switch (variant) {                                                                     \
        case 0: SFG_ONE(KERNEL, 128, MINB0, COUNT); break;                                     \
        case 1: SFG_ONE(KERNEL, 128, 6, COUNT); break;                                         \
        case 2: SFG_ONE(KERNEL, 256, 3, COUNT); break;                                         \
        case 4: SFG_ONE(KERNEL, 64, 16, COUNT); break;                                         \
        case 5: SFG_ONE(KERNEL, 512, 2, COUNT); break;                                         \
        case 8: SFG_ONE(KERNEL, 128, 5, COUNT); break;                                         \
        default: SFG_ONE(KERNEL, 256, 4, COUNT); break;                                        \
        }                                                                                      \
    } while (0)
#define SFG_ONE(KERNEL, T, M, COUNT)                                                           \
    do {                                                                                       \
        const int blocks = ((COUNT) + (T) - 1) / (T);                                          \
        const size_t smem = sizeof(float4) * 2 * (size_t)a.dict_n;                             \
        if (a.dict_n > 0 && a.dict_n <= kParamTuples && a.h_dict) {                            \
            Step2T pt;                                                                         \
            pt.a = a;                                                                          \
            std::memcpy(pt.tab, a.h_dict, sizeof(float4) * 2 * (size_t)a.dict_n);              \
            if (comp) KERNEL##_ct<true, T, M><<<blocks, T, 0, st>>>(pt);                        \
            else KERNEL##_ct<false, T, M><<<blocks, T, 0, st>>>(pt);                            \
        } else if (a.dict_n > 0) {                                                             \
            if (comp) KERNEL<true, T, M, true><<<blocks, T, smem, st>>>(a);                    \
            else KERNEL<false, T, M, true><<<blocks, T, smem, st>>>(a);                        \
        } else {                                                                               \
            if (comp) KERNEL<true, T, M, false><<<blocks, T, 0, st>>>(a);                      \
            else KERNEL<false, T, M, false><<<blocks, T, 0, st>>>(a);                          \
        }                                                                                      \
    } while (0)

// dynamic shared memory a tile kernel may use, raised per device as needed
template <typename K>
static cudaError_t allow_smem(K kernel, size_t smem, int *cache)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return e != cudaSuccess ? e : cudaErrorInvalidDevice;
    if ((size_t)cache[dev] >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cache[dev] = (int)smem;
    return e;
}

cudaError_t launch_stepA_tile(const Step2 &a, bool comp, cudaStream_t st)
{
    static int cache[2][64];
    if (!a.tileA_off || a.dict_n <= 0 || a.dict_n > kDictMax || a.haloA_max <= 0 || a.haloA_max > kTileHaloMax)
        return cudaErrorInvalidValue;
    // the fused receiver gather runs on the first nrec threads
    const int rows = std::max(a.na, a.c.seis_row >= 0 ? a.c.nrec : 0);
    if (rows <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((rows + kTileRows - 1) / kTileRows);
    const size_t smem = sizeof(float4) * (3 * (size_t)a.haloA_max + 2 * (size_t)a.dict_n + 8 * (size_t)a.slotsA_max +
                                          2 * (size_t)kTileRows);
    cudaError_t e;
    if (comp) {
        if ((e = allow_smem(stepAT_kernel<true>, smem, cache[1])) != cudaSuccess) return e;
        stepAT_kernel<true><<<blocks, kTileRows, smem, st>>>(a);
    } else {
        if ((e = allow_smem(stepAT_kernel<false>, smem, cache[0])) != cudaSuccess) return e;
        stepAT_kernel<false><<<blocks, kTileRows, smem, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_stepZ_tile(const Step2 &a, bool comp, cudaStream_t st)
{
    static int cache[2][64];
    if (!a.tileZ_off || a.dict_n <= 0 || a.dict_n > kDictMax || a.haloZ_max <= 0 || a.haloZ_max > kTileHaloMax)
        return cudaErrorInvalidValue;
    const int nz = a.c.n - a.na;
    if (nz <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((nz + kTileRows - 1) / kTileRows);
    const size_t smem = sizeof(float4) * (6 * (size_t)a.haloZ_max + 2 * (size_t)a.dict_n + 8 * (size_t)a.slotsZ_max +
                                          6 * (size_t)kTileRows);
    cudaError_t e;
    if (comp) {
        if ((e = allow_smem(stepZT_kernel<true>, smem, cache[1])) != cudaSuccess) return e;
        stepZT_kernel<true><<<blocks, kTileRows, smem, st>>>(a);
    } else {
        if ((e = allow_smem(stepZT_kernel<false>, smem, cache[0])) != cudaSuccess) return e;
        stepZT_kernel<false><<<blocks, kTileRows, smem, st>>>(a);
    }
    return cudaGetLastError();
}

// staged slot streams (launch shape kSlotStageShape; value dictionary only)
static cudaError_t launch_stg(const Step2 &a, bool comp, bool classA, cudaStream_t st)
{
    static int cache[4][64];
    if (a.dict_n <= 0 || a.dict_n > kDictMax || a.max_row_len <= 0 || !a.dict) return cudaErrorInvalidValue;
    const int rows = classA ? std::max(a.na, a.c.seis_row >= 0 ? a.c.nrec : 0) : a.c.n - a.na;
    if (rows <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((rows + kStgThreads - 1) / kStgThreads);
    // slot rows of a block: at most (kStgThreads / 32) slices of max_row_len
    const size_t smem = sizeof(float4) * (2 * (size_t)a.dict_n + 16 * (size_t)(kStgThreads / 32) * a.max_row_len);
    cudaError_t e;
    if (classA) {
        if (comp) {
            if ((e = allow_smem(stepA_kernel_stg<true>, smem, cache[0])) != cudaSuccess) return e;
            stepA_kernel_stg<true><<<blocks, kStgThreads, smem, st>>>(a);
        } else {
            if ((e = allow_smem(stepA_kernel_stg<false>, smem, cache[1])) != cudaSuccess) return e;
            stepA_kernel_stg<false><<<blocks, kStgThreads, smem, st>>>(a);
        }
    } else {
        if (comp) {
            if ((e = allow_smem(stepZ_kernel_stg<true>, smem, cache[2])) != cudaSuccess) return e;
            stepZ_kernel_stg<true><<<blocks, kStgThreads, smem, st>>>(a);
        } else {
            if ((e = allow_smem(stepZ_kernel_stg<false>, smem, cache[3])) != cudaSuccess) return e;
            stepZ_kernel_stg<false><<<blocks, kStgThreads, smem, st>>>(a);
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_stepA(const Step2 &a, bool comp, int variant, cudaStream_t st)
{
    if (variant == kTileShape) return launch_stepA_tile(a, comp, st);
    if (variant == kSlotStageShape) return launch_stg(a, comp, true, st);
    if (a.dict_n > kDictMax || (a.dict_n > 0 && (!a.dict || !a.sellAd || !a.sellZd || !a.rowrho)))
        return cudaErrorInvalidValue;
    // the fused receiver gather runs on the first nrec threads
    SFG_SHAPES(stepA_kernel, std::max(a.na, a.c.seis_row >= 0 ? a.c.nrec : 0), 7);
    return cudaGetLastError();
}

cudaError_t launch_stepZ(const Step2 &a, bool comp, int variant, cudaStream_t st)
{
    if (variant == kTileShape) return launch_stepZ_tile(a, comp, st);
    if (variant == kSlotStageShape) return launch_stg(a, comp, false, st);
    if (a.dict_n > kDictMax || (a.dict_n > 0 && (!a.dict || !a.sellAd || !a.sellZd || !a.rowrho)))
        return cudaErrorInvalidValue;
    SFG_SHAPES(stepZ_kernel, a.c.n - a.na, 4);
    return cudaGetLastError();
}
#undef SFG_ONE

int step2_threads(int variant)
{
    switch (variant) {
    case 0: case 1: case 8: return 128;
    case 2: return 256;
    case 4: return 64;
    case 5: return 512;
    default: return 256;
    }
}

#define SFG_ONE(KERNEL, T, M, COUNT)                                                           \
    do {                                                                                       \
        const size_t smem = sizeof(float4) * 2 * (size_t)dict_max;                             \
        if (dict) {                                                                            \
            if (comp) KERNEL<true, T, M, true><<<(COUNT), T, smem, st>>>(descs, map, it);      \
            else KERNEL<false, T, M, true><<<(COUNT), T, smem, st>>>(descs, map, it);          \
        } else {                                                                               \
            if (comp) KERNEL<true, T, M, false><<<(COUNT), T, 0, st>>>(descs, map, it);        \
            else KERNEL<false, T, M, false><<<(COUNT), T, 0, st>>>(descs, map, it);            \
        }                                                                                      \
    } while (0)

cudaError_t launch_stepA_multi(const Step2 *descs, const int2 *map, int nblocks, bool dict, int dict_max, bool comp,
                               int variant, int it, cudaStream_t st)
{
    if (dict_max > kDictMax || (dict && dict_max <= 0)) return cudaErrorInvalidValue;
    SFG_SHAPES(stepA_multi, nblocks, 7);
    return cudaGetLastError();
}

cudaError_t launch_stepZ_multi(const Step2 *descs, const int2 *map, int nblocks, bool dict, int dict_max, bool comp,
                               int variant, int it, cudaStream_t st)
{
    if (dict_max > kDictMax || (dict && dict_max <= 0)) return cudaErrorInvalidValue;
    SFG_SHAPES(stepZ_multi, nblocks, 4);
    return cudaGetLastError();
}
#undef SFG_ONE
#undef SFG_SHAPES

template <typename K>
static long long batched_grid(K kernel, int threads, long long tasks, int warps, size_t smem)
{
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (per_sm < 1) per_sm = 1;
    const long long need = (tasks + warps - 1) / warps;
    return std::max<long long>(1, std::min<long long>((long long)sms * per_sm, need));
}

#define SFG_BATCH_ONE(KERNEL, C, P, SS, ROWS)                                                            \
    do {                                                                                                 \
        auto k = KERNEL<C, P, SS, false>;                                                                \
        const long long tasks = (long long)(ROWS) * ((SS) / (32 * (P)));                                 \
        KERNEL<C, P, SS, false><<<(unsigned)batched_grid(k, threads, tasks, warps, 0), threads, 0, st>>>(a); \
    } while (0)
#define SFG_BATCH_MM(KERNEL, P, SS, ROWS)                                                                \
    do {                                                                                                 \
        auto k = KERNEL<true, P, SS, true>;                                                              \
        const long long tasks = (long long)(ROWS) * ((SS) / (32 * (P)));                                 \
        KERNEL<true, P, SS, true><<<(unsigned)batched_grid(k, threads, tasks, warps, 0), threads, 0, st>>>(a); \
    } while (0)
#define SFG_BATCH_S(KERNEL, C, ROWS)                                                                     \
    do {                                                                                                 \
        if (a.S == 32) SFG_BATCH_ONE(KERNEL, C, 1, 32, ROWS);                                            \
        else if (a.S == 64 && spl == 1) SFG_BATCH_ONE(KERNEL, C, 1, 64, ROWS);                           \
        else if (a.S == 64) SFG_BATCH_ONE(KERNEL, C, 2, 64, ROWS);                                       \
        else if (spl == 1) SFG_BATCH_ONE(KERNEL, C, 1, 128, ROWS);                                       \
        else if (spl == 2) SFG_BATCH_ONE(KERNEL, C, 2, 128, ROWS);                                       \
        else SFG_BATCH_ONE(KERNEL, C, 4, 128, ROWS);                                                     \
    } while (0)
#define SFG_BATCH(KERNEL, ROWS)                                                                          \
    do {                                                                                                 \
        const int threads = 32 * warps;                                                                  \
        if (warps < 1 || warps > 8 || (spl != 1 && spl != 2 && spl != 4)) return cudaErrorInvalidValue;  \
        if ((a.S != 32 && a.S != 64 && a.S != 128) || a.S % (32 * spl) != 0 ||                           \
            warps % (a.S / (32 * spl)) != 0)                                                             \
            return cudaErrorInvalidValue;                                                                \
        if ((ROWS) <= 0) return cudaSuccess;                                                             \
        if (a.cmm) {   /* one model per shot: compensated precision, 32 or 64 shots */                   \
            if (!comp || a.S > 64 || spl > 2 || !a.sig) return cudaErrorInvalidValue;                     \
            if (a.S == 32) SFG_BATCH_MM(KERNEL, 1, 32, ROWS);                                            \
            else if (spl == 1) SFG_BATCH_MM(KERNEL, 1, 64, ROWS);                                        \
            else SFG_BATCH_MM(KERNEL, 2, 64, ROWS);                                                      \
        } else if (comp) SFG_BATCH_S(KERNEL, true, ROWS);                                                \
        else SFG_BATCH_S(KERNEL, false, ROWS);                                                           \
    } while (0)

// largest block of the batched class-A kernel (its launch bounds)
int stepA_batched_max_warps(int spl, bool models) { return spl == 2 && !models ? 4 : 8; }

cudaError_t launch_stepA_batched(const Step2 &a, bool comp, int spl, int warps, cudaStream_t st)
{
    if (warps > stepA_batched_max_warps(spl, a.cmm != nullptr)) return cudaErrorInvalidValue;
    // at least one warp for the receiver gather even without class-A rows
    SFG_BATCH(stepA_batched, std::max(a.na, 1));
    return cudaGetLastError();
}

cudaError_t launch_stepA_staged(const Step2 &a, bool comp, cudaStream_t st)
{
    if (a.S != 64 || a.cmm) return cudaErrorInvalidValue;
    const int threads = 256;
    const size_t smem = (size_t)(threads / 32) * 2 * SME * SREC;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long need = ((long long)std::max(a.na, 1) + threads / 32 - 1) / (threads / 32);
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(sms, need));
    cudaError_t e;
    if (comp) {
        e = cudaFuncSetAttribute(stepA_staged<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) stepA_staged<true><<<grid, threads, smem, st>>>(a);
    } else {
        e = cudaFuncSetAttribute(stepA_staged<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) stepA_staged<false><<<grid, threads, smem, st>>>(a);
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_stepZ_batched(const Step2 &a, bool comp, int spl, int warps, cudaStream_t st)
{
    SFG_BATCH(stepZ_batched, a.c.n - a.na);
    return cudaGetLastError();
}
#undef SFG_BATCH
#undef SFG_BATCH_S
#undef SFG_BATCH_ONE
#undef SFG_BATCH_MM

cudaError_t launch_gather2(const StepCommon &c, int na, const State32 &s, int S, cudaStream_t st)
{
    const int tot = c.nrec * S;
    if (tot > 0 && c.seis_row >= 0) gather2_kernel<<<(tot + 127) / 128, 128, 0, st>>>(c, na, s, S);
    return cudaGetLastError();
}

cudaError_t launch_snapshot2(const State32 &s, int n, int na, int S, const int *perm, double *su, double *sw,
                             long long shot_stride, cudaStream_t st)
{
    const long long tot = (long long)n * S;
    if (tot > 0)
        snapshot2_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(s, n, na, S, perm, su, sw, shot_stride);
    return cudaGetLastError();
}

cudaError_t build_sell_range(int r0, int r1, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                             const int *d_perm, const int *d_inv, int planes, float **d_sell, int **d_slice,
                             long long *slots, cudaStream_t st)
{
    const int n = r1 - r0, nsl = (n + 31) / 32;
    int *len = nullptr;
    cudaError_t e;
    if ((e = tmp_alloc((void **)&len, sizeof(int) * ((size_t)nsl + 1), st)) != cudaSuccess) return e;
    if ((e = keep_alloc(d_slice, sizeof(int) * ((size_t)nsl + 1), st)) != cudaSuccess) return e;
    if (nsl) range_slice_len<<<(nsl + 127) / 128, 128, 0, st>>>(r0, r1, d_up, d_perm, len);
    if ((e = exclusive_scan_int(len, *d_slice, nsl, st)) != cudaSuccess) return e;
    int tot = 0;
    cudaMemcpyAsync(&tot, *d_slice + nsl, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *slots = tot;
    if ((e = keep_alloc(d_sell, sizeof(float) * planes * 32 * std::max<size_t>(tot, 1), st)) != cudaSuccess) return e;
    if (nsl) range_sell_fill<<<nsl, 32, 0, st>>>(r0, r1, d_up, d_uj, d_ux, nnz, *d_slice, d_perm, d_inv, planes, *d_sell);
    e = cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaFreeAsync(len, st);
    return e;
}

cudaError_t build_rec_perm(int n, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                           const int *d_perm, const int *d_inv, const int *d_upp, float **d_rec, cudaStream_t st)
{
    cudaError_t e = keep_alloc(d_rec, sizeof(float) * 8 * std::max<long long>(nnz, 1), st);
    if (e != cudaSuccess) return e;
    if (n)
        rec_perm_fill<<<(unsigned)(((long long)n * 32 + 255) / 256), 256, 0, st>>>(n, d_up, d_uj, d_ux, nnz, d_perm,
                                                                                    d_inv, d_upp, *d_rec);
    return cudaGetLastError();
}

cudaError_t build_rec_fold(int n, int na, const int *d_up, const int *d_uj, const double *d_ux, long long nnz,
                           const int *d_perm, const int *d_inv, const int *d_upp, const double *d_c, float **d_rec,
                           cudaStream_t st)
{
    int nnz_a = 0;
    cudaError_t e = cudaMemcpyAsync(&nnz_a, d_upp + na, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = keep_alloc(d_rec, sizeof(float) * 8 * std::max(nnz_a, 1), st);
    if (e == cudaSuccess && na > 0) {
        rec_fold_fill<<<(na + 127) / 128, 128, 0, st>>>(na, n, d_up, d_uj, d_ux, nnz, d_perm, d_inv, d_upp, d_c, *d_rec);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t build_coef2(int n, int na, const float *d_coef32, const int *d_perm, float4 **d_coefA, float **d_imA,
                        float **d_coefZ, cudaStream_t st)
{
    cudaError_t e;
    if ((e = keep_alloc(d_coefA, sizeof(float4) * std::max(na, 1), st)) != cudaSuccess) return e;
    if ((e = keep_alloc(d_imA, sizeof(float) * std::max(na, 1), st)) != cudaSuccess) return e;
    if ((e = keep_alloc(d_coefZ, sizeof(float) * CREC * blk_rows(std::max(n - na, 1)), st)) != cudaSuccess) return e;
    // rows past the last class-Z row of the last block stay zero
    if ((e = cudaMemsetAsync(*d_coefZ, 0, sizeof(float) * CREC * blk_rows(std::max(n - na, 1)), st)) != cudaSuccess)
        return e;
    if (n) coef2_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, na, d_coef32, d_perm, *d_coefA, *d_imA, *d_coefZ);
    return cudaGetLastError();
}


// Reorders perm0 inside class A ([0, na)) and inside class Z by the Morton
// key of the nodes' coordinates (stable: equal keys keep mesh order), so that
// windows of consecutive rows are compact patches of the mesh.
static cudaError_t morton_order(int n, int na, int *perm0, const double *d_x, const double *d_y, double x0,
                                double x1, double y0, double y1, cudaStream_t st)
{
    const double sx = x1 > x0 ? 65535.0 / (x1 - x0) : 0.0, sy = y1 > y0 ? 65535.0 / (y1 - y0) : 0.0;
    unsigned *key = nullptr, *key2 = nullptr;
    int *val2 = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = cudaMallocAsync((void **)&key, sizeof(unsigned) * n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&key2, sizeof(unsigned) * n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&val2, sizeof(int) * n, st);
    if (e == cudaSuccess) {
        class_morton<<<(n + 255) / 256, 256, 0, st>>>(n, perm0, d_x, d_y, x0, sx, y0, sy, key);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, perm0, val2, std::max(na, n - na), 0, 32,
                                            st);
    if (e == cudaSuccess) e = cudaMallocAsync(&tmp, std::max<size_t>(tmp_bytes, 16), st);
    // the two classes one after the other (radix sort is stable)
    const int seg[2][2] = {{0, na}, {na, n}};
    for (int c = 0; c < 2 && e == cudaSuccess; c++) {
        const int b = seg[c][0], m = seg[c][1] - seg[c][0];
        if (m <= 1) continue;
        size_t tb = tmp_bytes;
        e = cub::DeviceRadixSort::SortPairs(tmp, tb, key + b, key2 + b, perm0 + b, val2 + b, m, 0, 32, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(perm0 + b, val2 + b, sizeof(int) * m, cudaMemcpyDeviceToDevice, st);
    }
    for (void *p : {(void *)key, (void *)key2, (void *)val2, tmp})
        if (p) cudaFreeAsync(p, st);
    return e;
}

cudaError_t build_classes(int n, const int *d_up, const int *d_uj, const double *d_mpml, int maxlen, int **d_perm,
                          int **d_inv, int **d_upp, int *na_out, int *npml_out, cudaStream_t st, int tile_rows,
                          const double *d_x, const double *d_y, double x0, double x1, double y0, double y1)
{
    if (maxlen < 0 || maxlen >= (1 << 19)) return cudaErrorInvalidValue;
    const int W = tile_rows > 0 ? tile_rows : 2048;
    if (W > 2048 || (W & (W - 1))) return cudaErrorInvalidValue;
    unsigned char *pml = nullptr, *zone = nullptr;
    int *isA = nullptr, *isZ = nullptr, *posA = nullptr, *posZ = nullptr, *perm0 = nullptr, *lenp = nullptr,
        *cnt = nullptr;
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t b) { if (e == cudaSuccess) e = cudaMallocAsync(p, std::max<size_t>(b, 4), st); };
    A((void **)&pml, n); A((void **)&zone, n);
    A((void **)&isA, sizeof(int) * n); A((void **)&isZ, sizeof(int) * n);
    A((void **)&posA, sizeof(int) * (n + 1)); A((void **)&posZ, sizeof(int) * (n + 1));
    A((void **)&perm0, sizeof(int) * n); A((void **)&lenp, sizeof(int) * n); A((void **)&cnt, sizeof(int));
    if (e == cudaSuccess) e = keep_alloc(d_perm, sizeof(int) * std::max(n, 1), st);
    if (e == cudaSuccess) e = keep_alloc(d_inv, sizeof(int) * std::max(n, 1), st);
    if (e == cudaSuccess) e = keep_alloc(d_upp, sizeof(int) * (n + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(int), st);
    const int g = (n + 255) / 256;
    int na = 0, npml = 0;
    if (e == cudaSuccess && n > 0) {
        class_flags<<<g, 256, 0, st>>>(n, d_mpml, pml, zone, cnt);
        class_zone<<<g, 256, 0, st>>>(n, d_up, d_uj, pml, zone);
        class_split<<<g, 256, 0, st>>>(n, zone, isA, isZ);
        e = cudaGetLastError();
        // a class-A row count that is a multiple of 32: the one-shot state
        // blocks of the two classes then line up (blk4(i - na) = blk4(i) -
        // 3 na), and the last few class-A rows carry split fields instead,
        // which the class-Z step handles like any row outside the M-PML
        int na0 = 0;
        if (e == cudaSuccess) e = exclusive_scan_int(isA, posA, n, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&na0, posA + n, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && na0 % 32) {
            class_align<<<g, 256, 0, st>>>(n, na0 % 32, posA, zone);
            class_split<<<g, 256, 0, st>>>(n, zone, isA, isZ);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = exclusive_scan_int(isA, posA, n, st);
        if (e == cudaSuccess) e = exclusive_scan_int(isZ, posZ, n, st);
        if (e == cudaSuccess) {
            class_scatter<<<g, 256, 0, st>>>(n, zone, posA, posZ, perm0);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&na, posA + n, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&npml, cnt, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && d_x && d_y) e = morton_order(n, na, perm0, d_x, d_y, x0, x1, y0, y1, st);
        if (e == cudaSuccess) {
            const int windows = (na + W - 1) / W + (n - na + W - 1) / W;
            class_windows<<<windows, std::min(W, 1024), 0, st>>>(n, na, maxlen, d_up, pml, perm0, *d_perm, W);
            class_inverse<<<g, 256, 0, st>>>(n, *d_perm, d_up, *d_inv, lenp);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = exclusive_scan_int(lenp, *d_upp, n, st);
    }
    for (void *p : {(void *)pml, (void *)zone, (void *)isA, (void *)isZ, (void *)posA, (void *)posZ, (void *)perm0,
                    (void *)lenp, (void *)cnt})
        if (p) cudaFreeAsync(p, st);
    *na_out = na;
    *npml_out = npml;
    return e;
}


// ------------------------------------------------ staged-gather tiles

namespace {

constexpr int kTileCand = 4096;   // references outside a tile collected before removing repeats

// Bitonic sort of P keys (a power of two) in shared memory by the block.
__device__ void block_bitonic(unsigned *key, int P)
{
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool asc = (i & k) == 0;
                    const unsigned a = key[i], b = key[ixj];
                    if ((a > b) == asc) { key[i] = b; key[ixj] = a; }
                }
            }
            __syncthreads();
        }
}

// Tile t of permuted rows [r0, r1): the distinct rows outside the tile that
// its rows reference, ascending.  ext == nullptr: their count into cnt[t]
// (kTileHaloMax + 1 when more references than fit); else written to
// ext[off[t] ...].
__global__ void __launch_bounds__(256) tile_halo(int r0, int r1, const int *__restrict__ up,
                                                 const int *__restrict__ uj, const int *__restrict__ perm,
                                                 const int *__restrict__ inv, int *__restrict__ cnt,
                                                 const int *__restrict__ off, int *__restrict__ ext)
{
    __shared__ unsigned cand[kTileCand];
    __shared__ int ncand, part[257];
    const int t = blockIdx.x;
    const int w0 = r0 + t * kTileRows, w1 = min(r1, w0 + kTileRows);
    if (threadIdx.x == 0) ncand = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < w1 - w0; k += blockDim.x) {
        const int r = perm[w0 + k];
        for (int e = up[r]; e < up[r + 1]; e++) {
            const int c = inv[uj[e]];
            if (c < w0 || c >= w1) {
                const int p = atomicAdd(&ncand, 1);
                if (p < kTileCand) cand[p] = (unsigned)c;
            }
        }
    }
    __syncthreads();
    const int m = ncand;
    if (m > kTileCand) {
        if (threadIdx.x == 0 && !ext) cnt[t] = kTileHaloMax + 1;
        return;
    }
    int P = 1;
    while (P < m) P <<= 1;
    for (int k = m + threadIdx.x; k < P; k += blockDim.x) cand[k] = 0xFFFFFFFFu;
    __syncthreads();
    block_bitonic(cand, P);
    // first entry of each run of equal rows: count per thread chunk, scan
    const int chunk = (P + blockDim.x - 1) / blockDim.x;
    const int k0 = threadIdx.x * chunk, k1 = min(m, k0 + chunk);
    int mine = 0;
    for (int k = k0; k < k1; k++) mine += (k == 0 || cand[k] != cand[k - 1]);
    part[threadIdx.x + 1] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        part[0] = 0;
        for (int i = 1; i <= (int)blockDim.x; i++) part[i] += part[i - 1];
    }
    __syncthreads();
    if (!ext) {
        if (threadIdx.x == 0) cnt[t] = part[blockDim.x];
        return;
    }
    int o = off[t] + part[threadIdx.x];
    for (int k = k0; k < k1; k++)
        if (k == 0 || cand[k] != cand[k - 1]) ext[o++] = (int)cand[k];
}

// Packed slots (halo position << 16 | tuple id) of the rows of [r0, r1) in
// the SELL-32 slices sp; padding slots name the row itself with the zero tuple.
__global__ void tile_sell_fill(int r0, int r1, const int *__restrict__ up, const int *__restrict__ uj,
                               const int *__restrict__ tid, int zero_id, const int *__restrict__ sp,
                               const int *__restrict__ perm, const int *__restrict__ inv, const int *__restrict__ off,
                               const int *__restrict__ ext, unsigned *__restrict__ sell)
{
    const int s = blockIdx.x, lane = threadIdx.x;
    const int n = r1 - r0, r = s * 32 + lane;
    const int t = (s * 32) / kTileRows;
    const int w0 = r0 + t * kTileRows, w1 = min(r1, w0 + kTileRows);
    const int *ex = ext + off[t];
    const int ne = off[t + 1] - off[t];
    const int s0 = sp[s], s1 = sp[s + 1];
    const int o = r < n ? perm[r0 + r] : 0;
    const int a0 = r < n ? up[o] : 0, len = r < n ? up[o + 1] - a0 : 0;
    const unsigned own = r < n ? (unsigned)(r0 + r - w0) : 0u;
    for (int k = 0; k < s1 - s0; k++) {
        unsigned loc = own, id = (unsigned)zero_id;
        if (k < len) {
            const int c = inv[uj[a0 + k]];
            if (c >= w0 && c < w1) {
                loc = (unsigned)(c - w0);
            } else {
                int lo = 0, hi = ne;          // first external entry >= c (present by construction)
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (ex[mid] < c) lo = mid + 1;
                    else hi = mid;
                }
                loc = (unsigned)(w1 - w0 + lo);
            }
            id = (unsigned)tid[a0 + k];
        }
        sell[(size_t)(s0 + k) * 32 + lane] = (loc << 16) | id;
    }
}

}  // namespace

cudaError_t build_tiles(int r0, int r1, const int *d_up, const int *d_uj, const int *d_tid, int zero_id,
                        const int *d_perm, const int *d_inv, const int *d_slice, long long slots, int **d_off,
                        int **d_ext, unsigned **d_sell, int *halo_max, int *slots_max, cudaStream_t st)
{
    *d_off = nullptr;
    *d_ext = nullptr;
    *d_sell = nullptr;
    *halo_max = 0;
    *slots_max = 0;
    const int n = r1 - r0;
    if (n <= 0) return cudaSuccess;
    const int ntiles = (n + kTileRows - 1) / kTileRows, nsl = (n + 31) / 32;
    {
        // slot rows per tile, from the slice pointers
        std::vector<int> sp(nsl + 1);
        cudaError_t e0 = cudaMemcpyAsync(sp.data(), d_slice, sizeof(int) * (nsl + 1), cudaMemcpyDeviceToHost, st);
        if (e0 == cudaSuccess) e0 = cudaStreamSynchronize(st);
        if (e0 != cudaSuccess) return e0;
        constexpr int per = kTileRows / 32;
        for (int t = 0; t < ntiles; t++) *slots_max = std::max(*slots_max, sp[std::min(nsl, (t + 1) * per)] - sp[t * per]);
    }
    int *cnt = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&cnt, sizeof(int) * (ntiles + 1), st);
    if (e != cudaSuccess) return e;
    tile_halo<<<ntiles, 256, 0, st>>>(r0, r1, d_up, d_uj, d_perm, d_inv, cnt, nullptr, nullptr);
    e = cudaGetLastError();
    std::vector<int> h(ntiles);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), cnt, sizeof(int) * ntiles, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    int hmax = 0;
    for (int t = 0; t < ntiles && e == cudaSuccess; t++)
        hmax = std::max(hmax, std::min(kTileRows, n - t * kTileRows) + h[t]);
    if (e != cudaSuccess || hmax > kTileHaloMax) {
        cudaFreeAsync(cnt, st);
        *halo_max = e == cudaSuccess ? -1 : 0;
        return e;
    }
    e = keep_alloc(d_off, sizeof(int) * (ntiles + 1), st);
    if (e == cudaSuccess) e = exclusive_scan_int(cnt, *d_off, ntiles, st);
    int tot = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot, *d_off + ntiles, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = keep_alloc(d_ext, sizeof(int) * std::max(tot, 1), st);
    if (e == cudaSuccess) {
        tile_halo<<<ntiles, 256, 0, st>>>(r0, r1, d_up, d_uj, d_perm, d_inv, cnt, *d_off, *d_ext);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = keep_alloc(d_sell, sizeof(unsigned) * 32 * std::max<long long>(slots, 1), st);
    if (e == cudaSuccess) {
        tile_sell_fill<<<nsl, 32, 0, st>>>(r0, r1, d_up, d_uj, d_tid, zero_id, d_slice, d_perm, d_inv, *d_off,
                                           *d_ext, *d_sell);
        e = cudaGetLastError();
    }
    cudaFreeAsync(cnt, st);
    *halo_max = hmax;
    return e;
}

cudaError_t build_rec_geo(int n, const int *d_up, const double *d_ux, long long nnz, const int *d_perm,
                          const int *d_upp, const double *d_rho0, const float *d_recp, float **d_rec, cudaStream_t st)
{
    cudaError_t e = cudaMallocAsync((void **)d_rec, sizeof(float) * 8 * std::max<long long>(nnz, 1), st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(*d_rec, d_recp, sizeof(float) * 8 * nnz, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && n > 0) {
        rec_geo_fill<<<(n + 255) / 256, 256, 0, st>>>(n, d_up, d_ux, d_perm, d_upp, d_rho0, *d_rec);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t mass_row_sums_geo(int n, const int *d_up, const double *d_ux, const double *d_rho0, double *d_out,
                              cudaStream_t st)
{
    if (n > 0) row_sums_geo<<<(n + 255) / 256, 256, 0, st>>>(n, d_up, d_ux, d_rho0, d_out);
    return cudaGetLastError();
}

}  // namespace sfg
