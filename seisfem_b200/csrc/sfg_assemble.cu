// sfg_assemble.cu -- FP64 element assembly, lumped mass, M-PML profiles and
// COO -> canonical CSR on the GPU.
//
// Compiled with -fmad=false: no multiply-add contraction, so every FP64
// value reproduces the reference's scalar C loops bit for bit
// (assemble/*_sparse_*.c, pml/abc_mpml.c, sparse_matrix/coo2csr_lib.f90).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "sfg_elem.cuh"
#include "sfg_internal.h"
#include "sfg_mpml.cuh"

namespace sfg {

// ------------------------------------------------------------------ scan

namespace {
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long *sh, long long &total)
{
    // Hillis-Steele over one block (sh has blockDim.x entries)
    int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int off = 1; off < blockDim.x; off <<= 1) {
        long long a = t >= off ? sh[t - off] : 0;
        __syncthreads();
        sh[t] += a;
        __syncthreads();
    }
    total = sh[blockDim.x - 1];
    long long incl = sh[t];
    __syncthreads();
    return incl - v;
}

__global__ void scan_tile_sums(const int *in, int n, long long *tile_sum)
{
    __shared__ long long sh[SCAN_THREADS];
    long long base = (long long)blockIdx.x * SCAN_TILE;
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    long long tot;
    block_exclusive_scan(s, sh, tot);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

__global__ void scan_tile_offsets(long long *tile_sum, int ntiles)
{
    // one block: exclusive scan of the tile sums, in chunks of blockDim
    __shared__ long long sh[SCAN_THREADS];
    long long carry = 0;
    for (int base = 0; base < ntiles; base += SCAN_THREADS) {
        int i = base + threadIdx.x;
        long long v = i < ntiles ? tile_sum[i] : 0;
        long long tot;
        long long ex = block_exclusive_scan(v, sh, tot);
        if (i < ntiles) tile_sum[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sum[ntiles] = carry;
}

__global__ void scan_tiles(const int *in, int *out, int n, const long long *tile_off)
{
    // each thread owns SCAN_ITEMS consecutive items of the tile
    __shared__ long long sh[SCAN_THREADS];
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    long long tot;
    long long ex = block_exclusive_scan(s, sh, tot) + tile_off[blockIdx.x];
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + k;
        if (i < n) out[i] = (int)ex;
        ex += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = (int)tile_off[gridDim.x];
}
}  // namespace

// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total.
cudaError_t exclusive_scan_int(const int *d_in, int *d_out, int n, cudaStream_t st)
{
    int ntiles = std::max(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    long long *tile = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&tile, sizeof(long long) * (ntiles + 1), st);
    if (e != cudaSuccess) return e;
    scan_tile_sums<<<ntiles, SCAN_THREADS, 0, st>>>(d_in, n, tile);
    scan_tile_offsets<<<1, SCAN_THREADS, 0, st>>>(tile, ntiles);
    scan_tiles<<<ntiles, SCAN_THREADS, 0, st>>>(d_in, d_out, n, tile);
    e = cudaGetLastError();
    cudaFreeAsync(tile, st);
    return e;
}

// Lowest position k of an element_node entry outside [1, N] (atomicMin on
// *first, which the caller sets to all ones).
__global__ void element_node_check(const int *__restrict__ en, long long cnt, int N, unsigned long long *first)
{
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (long long)gridDim.x * blockDim.x)
        if (en[k] < 1 || en[k] > N) atomicMin(first, (unsigned long long)k);
}

cudaError_t check_element_nodes(const int *d_en, long long cnt, int N, long long *first_bad, cudaStream_t st)
{
    *first_bad = -1;
    unsigned long long *d_first = nullptr, h = ~0ull;
    cudaError_t e = tmp_alloc((void **)&d_first, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_first, 0xff, sizeof(unsigned long long), st);
    if (e == cudaSuccess && cnt > 0) {
        element_node_check<<<(unsigned)std::min<long long>((cnt + 255) / 256, 148 * 16), 256, 0, st>>>(d_en, cnt, N,
                                                                                                        d_first);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_first, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (d_first) cudaFreeAsync(d_first, st);
    if (e == cudaSuccess && h != ~0ull) *first_bad = (long long)h;
    return e;
}

// ------------------------------------------------------- element matrices

struct MatList { int m[8]; };   // -1: consistent mass (rho), 0..6: stiffness type

// Shape functions and their r/s derivatives at every quadrature point of the
// element type: tab[(3*q + c)*16 + k], c = 0 value, 1 d/dr, 2 d/ds.  They do
// not depend on the element, so they are evaluated once per set-up (same
// arithmetic as a per-element evaluation, hence the same bits).
__global__ void shape_table_kernel(int tc, double *tab)
{
    const int q = threadIdx.x;
    if (q >= quad_count(tc)) return;
    double r, s, w;
    quad_point(tc, q, r, s, w);
    double sv[16], sdr[16], sds[16];
    shape_eval(tc, r, s, sv, sdr, sds);
    const int p = elem_order(tc);
    for (int k = 0; k < p; k++) {
        tab[(3 * q + 0) * 16 + k] = sv[k];
        tab[(3 * q + 1) * 16 + k] = sdr[k];
        tab[(3 * q + 2) * 16 + k] = sds[k];
    }
}

// Element matrices as COO: entry e*p*p + iq*p + jq integrates the requested
// matrices in the reference's quadrature order (mass_sparse_q4.c:199-256,
// stiffness_sparse_q4.c:202-271).  A block holds EB elements; its first pass
// computes drdx, drdy, dsdx, dsdy and area * w of every (element, quadrature
// point) once into shared memory, the second pass forms every entry from
// them, one thread per entry.
__global__ void element_coo_shared(int tc, int p, int E, int EB, const int *__restrict__ en,
                                   const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ rho, int nmat, MatList ml,
                                   const double *__restrict__ tab, int *__restrict__ ci, int *__restrict__ cj,
                                   double *__restrict__ cx, int *flags)
{
    extern __shared__ double geo[];   // [EB][nq][5]: drdx drdy dsdx dsdy area*w
    const int pp = p * p, nq = quad_count(tc);
    const int e0 = blockIdx.x * EB;
    const int ne = min(EB, E - e0);
    for (int k = threadIdx.x; k < ne * nq; k += blockDim.x) {
        const int le = k / nq, q = k - le * nq, e = e0 + le;
        ElemGeom g;
        elem_geom(tc, en + (long long)e * p, x, y, g);
        if (g.area == 0.0 && q == 0) atomicOr(flags, FLAG_ZERO_AREA);
        double r, s, w;
        quad_point(tc, q, r, s, w);
        double *o = geo + (size_t)k * 5;
        map_point(tc, g, r, s, o[0], o[1], o[2], o[3]);
        o[4] = g.area * w;
    }
    __syncthreads();
    const long long nnz = (long long)E * pp;
    for (int k = threadIdx.x; k < ne * pp; k += blockDim.x) {
        const int le = k / pp, rem = k - le * pp, iq = rem / p, jq = rem - iq * p;
        const int e = e0 + le;
        const long long t = (long long)e * pp + rem;
        const int *enE = en + (long long)e * p;
        const int ip = enE[iq] - 1, jp = enE[jq] - 1;
        const double rho_ip = rho ? rho[ip] : 0.0;
        double acc[8];
#pragma unroll
        for (int m = 0; m < 8; m++) acc[m] = 0.0;
        for (int q = 0; q < nq; q++) {
            const double *gq = geo + ((size_t)le * nq + q) * 5;
            const double drdx = gq[0], drdy = gq[1], dsdx = gq[2], dsdy = gq[3], aw = gq[4];
            const double *t0 = tab + 3 * q * 16, *t1 = t0 + 16, *t2 = t0 + 32;
            double phi_i = t0[iq], phi_j = t0[jq];
            double dxi = t1[iq] * drdx + t2[iq] * dsdx;
            double dyi = t1[iq] * drdy + t2[iq] * dsdy;
            double dxj = t1[jq] * drdx + t2[jq] * dsdx;
            double dyj = t1[jq] * drdy + t2[jq] * dsdy;
            for (int m = 0; m < nmat; m++) {
                double term;
                switch (ml.m[m]) {
                case -1: term = aw * rho_ip * phi_i * phi_j; break;
                case 0: term = aw * (dxi * dxj + dyi * dyj); break;
                case 1: term = aw * (dxi * dxj); break;
                case 2: term = aw * (dyi * dyj); break;
                case 3: term = aw * (dxi * dyj); break;
                case 4: term = aw * (dyi * dxj); break;
                case 5: term = aw * (phi_i * dxj); break;
                default: term = aw * (phi_i * dyj); break;
                }
                acc[m] = acc[m] + term;
            }
        }
        if (ci) ci[t] = ip;
        if (cj) cj[t] = jp;
        for (int m = 0; m < nmat; m++) cx[(long long)m * nnz + t] = acc[m];
    }
}

// The same entries for the set-up's seven matrices (consistent mass, then
// stiffness types 1..6) with the element type known at compile time: the
// quadrature and matrix loops unroll, and the shape table sits in shared
// memory.  Every term and sum is the one element_coo_shared forms, in the
// same order (this file is compiled without FMA contraction), so the bits
// are the same.
template <int TC>
__global__ void __launch_bounds__(256) element_coo_std7(int E, int EB, const int *__restrict__ en,
                                                        const double *__restrict__ x, const double *__restrict__ y,
                                                        const double *__restrict__ rho,
                                                        const double *__restrict__ tab, int *__restrict__ ci,
                                                        int *__restrict__ cj, double *__restrict__ cx, int *flags)
{
    constexpr int P = elem_order(TC), PP = P * P, NQ = quad_count(TC);
    __shared__ double stab[NQ * 48];
    extern __shared__ double geo[];   // [EB][NQ][5]: drdx drdy dsdx dsdy area*w
    for (int k = threadIdx.x; k < NQ * 48; k += blockDim.x) stab[k] = tab[k];
    const int e0 = blockIdx.x * EB;
    const int ne = min(EB, E - e0);
    for (int k = threadIdx.x; k < ne * NQ; k += blockDim.x) {
        const int le = k / NQ, q = k - le * NQ, e = e0 + le;
        ElemGeom g;
        elem_geom(TC, en + (long long)e * P, x, y, g);
        if (g.area == 0.0 && q == 0) atomicOr(flags, FLAG_ZERO_AREA);
        double r, s, w;
        quad_point(TC, q, r, s, w);
        double *o = geo + (size_t)k * 5;
        map_point(TC, g, r, s, o[0], o[1], o[2], o[3]);
        o[4] = g.area * w;
    }
    __syncthreads();
    const long long nnz = (long long)E * PP;
    for (int k = threadIdx.x; k < ne * PP; k += blockDim.x) {
        const int le = k / PP, rem = k - le * PP, iq = rem / P, jq = rem - iq * P;
        const int e = e0 + le;
        const long long t = (long long)e * PP + rem;
        const int *enE = en + (long long)e * P;
        const int ip = enE[iq] - 1, jp = enE[jq] - 1;
        const double rho_ip = rho[ip];
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0, a6 = 0.0;
        const double *gq = geo + (size_t)le * NQ * 5;
#pragma unroll 4
        for (int q = 0; q < NQ; q++, gq += 5) {
            const double drdx = gq[0], drdy = gq[1], dsdx = gq[2], dsdy = gq[3], aw = gq[4];
            const double *t0 = stab + 3 * q * 16, *t1 = t0 + 16, *t2 = t0 + 32;
            const double phi_i = t0[iq], phi_j = t0[jq];
            const double dxi = t1[iq] * drdx + t2[iq] * dsdx;
            const double dyi = t1[iq] * drdy + t2[iq] * dsdy;
            const double dxj = t1[jq] * drdx + t2[jq] * dsdx;
            const double dyj = t1[jq] * drdy + t2[jq] * dsdy;
            a0 = a0 + aw * rho_ip * phi_i * phi_j;
            a1 = a1 + aw * (dxi * dxj);
            a2 = a2 + aw * (dyi * dyj);
            a3 = a3 + aw * (dxi * dyj);
            a4 = a4 + aw * (dyi * dxj);
            a5 = a5 + aw * (phi_i * dxj);
            a6 = a6 + aw * (phi_i * dyj);
        }
        ci[t] = ip;
        cj[t] = jp;
        cx[t] = a0;
        cx[nnz + t] = a1;
        cx[2 * nnz + t] = a2;
        cx[3 * nnz + t] = a3;
        cx[4 * nnz + t] = a4;
        cx[5 * nnz + t] = a5;
        cx[6 * nnz + t] = a6;
    }
}

cudaError_t launch_element_coo(int tc, int E, const int *d_en, const double *d_x, const double *d_y,
                               const double *d_rho, int nmat, const int *mats, int *d_ci, int *d_cj,
                               double *d_cx, int *d_flags, cudaStream_t st)
{
    int p = elem_order(tc);
    long long nnz = (long long)E * p * p;
    MatList ml;
    for (int m = 0; m < 8; m++) ml.m[m] = m < nmat ? mats[m] : 0;
    double *tab = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&tab, sizeof(double) * 36 * 3 * 16, st);
    if (e != cudaSuccess) return e;
    shape_table_kernel<<<1, 64, 0, st>>>(tc, tab);
    const int threads = 256, pp = p * p, nq = quad_count(tc);
    const int EB = std::max(1, threads / pp);
    const long long blocks = ((long long)E + EB - 1) / EB;
    const size_t smem = sizeof(double) * 5 * (size_t)EB * nq;
    const bool std7 = nmat == 7 && d_rho && d_ci && d_cj && mats[0] == -1 && mats[1] == 1 && mats[2] == 2 &&
                      mats[3] == 3 && mats[4] == 4 && mats[5] == 5 && mats[6] == 6;
    if (blocks > 0 && std7) {
        switch (tc) {
#define SFG_STD7(T) case T: element_coo_std7<T><<<(unsigned)blocks, threads, smem, st>>>(E, EB, d_en, d_x, d_y, \
                        d_rho, tab, d_ci, d_cj, d_cx, d_flags); break;
        SFG_STD7(T3) SFG_STD7(T6) SFG_STD7(T10) SFG_STD7(Q4) SFG_STD7(Q9) SFG_STD7(Q16)
#undef SFG_STD7
        default: break;
        }
    } else if (blocks > 0)
        element_coo_shared<<<(unsigned)blocks, threads, smem, st>>>(tc, p, E, EB, d_en, d_x, d_y, d_rho, nmat,
                                                                     ml, tab, d_ci, d_cj, d_cx, d_flags);
    e = cudaGetLastError();
    cudaFreeAsync(tab, st);
    return e;
}

// ------------------------------------------------------------ lumped mass

// Per element: the sums of all mass terms and of the diagonal terms, each in
// the element's own (quad, iq, jq) order (mass_sparse_q4.c:238-246).
__global__ void element_mass_sums(int tc, int p, int E, const int *__restrict__ en,
                                  const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ rho, const double *__restrict__ tab,
                                  double *__restrict__ part)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int *enE = en + (long long)e * p;
    ElemGeom g;
    elem_geom(tc, enE, x, y, g);
    double ms = 0.0, ds = 0.0;
    int nq = quad_count(tc);
    for (int q = 0; q < nq; q++) {
        double r, s, w;
        quad_point(tc, q, r, s, w);
        const double *sv = tab + 3 * q * 16;
        double aw = g.area * w;
        for (int iq = 0; iq < p; iq++) {
            int ip = enE[iq] - 1;
            double a = aw * rho[ip];
            for (int jq = 0; jq < p; jq++) {
                double term = a * sv[iq] * sv[jq];
                ms = ms + term;
                if (enE[jq] - 1 == ip) ds = ds + term;
            }
        }
    }
    part[2 * (long long)e] = ms;
    part[2 * (long long)e + 1] = ds;
}

// Deterministic reduction of the per-element sums: fixed chunking per
// thread, then a fixed-shape tree (one block).
__global__ void reduce_pairs(const double *__restrict__ part, int E, double *out2)
{
    __shared__ double sm[1024], sd[1024];
    int t = threadIdx.x;
    long long chunk = ((long long)E + blockDim.x - 1) / blockDim.x;
    long long a = t * chunk, b = min((long long)E, a + chunk);
    double ms = 0.0, ds = 0.0;
    for (long long e = a; e < b; e++) { ms = ms + part[2 * e]; ds = ds + part[2 * e + 1]; }
    sm[t] = ms;
    sd[t] = ds;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (t < off) { sm[t] = sm[t] + sm[t + off]; sd[t] = sd[t] + sd[t + off]; }
        __syncthreads();
    }
    if (t == 0) { out2[0] = sm[0]; out2[1] = sd[0]; }
}

// Per node: the diagonal mass terms in (element, quad) order; the node's COO
// row lists its entries in ascending COO index, i.e. by element.
__global__ void node_lumped_mass(int tc, int p, int N, const int *__restrict__ en,
                                 const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ rho, const int *__restrict__ row_start,
                                 const int *__restrict__ bucket, const int *__restrict__ cj,
                                 const double *__restrict__ sums, const double *__restrict__ tab,
                                 double *__restrict__ mass)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    int pp = p * p;
    double m = 0.0;
    int nq = quad_count(tc);
    // the row's COO entries ascend, in runs of p: row iq of each element
    // that holds node r (entries e pp + iq p + j, j = 0 .. p-1); its
    // diagonal entry is the run's iq-th
    for (int k = row_start[r]; k < row_start[r + 1]; k += p) {
        const int c0 = bucket[k];
        const int e0 = c0 / pp, iq0 = (c0 - e0 * pp) / p;
        const int c = c0 + iq0;
        if (cj[c] != r) continue;
        int e = c / pp, rem = c - e * pp, iq = rem / p, jq = rem - iq * p;
        const int *enE = en + (long long)e * p;
        ElemGeom g;
        elem_geom(tc, enE, x, y, g);
        for (int q = 0; q < nq; q++) {
            double rr, ss, w;
            quad_point(tc, q, rr, ss, w);
            const double *sv = tab + 3 * q * 16;
            m = m + g.area * w * rho[r] * sv[iq] * sv[jq];
        }
    }
    // mass_sparse_q4.c:259-263
    mass[r] = m * sums[0] / sums[1];
}

cudaError_t launch_lumped_mass(int tc, int N, int E, const int *d_en, const double *d_x,
                               const double *d_y, const double *d_rho, const int *d_row_start,
                               const int *d_bucket, const int *d_cj, double *d_mass,
                               double *d_scratch, int *d_flags, cudaStream_t st)
{
    (void)d_flags;
    int p = elem_order(tc);
    double *tab = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&tab, sizeof(double) * 36 * 3 * 16, st);
    if (e != cudaSuccess) return e;
    shape_table_kernel<<<1, 64, 0, st>>>(tc, tab);
    element_mass_sums<<<(E + 127) / 128, 128, 0, st>>>(tc, p, E, d_en, d_x, d_y, d_rho, tab, d_scratch);
    double *sums = d_scratch + 2 * (size_t)E;
    reduce_pairs<<<1, 1024, 0, st>>>(d_scratch, E, sums);
    node_lumped_mass<<<(N + 127) / 128, 128, 0, st>>>(tc, p, N, d_en, d_x, d_y, d_rho, d_row_start,
                                                       d_bucket, d_cj, sums, tab, d_mass);
    e = cudaGetLastError();
    cudaFreeAsync(tab, st);
    return e;
}

// ------------------------------------------------------------------ M-PML

// One thread per node, region tests in the reference's order
// (pml/abc_mpml.c:73-199).  d0x/d0y come from the host (log10 of the host
// library, abc_mpml.c:60-61).  Nodes that no element references keep 0.
__global__ void mpml_kernel(int N, const double *__restrict__ xa, const double *__restrict__ ya,
                            const int *__restrict__ row_start, double d0x, double d0y, double tx,
                            double ty, double x0, double x1, double y0, double y1, int uxmin,
                            int uxmax, int uymin, int uymax, double *__restrict__ out)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double pxy = 0.15, pyx = 0.15;
    double vdx = 0.0, vdy = 0.0, vdxx = 0.0, vdyy = 0.0;
    if (row_start == nullptr || row_start[p + 1] > row_start[p])
        mpml_profile(xa[p], ya[p], d0x, d0y, tx, ty, x0, x1, y0, y1, uxmin, uxmax, uymin, uymax, vdx, vdy, vdxx,
                     vdyy);
    out[p] = vdx;
    out[(size_t)N + p] = vdy;
    out[2 * (size_t)N + p] = vdxx;
    out[3 * (size_t)N + p] = vdyy;
    out[4 * (size_t)N + p] = pyx * vdxx;
    out[5 * (size_t)N + p] = pxy * vdyy;
}

cudaError_t launch_mpml(int N, const double *d_x, const double *d_y, const int *d_row_start,
                        double d0x, double d0y, double tx, double ty, double x0, double x1,
                        double y0, double y1, int uxmin, int uxmax, int uymin, int uymax,
                        double *d_out6, cudaStream_t st)
{
    mpml_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, d_x, d_y, d_row_start, d0x, d0y, tx, ty, x0, x1, y0,
                                                  y1, uxmin, uxmax, uymin, uymax, d_out6);
    return cudaGetLastError();
}

// ------------------------------------------------------- COO -> CSR rows

__global__ void row_count_kernel(const int *__restrict__ ci, long long nnz, int N, int *cnt, int *flags)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    int r = ci[k];
    if (r < 0 || r >= N) { atomicOr(flags, FLAG_BADINDEX); return; }
    atomicAdd(&cnt[r], 1);
}

__global__ void row_fill_kernel(const int *__restrict__ ci, long long nnz, int N,
                                const int *__restrict__ row_start, int *cursor, int *bucket)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    int r = ci[k];
    if (r < 0 || r >= N) return;
    int pos = atomicAdd(&cursor[r], 1);
    bucket[row_start[r] + pos] = (int)k;
}

// selection sort with Fortran minloc semantics (coo2csr_lib.f90:256-267)
__device__ void interchange_sort_dev(int *v, int *m, int n)
{
    for (int i = 0; i < n - 1; i++) {
        int best = i, bv = v[i];
        for (int k = i + 1; k < n; k++) {
            int vk = v[k];
            if (vk < bv) { best = k; bv = vk; }
        }
        if (best != i) {
            int t = v[i]; v[i] = v[best]; v[best] = t;
            t = m[i]; m[i] = m[best]; m[best] = t;
        }
    }
}

// iargsort_quicksort (coo2csr_lib.f90:191-246) on vec/map[0..n); returns
// false when its explicit stack or a scan would leave the segment.
__device__ bool iargsort_dev(int *vec, int *map, int n)
{
    constexpr int LEVELS = 64, SMALL = 20;
    int lb[LEVELS + 1], ub[LEVELS + 1];
    if (n <= 0) return true;
    int sp = 0;
    lb[0] = 0;
    ub[0] = n - 1;
    while (sp >= 0) {
        int left = lb[sp], right = ub[sp];
        if (right - left < SMALL) {
            if (left < right) interchange_sort_dev(vec + left, map + left, right - left + 1);
            sp--;
            continue;
        }
        int lo = left, hi = right;
        int pivot = (vec[left] + vec[right]) / 2;
        left--;
        right++;
        for (;;) {
            do { left++; } while (left <= hi && vec[left] < pivot);
            do { right--; } while (right >= lo && vec[right] > pivot);
            if (left > hi || right < lo) return false;
            if (left < right) {
                int t = vec[left]; vec[left] = vec[right]; vec[right] = t;
                t = map[left]; map[left] = map[right]; map[right] = t;
            } else if (left == right) {
                if (left == lb[sp]) left++; else right--;
                break;
            } else {
                break;
            }
        }
        if (sp + 1 > LEVELS) return false;
        ub[sp + 1] = ub[sp];
        lb[sp + 1] = left;
        ub[sp] = right;
        sp++;
    }
    return true;
}

// Pass 1, one thread per row: restore COO order inside the row (the bucket
// was filled with atomics) and replay the Fortran sort (vec = column + 1,
// map = the permutation of the row's entries).
__global__ void canon_pass1(int N, long long nnz, const int *__restrict__ row_start, int *__restrict__ bucket,
                            const int *__restrict__ cj, int *__restrict__ vec, int *__restrict__ map, int *maxlen,
                            int *flags)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    int r1 = row_start[r], r2 = row_start[r + 1], l = r2 - r1;
    int *b = bucket + r1;
    for (int i = 1; i < l; i++) {   // insertion sort of COO indices
        int key = b[i], k = i - 1;
        while (k >= 0 && b[k] > key) { b[k + 1] = b[k]; k--; }
        b[k + 1] = key;
    }
    int *v = vec + r1, *m = map + r1;
    for (int i = 0; i < l; i++) { v[i] = cj[b[i]] + 1; m[i] = i; }
    if (!iargsort_dev(v, m, l)) { atomicOr(flags, FLAG_SORT_STACK); return; }
    atomicMax(maxlen, l);
}

// Pass 2, one warp per row: each run of equal columns in the sorted row is
// one union entry u, summed by the lane that holds the run's first position,
// in the sorted order (coo2csr_lib.f90's accumulation, so the sums round the
// same).  The sums go to row-local scratch (tx[s][row_start + u], tc), and
// the row's union length and per-stream nonzero counts to cnt_union, cnt_v.
__global__ void canon_sums(int N, int nv, long long nnz, const int *__restrict__ row_start,
                           const int *__restrict__ bucket, const double *__restrict__ cx,
                           const int *__restrict__ vec, const int *__restrict__ map, int *__restrict__ tc,
                           double *__restrict__ tx, int *__restrict__ cnt_union, int *__restrict__ cnt_v)
{
    const int lane = threadIdx.x & 31;
    const long long wr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wr >= N) return;
    const int r = (int)wr;
    const int r1 = row_start[r], l = row_start[r + 1] - r1;
    const int *b = bucket + r1, *v = vec + r1, *m = map + r1;
    int base = 0;
    int nz[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k0 = 0; k0 < l; k0 += 32) {
        const int k = k0 + lane;
        const int col = k < l ? v[k] : 0;
        const bool start = k < l && (k == 0 || v[k - 1] != col);
        const unsigned mask = __ballot_sync(0xffffffffu, start);
        if (start) {
            const int u = base + __popc(mask & ((1u << lane) - 1u));
            double xs[8];
            for (int s = 0; s < nv; s++) xs[s] = cx[(long long)s * nnz + b[m[k]]];
            for (int kk = k + 1; kk < l && v[kk] == col; kk++)
                for (int s = 0; s < nv; s++) xs[s] = xs[s] + cx[(long long)s * nnz + b[m[kk]]];
            tc[r1 + u] = col - 1;
            for (int s = 0; s < nv; s++) {
                tx[(long long)s * nnz + r1 + u] = xs[s];
                nz[s] += (xs[s] != 0.0);
            }
        }
        base += __popc(mask);
    }
    for (int s = 0; s < nv; s++) {
        int c = nz[s];
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt_v[(long long)s * N + r] = c;
    }
    if (lane == 0) cnt_union[r] = base;
}

// Pass 3, one warp per row: the union pattern and every stream's canonical
// CSR (its nonzero sums, in column order) from the row-local scratch.
__global__ void canon_pass2(int N, int nv, long long nnz, const int *__restrict__ row_start,
                            const int *__restrict__ tc, const double *__restrict__ tx,
                            const int *__restrict__ cnt_union, const int *__restrict__ up, int *__restrict__ uj,
                            double *__restrict__ ux, long long union_nnz, int *const *__restrict__ vp_,
                            int *const *__restrict__ vj_, double *const *__restrict__ vx_)
{
    const int lane = threadIdx.x & 31;
    const long long wr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wr >= N) return;
    const int r = (int)wr;
    const int r1 = row_start[r], nu = cnt_union[r];
    if (uj) {
        const long long uo = up[r];
        for (int u = lane; u < nu; u += 32) {
            uj[uo + u] = tc[r1 + u];
            for (int s = 0; s < nv; s++) ux[(long long)s * union_nnz + uo + u] = tx[(long long)s * nnz + r1 + u];
        }
    }
    for (int s = 0; s < nv; s++) {
        if (!vj_[s]) continue;
        int vo = vp_[s][r];
        for (int u0 = 0; u0 < nu; u0 += 32) {
            const int u = u0 + lane;
            const double x = u < nu ? tx[(long long)s * nnz + r1 + u] : 0.0;
            const bool keep = u < nu && x != 0.0;
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int o = vo + __popc(mask & ((1u << lane) - 1u));
                vj_[s][o] = tc[r1 + u];
                vx_[s][o] = x;
            }
            vo += __popc(mask);
        }
    }
}

// Nonzeros of each stream: blocks (b, s) stride over cnt_v[s][0 .. N) and
// add their sums to tot[s] (zeroed by the caller).
__global__ void __launch_bounds__(256) count_totals(int N, const int *__restrict__ cnt_v,
                                                    unsigned long long *__restrict__ tot)
{
    __shared__ long long red[8];
    const int s = blockIdx.y;
    long long c = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x)
        c += cnt_v[(long long)s * N + r];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        atomicAdd(&tot[s], (unsigned long long)t);
    }
}

// One warp per row: the nonzero union entries of every stream.
__global__ void union_nz_count(int N, int nv, const int *__restrict__ up, const double *__restrict__ ux,
                               long long union_nnz, int *__restrict__ cnt_v)
{
    const int lane = threadIdx.x & 31;
    const long long wr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wr >= N) return;
    const int r = (int)wr;
    const long long u0 = up[r];
    const int nu = up[r + 1] - (int)u0;
    for (int s = 0; s < nv; s++) {
        int c = 0;
        for (int u = lane; u < nu; u += 32) c += ux[(long long)s * union_nnz + u0 + u] != 0.0;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt_v[(long long)s * N + r] = c;
    }
}

// One warp per row: each stream's CSR row, its nonzero union entries in order.
__global__ void union_to_csr(int N, int nv, const int *__restrict__ up, const int *__restrict__ uj,
                             const double *__restrict__ ux, long long union_nnz, int *const *__restrict__ vp_,
                             int *const *__restrict__ vj_, double *const *__restrict__ vx_)
{
    const int lane = threadIdx.x & 31;
    const long long wr = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wr >= N) return;
    const int r = (int)wr;
    const long long u0 = up[r];
    const int nu = up[r + 1] - (int)u0;
    for (int s = 0; s < nv; s++) {
        int vo = vp_[s][r];
        for (int k0 = 0; k0 < nu; k0 += 32) {
            const int u = k0 + lane;
            const double x = u < nu ? ux[(long long)s * union_nnz + u0 + u] : 0.0;
            const bool keep = u < nu && x != 0.0;
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int o = vo + __popc(mask & ((1u << lane) - 1u));
                vj_[s][o] = uj[u0 + u];
                vx_[s][o] = x;
            }
            vo += __popc(mask);
        }
    }
}

#define SFG_TRY(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) { err = cudaGetErrorString(e_); return SFG_ERR_CUDA; } \
    } while (0)

void canon_free(CanonOut &o, bool keep_csr, cudaStream_t st)
{
    if (!keep_csr)
        for (auto &c : o.csr) { keep_free(c.p, st); keep_free(c.j, st); keep_free(c.x, st); c = DevCsr(); }
    if (o.row_start) cudaFreeAsync(o.row_start, st);
    if (o.bucket) cudaFreeAsync(o.bucket, st);
    o.row_start = nullptr;
    o.bucket = nullptr;
}

int canonicalize(int N, long long nnz, const int *d_ci, const int *d_cj, const double *d_cx, int nv,
                 bool want_union, bool want_csr, CanonOut &out, int *d_flags, cudaStream_t st,
                 std::string &err)
{
    if (nv < 1 || nv > 8 || nnz >= (1LL << 31) || N < 0) { err = "canonicalize: bad sizes"; return SFG_ERR_ARG; }
    int *cnt = nullptr, *cursor = nullptr, *vec = nullptr, *map = nullptr, *cu = nullptr,
        *cv = nullptr, *maxlen = nullptr, *tc = nullptr;
    double *tx = nullptr;
    size_t nn = (size_t)std::max<long long>(nnz, 1);
    const bool sums = want_union || want_csr;
    // temporaries (row buckets included) come from the device's pool
    SFG_TRY(tmp_alloc((void **)&cnt, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(tmp_alloc((void **)&cursor, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(tmp_alloc((void **)&out.row_start, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(tmp_alloc((void **)&out.bucket, sizeof(int) * nn, st));
    SFG_TRY(tmp_alloc((void **)&vec, sizeof(int) * nn, st));
    SFG_TRY(tmp_alloc((void **)&map, sizeof(int) * nn, st));
    SFG_TRY(tmp_alloc((void **)&cu, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(tmp_alloc((void **)&cv, sizeof(int) * (size_t)nv * ((size_t)N + 1), st));
    SFG_TRY(tmp_alloc((void **)&maxlen, sizeof(int), st));
    if (sums) {
        SFG_TRY(tmp_alloc((void **)&tc, sizeof(int) * nn, st));
        SFG_TRY(tmp_alloc((void **)&tx, sizeof(double) * (size_t)nv * nn, st));
    }
    SFG_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(cudaMemsetAsync(cursor, 0, sizeof(int) * ((size_t)N + 1), st));
    SFG_TRY(cudaMemsetAsync(maxlen, 0, sizeof(int), st));
    int tb = 256;
    unsigned gb = (unsigned)((nnz + tb - 1) / tb);
    if (gb) row_count_kernel<<<gb, tb, 0, st>>>(d_ci, nnz, N, cnt, d_flags);
    SFG_TRY(exclusive_scan_int(cnt, out.row_start, N, st));
    if (gb) row_fill_kernel<<<gb, tb, 0, st>>>(d_ci, nnz, N, out.row_start, cursor, out.bucket);
    unsigned gr = (unsigned)((N + 127) / 128);
    const unsigned gw = (unsigned)(((long long)N * 32 + 255) / 256);   // one warp per row
    if (gr) canon_pass1<<<gr, 128, 0, st>>>(N, nnz, out.row_start, out.bucket, d_cj, vec, map, maxlen, d_flags);
    if (gw && sums)
        canon_sums<<<gw, 256, 0, st>>>(N, nv, nnz, out.row_start, out.bucket, d_cx, vec, map, tc, tx, cu, cv);
    SFG_TRY(cudaGetLastError());
    int hflags = 0;
    SFG_TRY(cudaMemcpyAsync(&hflags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    SFG_TRY(cudaMemcpyAsync(&out.max_row_len, maxlen, sizeof(int), cudaMemcpyDeviceToHost, st));
    SFG_TRY(cudaStreamSynchronize(st));
    auto free_tmp = [&]() {
        for (void *t : {(void *)cnt, (void *)cursor, (void *)vec, (void *)map, (void *)cu, (void *)cv,
                        (void *)maxlen, (void *)tc, (void *)tx})
            if (t) cudaFreeAsync(t, st);
    };
    if (hflags & FLAG_BADINDEX) { free_tmp(); err = "COO row index out of range"; return SFG_ERR_BADINDEX; }
    if (hflags & FLAG_SORT_STACK) { free_tmp(); err = "row too long for the device sorter"; return SFG_ERR_ROWLEN; }

    // nonzeros of each stream (the CSR arrays themselves only with want_csr)
    long long *d_tot = nullptr;
    if (sums && !want_csr) {
        SFG_TRY(tmp_alloc((void **)&d_tot, sizeof(long long) * 8, st));
        SFG_TRY(cudaMemsetAsync(d_tot, 0, sizeof(long long) * 8, st));
        if (N > 0)
            count_totals<<<dim3((unsigned)std::min((N + 255) / 256, 128), nv), 256, 0, st>>>(
                N, cv, reinterpret_cast<unsigned long long *>(d_tot));
        SFG_TRY(cudaGetLastError());
        SFG_TRY(cudaMemcpyAsync(out.nnz_v, d_tot, sizeof(long long) * nv, cudaMemcpyDeviceToHost, st));
    }
    // row pointers: union + each stream
    int *up = nullptr;
    if (want_union) {
        SFG_TRY(keep_alloc(&up, sizeof(int) * ((size_t)N + 1), st));
        SFG_TRY(exclusive_scan_int(cu, up, N, st));
        int tot = 0;
        SFG_TRY(cudaMemcpyAsync(&tot, up + N, sizeof(int), cudaMemcpyDeviceToHost, st));
        SFG_TRY(cudaStreamSynchronize(st));
        out.union_nnz = tot;
        out.up = up;
        SFG_TRY(keep_alloc(&out.uj, sizeof(int) * std::max<size_t>(tot, 1), st));
        SFG_TRY(keep_alloc(&out.ux, sizeof(double) * (size_t)nv * std::max<size_t>(tot, 1), st));
    }
    int *dvp[8] = {nullptr}, *dvj[8] = {nullptr};
    double *dvx[8] = {nullptr};
    if (want_csr) {
        for (int s = 0; s < nv; s++) {
            DevCsr &c = out.csr[s];
            SFG_TRY(keep_alloc(&c.p, sizeof(int) * ((size_t)N + 1), st));
            SFG_TRY(exclusive_scan_int(cv + (size_t)s * N, c.p, N, st));
            int tot = 0;
            SFG_TRY(cudaMemcpyAsync(&tot, c.p + N, sizeof(int), cudaMemcpyDeviceToHost, st));
            SFG_TRY(cudaStreamSynchronize(st));
            c.nnz = tot;
            out.nnz_v[s] = tot;
            SFG_TRY(keep_alloc(&c.j, sizeof(int) * std::max<size_t>(tot, 1), st));
            SFG_TRY(keep_alloc(&c.x, sizeof(double) * std::max<size_t>(tot, 1), st));
            dvp[s] = c.p; dvj[s] = c.j; dvx[s] = c.x;
        }
    }
    int **d_tab = nullptr;
    SFG_TRY(tmp_alloc((void **)&d_tab, sizeof(void *) * 24, st));
    void *htab[24];
    for (int s = 0; s < 8; s++) { htab[s] = dvp[s]; htab[8 + s] = dvj[s]; htab[16 + s] = dvx[s]; }
    SFG_TRY(cudaMemcpyAsync(d_tab, htab, sizeof(htab), cudaMemcpyHostToDevice, st));
    if (gw && sums)
        canon_pass2<<<gw, 256, 0, st>>>(N, nv, nnz, out.row_start, tc, tx, cu, out.up, out.uj, out.ux,
                                        out.union_nnz, d_tab, d_tab + 8, (double *const *)(d_tab + 16));
    SFG_TRY(cudaGetLastError());
    SFG_TRY(cudaStreamSynchronize(st));
    cudaFreeAsync(d_tab, st);
    if (d_tot) cudaFreeAsync(d_tot, st);
    free_tmp();
    return SFG_OK;
}

int csr_from_union(int N, int nv, const int *d_up, const int *d_uj, const double *d_ux, long long union_nnz,
                   DevCsr *out, cudaStream_t st, std::string &err)
{
    if (nv < 1 || nv > 8 || N < 0) { err = "csr_from_union: bad sizes"; return SFG_ERR_ARG; }
    int *cv = nullptr, **d_tab = nullptr;
    long long tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    SFG_TRY(tmp_alloc((void **)&cv, sizeof(int) * (size_t)nv * ((size_t)N + 1), st));
    const unsigned gw = (unsigned)(((long long)N * 32 + 255) / 256);
    if (gw) union_nz_count<<<gw, 256, 0, st>>>(N, nv, d_up, d_ux, union_nnz, cv);
    SFG_TRY(cudaGetLastError());
    for (int s = 0; s < nv; s++) {
        SFG_TRY(keep_alloc(&out[s].p, sizeof(int) * ((size_t)N + 1), st));
        SFG_TRY(exclusive_scan_int(cv + (size_t)s * N, out[s].p, N, st));
    }
    int htot[8];
    for (int s = 0; s < nv; s++)
        SFG_TRY(cudaMemcpyAsync(&htot[s], out[s].p + N, sizeof(int), cudaMemcpyDeviceToHost, st));
    SFG_TRY(cudaStreamSynchronize(st));
    void *htab[24] = {nullptr};
    for (int s = 0; s < nv; s++) {
        tot[s] = htot[s];
        out[s].nnz = tot[s];
        SFG_TRY(keep_alloc(&out[s].j, sizeof(int) * std::max<long long>(tot[s], 1), st));
        SFG_TRY(keep_alloc(&out[s].x, sizeof(double) * std::max<long long>(tot[s], 1), st));
        htab[s] = out[s].p; htab[8 + s] = out[s].j; htab[16 + s] = out[s].x;
    }
    SFG_TRY(tmp_alloc((void **)&d_tab, sizeof(void *) * 24, st));
    SFG_TRY(cudaMemcpyAsync(d_tab, htab, sizeof(htab), cudaMemcpyHostToDevice, st));
    if (gw) union_to_csr<<<gw, 256, 0, st>>>(N, nv, d_up, d_uj, d_ux, union_nnz, d_tab, d_tab + 8,
                                             (double *const *)(d_tab + 16));
    SFG_TRY(cudaGetLastError());
    SFG_TRY(cudaStreamSynchronize(st));
    cudaFreeAsync(d_tab, st);
    cudaFreeAsync(cv, st);
    return SFG_OK;
}

}  // namespace sfg
