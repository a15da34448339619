// sfg_acoustic.cu -- the scalar acoustic solvers on the GPU:
//   time_evolution/acoustic.c:1-223      (no absorbing boundary)
//   time_evolution/acoustic_pml.c:3-485  (split-field classical PML)
// with solver "masslump".
//
// Set-up reuses the elastic path's device assembly: element matrices (M with
// density 1 -- the two files call mass_sparse_all without a density -- and
// stiffness type 0, or types 1, 5, 2, 6 with PML), the canonical CSR per
// matrix (bit-exact with coo2csr_lib.f90), their union pattern with explicit
// zeros, and the lumped mass.  The PML profile (pml/abc_pml.c:41-103) is
// formed on the host, like the M-PML of the elastic path.
//
// The time loop is one fused FP64 kernel per step, captured in a CUDA graph:
// every product of the step (3 without PML, 10 with) is summed per row in the
// canonical column order from 0.0 (sparse_matrix/csr_matvec.c:7-16), the
// right-hand sides are evaluated in the reference's expression order, and the
// lumped solve divides (this unit is compiled with -fmad=false).  An explicit
// zero of the union pattern adds +-0 to a row sum, which leaves it unchanged,
// so the results equal the reference's per-matrix CSR products bit for bit.
//
// Layout in HBM: the union pattern in SELL-32 slices of 32 consecutive rows
// (mesh order), slot k of row i at [(sbase[i/32] + k) * 32 + i%32]; columns as
// int32 and the NV matrix values of a slot as NV doubles, each plane of 32
// lanes contiguous, so a warp's loads of one slot are fully coalesced.  Rows
// loop to their own length: padding slots are never read.  Streams read once
// per step (slots, per-node coefficients) load with the evict-first hint,
// leaving L1 to the neighbour gathers.  State vectors are
// FP64 [N]: u_old / u_now / u_new rotate through three buffers (acoustic.c),
// u1 and u2 likewise, p1, p2 and u through two (acoustic_pml.c).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/seisfem_acoustic.h"
#include "sfg_internal.h"

using namespace sfg;

namespace {

constexpr int kThreads = 256;

// one fused step's inputs (pointers of this step's buffers)
struct AcStep {
    int N, src;
    double ps;                         // Ricker amplitude of this step
    const int *sbase, *rlen, *col;
    const double *val;                 // [slots][NV][32]
    const double *cv;                  // ((vp * vp) * dt) * dt per node
    const double *m;                   // lumped mass
    const double *pdx, *pdy, *pdxx, *pdyy;   // PML profiles (PML only)
    double dt;
    // acoustic.c: a = u_old, b = u_now, c = u_new
    // acoustic_pml.c: u1 old/now/new, u2 old/now/new, p1 / p2 / u now and new
    const double *u1o, *u1n, *u2o, *u2n, *p1n, *p2n, *un;
    double *u1w, *u2w, *p1w, *p2w, *uw;
    double *snap;                      // snapshot row of this step, or nullptr
    double *energy;                    // energy[it]
};

__device__ __forceinline__ void block_energy_add(double e, double *out)
{
    __shared__ double part[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += part[w];
        atomicAdd(out, s);
    }
}

// acoustic.c:139-165, 168-183 (masslump), 185-188 (energy)
__global__ void __launch_bounds__(kThreads) acoustic_step(const AcStep a)
{
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double e = 0.0;
    if (i < a.N) {
        const int lane = i & 31, base = __ldg(a.sbase + (i >> 5)), len = __ldg(a.rlen + i);
        const int *cp = a.col + (size_t)base * 32 + lane;
        const double *vq = a.val + (size_t)base * 2 * 32 + lane;
        double y1 = 0.0, y2 = 0.0, y3 = 0.0;   // K u_now, M u_now, M u_old
        int jn = len > 0 ? __ldcs(cp) : 0;      // the next slot's column, one slot ahead
        for (int k = 0; k < len; k++) {
            const int j = jn;
            jn = k + 1 < len ? __ldcs(cp + (size_t)(k + 1) * 32) : 0;
            const double mv = __ldcs(vq + (size_t)k * 64), kv = __ldcs(vq + (size_t)k * 64 + 32);
            const double b = __ldg(a.u1n + j), o = __ldg(a.u1o + j);
            y1 = y1 + kv * b;
            y2 = y2 + mv * b;
            y3 = y3 + mv * o;
        }
        const double rhs = (double)(i == a.src) * a.ps - __ldcs(a.cv + i) * y1 + 2.0 * y2 - y3;
        const double m = __ldcs(a.m + i);
        const double u = m != 0.0 ? rhs / (1.0 * m) : __ldg(a.u1n + i);
        a.u1w[i] = u;
        if (a.snap) a.snap[i] = u;
        e = u * u;
    }
    block_energy_add(e, a.energy);
}

// the 10 products of one row of the PML step, summed in slot order
struct PmlSums {
    // x1 = M u1_now, x2 = M u1_old, x3 = M p1_now, x4 = K1 u_now, x5 = K5 u_now,
    // z1 = M u2_now, z2 = M u2_old, z3 = M p2_now, z4 = K2 u_now, z5 = K6 u_now
    double x1 = 0.0, x2 = 0.0, x3 = 0.0, x4 = 0.0, x5 = 0.0;
    double z1 = 0.0, z2 = 0.0, z3 = 0.0, z4 = 0.0, z5 = 0.0;
    __device__ __forceinline__ void add(const AcStep &a, int j, const double *v)
    {
        const double mv = __ldcs(v), k1 = __ldcs(v + 32), k5 = __ldcs(v + 64), k2 = __ldcs(v + 96),
                     k6 = __ldcs(v + 128);
        const double u = __ldg(a.un + j);
        x1 = x1 + mv * __ldg(a.u1n + j);
        x2 = x2 + mv * __ldg(a.u1o + j);
        x3 = x3 + mv * __ldg(a.p1n + j);
        x4 = x4 + k1 * u;
        x5 = x5 + k5 * u;
        z1 = z1 + mv * __ldg(a.u2n + j);
        z2 = z2 + mv * __ldg(a.u2o + j);
        z3 = z3 + mv * __ldg(a.p2n + j);
        z4 = z4 + k2 * u;
        z5 = z5 + k6 * u;
    }
};

// acoustic_pml.c:277-353 (four split equations), 355-375 (masslump),
// 432-439 (u = u1 + u2, energy).  The next slot's column is loaded before the
// current slot's gathers are used, so its latency overlaps them (measured:
// 72.3 against 86.0 ms per 1000 steps of a 641,601-node mesh; two slots ahead
// 81.2 ms), and the kernel needs 48 registers (5 blocks of 256 per SM).
__global__ void __launch_bounds__(kThreads) acoustic_pml_step(const AcStep a)
{
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double e = 0.0;
    if (i < a.N) {
        const int lane = i & 31, base = __ldg(a.sbase + (i >> 5)), len = __ldg(a.rlen + i);
        const int *cp = a.col + (size_t)base * 32 + lane;
        const double *vq = a.val + (size_t)base * 5 * 32 + lane;
        PmlSums s;
        int jn = len > 0 ? __ldcs(cp) : 0;
        for (int k = 0; k < len; k++) {
            const int j = jn;
            jn = k + 1 < len ? __ldcs(cp + (size_t)(k + 1) * 32) : 0;
            s.add(a, j, vq + (size_t)k * 160);
        }
        const double x1 = s.x1, x2 = s.x2, x3 = s.x3, x4 = s.x4, x5 = s.x5;
        const double z1 = s.z1, z2 = s.z2, z3 = s.z3, z4 = s.z4, z5 = s.z5;
        const double dt = a.dt, cv = __ldcs(a.cv + i);
        const double dx = __ldcs(a.pdx + i), dy = __ldcs(a.pdy + i);
        const double dxx = __ldcs(a.pdxx + i), dyy = __ldcs(a.pdyy + i);
        // the M p products of equations 2 and 4 repeat those of 1 and 3 (same
        // rows, same order, same operands): x3, z3
        const double rhs1 = 2.0 * x1 - x2 - 2.0 * dt * dx * x1 + 2 * dt * dx * x2 - dt * dt * dx * dx * x1 +
                            cv * x4 + cv * x3 + (double)(i == a.src) * a.ps;
        const double rhs2 = x3 - dt * dx * x3 - dt * dxx * x5;
        const double rhs3 = 2.0 * z1 - z2 - 2.0 * dt * dy * z1 + 2 * dt * dy * z2 - dt * dt * dy * dy * z1 +
                            cv * z4 + cv * z3;
        const double rhs4 = z3 - dt * dy * z3 - dt * dyy * z5;
        const double m = __ldcs(a.m + i);
        double u1, p1, u2, p2;
        if (m != 0.0) {
            u1 = rhs1 / (1.0 * m);
            p1 = rhs2 / (1.0 * m);
            u2 = rhs3 / (1.0 * m);
            p2 = rhs4 / (1.0 * m);
        } else {   // the reference prints an error and leaves the values
            u1 = __ldg(a.u1n + i);
            p1 = __ldg(a.p1n + i);
            u2 = __ldg(a.u2n + i);
            p2 = __ldg(a.p2n + i);
        }
        const double u = u1 + u2;
        a.u1w[i] = u1;
        a.u2w[i] = u2;
        a.p1w[i] = p1;
        a.p2w[i] = p2;
        a.uw[i] = u;
        if (a.snap) a.snap[i] = u;
        e = u * u;
    }
    block_energy_add(e, a.energy);
}

// ---------------------------------------------------------------- set-up

// per slice of 32 rows: the longest row
__global__ void slice_len(int N, const int *__restrict__ up, int *__restrict__ slen, int *__restrict__ rlen)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ns = (N + 31) / 32;
    if (i >= ns * 32) return;
    const int l = i < N ? up[i + 1] - up[i] : 0;
    if (i < N) rlen[i] = l;
    int mx = l;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((i & 31) == 0) slen[i >> 5] = mx;
}

// SELL-32 slots of the union pattern: columns and NV value planes
__global__ void sell_fill(int N, int nv, long long unnz, const int *__restrict__ up, const int *__restrict__ uj,
                          const double *__restrict__ ux, const int *__restrict__ sbase, int *__restrict__ col,
                          double *__restrict__ val)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int s = i >> 5, lane = i & 31, r0 = up[i], len = up[i + 1] - r0;
    const int b = sbase[s], n = sbase[s + 1] - b;
    for (int k = 0; k < n; k++) {
        const size_t slot = (size_t)b + k;
        const bool real = k < len;
        col[slot * 32 + lane] = real ? uj[r0 + k] : i;
        for (int v = 0; v < nv; v++)
            val[(slot * nv + v) * 32 + lane] = real ? ux[(size_t)v * unnz + r0 + k] : 0.0;
    }
}

__global__ void fill_value(double *p, int n, double v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// device buffers of one run (from the device's stream-ordered pool), released
// in stream order on every return path
struct Bufs {
    cudaStream_t st;
    std::vector<void *> ptrs;
    explicit Bufs(cudaStream_t s) : st(s) {}
    ~Bufs() { for (void *p : ptrs) keep_free(p, st); }
    template <typename T>
    cudaError_t get(T **p, size_t n)
    {
        cudaError_t e = keep_alloc(p, sizeof(T) * std::max<size_t>(n, 1), st);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

// pml/abc_pml.c:41-103 (region tests in the reference's order), host FP64
void abc_pml_host(int N, long long nref, const int *en, const double *x, const double *y, int nx, int ny,
                  double h, double xmin, double xmax, double ymin, double ymax, double vp_max, double *pdx,
                  double *pdy, double *pdxx, double *pdyy)
{
    const double Rcoef = 0.0001;
    const double tx = h * nx, ty = h * ny;
    const double x0 = xmin + tx, x1 = xmax - tx, y0 = ymin + ty, y1 = ymax - ty;
    const double d0x = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * tx);
    const double d0y = 3.0 * vp_max * std::log10(1.0 / Rcoef) / (2.0 * ty);
    for (int i = 0; i < N; i++) pdx[i] = pdy[i] = pdxx[i] = pdyy[i] = 0.0;
    for (long long k = 0; k < nref; k++) {
        const int p = en[k] - 1;
        const double X = x[p], Y = y[p];
        if (X <= x0) {
            pdx[p] = d0x * ((x0 - X) / tx) * ((x0 - X) / tx);
            pdxx[p] = -d0x * 2 * (x0 - X) / (tx * tx);
        } else if (X >= x1) {
            pdx[p] = d0x * ((X - x1) / tx) * ((X - x1) / tx);
            pdxx[p] = d0x * 2 * (X - x1) / (tx * tx);
        } else {
            pdx[p] = 0.0;
            pdxx[p] = 0.0;
        }
        if (Y <= y0) {
            pdy[p] = d0y * ((y0 - Y) / ty) * ((y0 - Y) / ty);
            pdyy[p] = -d0y * 2 * (y0 - Y) / (ty * ty);
        } else if (Y >= y1) {
            pdy[p] = d0y * ((Y - y1) / ty) * ((Y - y1) / ty);
            pdyy[p] = d0y * 2 * (Y - y1) / (ty * ty);
        } else {
            pdy[p] = 0.0;
            pdyy[p] = 0.0;
        }
    }
}

int type_code(const char *t)
{
    static const char *names[] = {"T3", "T6", "T10", "Q4", "Q9", "Q16"};
    if (!t) return -1;
    for (int i = 0; i < 6; i++)
        if (std::strcmp(t, names[i]) == 0) return i + 1;
    return -1;
}

}  // namespace

#define ACK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return ctx_fail(ctx, e_ == cudaErrorMemoryAllocation ? SFG_ERR_OOM : SFG_ERR_CUDA,    \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

extern "C" int sfg_acoustic_snapshot_rows(int step, int pml)
{
    return sfg_snapshot_rows(step, pml ? 20 : 10);
}

extern "C" int sfg_acoustic_run(sfg_ctx *ctx, const sfg_mesh *m, const double *vp, const sfg_acoustic_desc *d,
                                double *snap, double *energy, sfg_acoustic_stats *stats)
{
    if (!ctx || !m || !vp || !d) return SFG_ERR_ARG;
    const int tc = type_code(m->type);
    if (tc < 0) return ctx_fail(ctx, SFG_ERR_ARG, "unknown element type");
    const int p = elem_order_host(tc), N = m->node_num, E = m->element_num;
    if (m->element_order != p || N <= 0 || E <= 0 || !m->element_node || !m->x || !m->y || d->step < 3 ||
        !(d->dt > 0.0))
        return ctx_fail(ctx, SFG_ERR_ARG, "inconsistent acoustic run description");
    const long long nnz = (long long)E * p * p;
    if (nnz >= (1LL << 31)) return ctx_fail(ctx, SFG_ERR_ARG, "COO size exceeds 2^31");
    if (d->source_node < -1 || d->source_node >= N) return ctx_fail(ctx, SFG_ERR_BADINDEX, "source node out of range");
    for (long long k = 0; k < (long long)E * p; k++)
        if (m->element_node[k] < 1 || m->element_node[k] > N)
            return ctx_fail(ctx, SFG_ERR_BADINDEX, "element_node entry out of range at " + std::to_string(k));
    if (d->pml && (m->pml_nx <= 0 || m->pml_ny <= 0 || !(m->edge_size > 0.0)))
        return ctx_fail(ctx, SFG_ERR_ARG, "PML thickness and edge size must be positive");
    ACK(cudaSetDevice(ctx_device(ctx)));
    cudaStream_t st = ctx_stream(ctx);
    const auto t_setup = std::chrono::steady_clock::now();
    const int pml = d->pml ? 1 : 0, NV = pml ? 5 : 2;
    Bufs B(st);

    // element matrices: M (density 1) and K0, or M, K1, K5, K2, K6
    int *d_en, *d_flags, *d_ci, *d_cj;
    double *d_x, *d_y, *d_one, *d_cx;
    ACK(B.get(&d_en, (size_t)E * p));
    ACK(B.get(&d_x, N));
    ACK(B.get(&d_y, N));
    ACK(B.get(&d_one, N));
    ACK(B.get(&d_flags, 1));
    ACK(B.get(&d_ci, nnz));
    ACK(B.get(&d_cj, nnz));
    ACK(B.get(&d_cx, (size_t)NV * nnz));
    ACK(cudaMemcpyAsync(d_en, m->element_node, sizeof(int) * E * p, cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(d_x, m->x, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    ACK(cudaMemcpyAsync(d_y, m->y, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    ACK(cudaMemsetAsync(d_flags, 0, sizeof(int), st));
    fill_value<<<(N + 255) / 256, 256, 0, st>>>(d_one, N, 1.0);
    const int mats_ac[2] = {-1, 0}, mats_pml[5] = {-1, 1, 5, 2, 6};
    ACK(launch_element_coo(tc, E, d_en, d_x, d_y, d_one, NV, pml ? mats_pml : mats_ac, d_ci, d_cj, d_cx, d_flags,
                           st));
    int hflags = 0;
    ACK(cudaMemcpyAsync(&hflags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    if (hflags & FLAG_ZERO_AREA) return ctx_fail(ctx, SFG_ERR_ZERO_AREA, "an element has zero area");
    CanonOut co;
    std::string err;
    int rc = canonicalize(N, nnz, d_ci, d_cj, d_cx, NV, true, true, co, d_flags, st, err);
    struct CanonGuard {
        CanonOut &c;
        cudaStream_t s;
        ~CanonGuard()
        {
            canon_free(c, false, s);
            keep_free(c.up, s); keep_free(c.uj, s); keep_free(c.ux, s);
        }
    } guard{co, st};
    if (rc != SFG_OK) return ctx_fail(ctx, rc, "acoustic canonical CSR: " + err);

    // lumped mass (mass_sparse_q4.c:238-263 with density 1), or the caller's
    double *d_m, *d_scr;
    ACK(B.get(&d_m, N));
    if (d->mass_lump) {
        ACK(cudaMemcpyAsync(d_m, d->mass_lump, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    } else {
        ACK(B.get(&d_scr, 2 * (size_t)E + 2));
        ACK(launch_lumped_mass(tc, N, E, d_en, d_x, d_y, d_one, co.row_start, co.bucket, d_cj, d_m, d_scr,
                               d_flags, st));
    }

    // per-node coefficients: ((vp * vp) * dt) * dt (acoustic.c:164,
    // acoustic_pml.c:302-303) and the PML profile
    const double dt = d->dt;
    std::vector<double> h(N);
    for (int i = 0; i < N; i++) h[i] = vp[i] * vp[i] * dt * dt;
    double *d_cv;
    ACK(B.get(&d_cv, N));
    ACK(cudaMemcpyAsync(d_cv, h.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
    double *d_pml = nullptr;
    if (pml) {
        double vp_max = vp[0];   // acoustic_pml.c:175-179
        for (int i = 0; i < N; i++) if (vp[i] > vp_max) vp_max = vp[i];
        std::vector<double> prof(4 * (size_t)N);
        abc_pml_host(N, (long long)E * p, m->element_node, m->x, m->y, m->pml_nx, m->pml_ny, m->edge_size,
                     m->xmin, m->xmax, m->ymin, m->ymax, vp_max, prof.data(), prof.data() + N,
                     prof.data() + 2 * (size_t)N, prof.data() + 3 * (size_t)N);
        ACK(B.get(&d_pml, 4 * (size_t)N));
        ACK(cudaMemcpyAsync(d_pml, prof.data(), sizeof(double) * prof.size(), cudaMemcpyHostToDevice, st));
    }

    // SELL-32 slots of the union pattern
    const int ns = (N + 31) / 32;
    int *d_slen, *d_sbase, *d_rlen, *d_col;
    double *d_val;
    ACK(B.get(&d_slen, ns + 1));
    ACK(B.get(&d_sbase, ns + 1));
    ACK(B.get(&d_rlen, N));
    slice_len<<<(ns * 32 + 255) / 256, 256, 0, st>>>(N, co.up, d_slen, d_rlen);
    ACK(exclusive_scan_int(d_slen, d_sbase, ns, st));
    int slots = 0;
    ACK(cudaMemcpyAsync(&slots, d_sbase + ns, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACK(cudaStreamSynchronize(st));
    ACK(B.get(&d_col, (size_t)slots * 32));
    ACK(B.get(&d_val, (size_t)slots * 32 * NV));
    sell_fill<<<(N + 255) / 256, 256, 0, st>>>(N, NV, co.union_nnz, co.up, co.uj, co.ux, d_sbase, d_col, d_val);
    ACK(cudaGetLastError());

    // state: three rotating buffers of u1 (and u2), two of p1, p2, u; all zero
    const int nstate = pml ? 12 : 3;
    double *d_state;
    ACK(B.get(&d_state, (size_t)nstate * N));
    ACK(cudaMemsetAsync(d_state, 0, sizeof(double) * nstate * N, st));
    auto S = [&](int k) { return d_state + (size_t)k * N; };
    const int rows = sfg_acoustic_snapshot_rows(d->step, pml);
    double *d_snap = nullptr, *d_energy;
    if (snap) {
        ACK(B.get(&d_snap, (size_t)rows * N));
        ACK(cudaMemsetAsync(d_snap, 0, sizeof(double) * N, st));   // the zero row
    }
    ACK(B.get(&d_energy, d->step));
    ACK(cudaMemsetAsync(d_energy, 0, sizeof(double) * d->step, st));
    ACK(cudaStreamSynchronize(st));
    const double setup_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();

    // the time loop as one graph
    const int every = pml ? 20 : 10;
    AcStep a{};
    a.N = N; a.src = d->source_node; a.sbase = d_sbase; a.rlen = d_rlen; a.col = d_col; a.val = d_val;
    a.cv = d_cv; a.m = d_m; a.dt = dt;
    if (pml) { a.pdx = d_pml; a.pdy = d_pml + N; a.pdxx = d_pml + 2 * (size_t)N; a.pdyy = d_pml + 3 * (size_t)N; }
    const unsigned grid = (unsigned)((N + kThreads - 1) / kThreads);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ACK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int row = 1, launches = 0;
    for (int it = 2; it < d->step; it++) {
        const int r = it % 3;   // rotation: old = r, now = (r + 1) % 3, new = (r + 2) % 3
        const int q = it & 1;   // p1, p2, u: now = q, new = 1 - q
        a.ps = ricker_amplitude(d->f0, d->t0, 1.0, (it + 1) * dt);
        a.energy = d_energy + it;
        a.snap = (snap && (it + 1) % every == 0) ? d_snap + (size_t)row++ * N : nullptr;
        if (!pml) {
            a.u1o = S(r); a.u1n = S((r + 1) % 3); a.u1w = S((r + 2) % 3);
            acoustic_step<<<grid, kThreads, 0, st>>>(a);
        } else {
            a.u1o = S(r); a.u1n = S((r + 1) % 3); a.u1w = S((r + 2) % 3);
            a.u2o = S(3 + r); a.u2n = S(3 + (r + 1) % 3); a.u2w = S(3 + (r + 2) % 3);
            a.p1n = S(6 + q); a.p1w = S(7 - q);
            a.p2n = S(8 + q); a.p2w = S(9 - q);
            a.un = S(10 + q); a.uw = S(11 - q);
            acoustic_pml_step<<<grid, kThreads, 0, st>>>(a);
        }
        launches++;
    }
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        return ctx_fail(ctx, SFG_ERR_CUDA, std::string("acoustic graph: ") + cudaGetErrorString(ce));
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    ce = cudaGraphLaunch(exec, st);
    cudaEventRecord(e1, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    float loop_ms = 0.f;
    cudaEventElapsedTime(&loop_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    if (ce != cudaSuccess) return ctx_fail(ctx, SFG_ERR_CUDA, std::string("acoustic loop: ") + cudaGetErrorString(ce));

    // energy bound of the PML solver (acoustic_pml.c:440-446)
    std::vector<double> en(d->step);
    ACK(cudaMemcpy(en.data(), d_energy, sizeof(double) * d->step, cudaMemcpyDeviceToHost));
    int blow = -1;
    if (pml)
        for (int it = 2; it < d->step; it++)
            if (en[it] > 10e6) { blow = it; break; }
    const int last = blow >= 0 ? blow : d->step;   // steps it < last were completed
    if (energy) {
        for (int it = 0; it < d->step; it++) energy[it] = it < last ? en[it] : 0.0;
    }
    if (snap) {
        const int keep = sfg_snapshot_rows(last, every);
        ACK(cudaMemcpy(snap, d_snap, sizeof(double) * (size_t)keep * N, cudaMemcpyDeviceToHost));
        if (keep < rows) std::memset(snap + (size_t)keep * N, 0, sizeof(double) * (size_t)(rows - keep) * N);
    }
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->setup_ms = setup_ms;
        stats->loop_ms = loop_ms;
        stats->union_nnz = co.union_nnz;
        for (int k = 0; k < NV; k++) stats->csr_nnz[k] = co.csr[k].nnz;
        stats->kernel_launches = launches;
        stats->blowup_step = blow;
    }
    if (blow >= 0) return ctx_fail(ctx, SFG_ERR_BLOWUP, "energy exceeds maximum value at step " + std::to_string(blow));
    return SFG_OK;
}
