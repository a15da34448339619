// sfg_dict.cu -- value dictionary of the step matrices for the one-shot
// fused kernels.
//
// A mesh built from congruent elements (structured Q4 / Q9 / T6 grids) gives
// union entries that carry only a few dozen distinct value tuples
// (M / rho_row, K1..K6): the element matrices repeat, and M is the row's
// density times a geometric matrix (mass_sparse_q4.c:252 scales by the
// row node's rho).  They differ only by FP64 rounding noise far below FP32
// resolution (entries that are zero in exact arithmetic come out as ~1e-17 of
// the matrix's largest entry).  Each tuple component is quantised to 2^-40 of
// its matrix's largest magnitude; when at most kDictMax distinct tuples
// remain, the SELL slots of the one-shot kernels carry (column, tuple id) --
// 8 bytes instead of 24 or 32 -- the kernels read the tuple from shared
// memory, and scale the mass products by the row's density.  Meshes with more
// distinct tuples keep the full-value slots.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "sfg_internal.h"
#include "sfg_step32.cuh"

namespace sfg {

namespace {

constexpr int kCap = 8192;          // hash slots (a power of two)
constexpr int kShift = 40;          // quantum = largest magnitude * 2^-40

struct DictScratch {
    unsigned long long scale[7];    // largest |value| per matrix (FP64 bits; positive, so they order as integers)
    unsigned long long keys[kCap];  // tuple hash, 0 = empty
    long long q[kCap][7];           // quantised tuple of the slot's first writer
    int ids[kCap];                  // compact tuple id per occupied slot
    int count;                      // occupied slots
    int bad;                        // probe overflow or hash collision
};

__device__ __forceinline__ double entry_value(const double *ux, long long nnz, long long e, int k, double rho)
{
    const double v = ux[k * nnz + e];
    return k == 0 ? v / rho : v;
}

// row of union entry e (rows' entries are contiguous and ordered)
__device__ __forceinline__ int row_of(const int *__restrict__ up, int n, long long e)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (up[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// one thread per union entry (coalesced reads of the value planes)
// Largest magnitude per matrix: each thread strides over the union entries,
// the block reduces, and one atomic per block and matrix merges the blocks
// (a few hundred blocks, so the seven addresses see few atomics).
__global__ void __launch_bounds__(256) dict_scale(int n, const int *__restrict__ up, const double *__restrict__ ux,
                                                  long long nnz, const double *__restrict__ rho, DictScratch *s)
{
    __shared__ double red[8][7];
    double m[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
        const double rr = rho[row_of(up, n, e)];
        for (int k = 0; k < 7; k++) m[k] = fmax(m[k], fabs(entry_value(ux, nnz, e, k, rr)));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 7; k++) {
        double v = m[k];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) red[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double v = 0.0;
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) v = fmax(v, red[j][threadIdx.x]);
        if (v > 0.0) atomicMax(&s->scale[threadIdx.x], (unsigned long long)__double_as_longlong(v));
    }
}

__device__ __forceinline__ void quantise(const DictScratch *s, const double *v, long long *q)
{
    for (int k = 0; k < 7; k++) {
        const double sc = __longlong_as_double((long long)s->scale[k]);
        q[k] = sc > 0.0 ? __double2ll_rn(v[k] / ldexp(sc, -kShift)) : 0;
    }
}

__device__ __forceinline__ unsigned long long tuple_hash(const long long *q)
{
    unsigned long long h = 0x9E3779B97F4A7C15ull;
    for (int k = 0; k < 7; k++) {
        unsigned long long x = (unsigned long long)q[k] + 0x632BE59BD9B4E019ull * (k + 1);
        x ^= x >> 31;
        x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 29;
        h = (h ^ x) * 0x94D049BB133111EBull;
    }
    return h ? h : 1ull;
}

// Slot of a quantised tuple; the first writer of a slot records the tuple.
// Gives up (-1) once more than kDictMax tuples exist: the dictionary is then
// not used, and a full table would make every probe long.
__device__ int dict_insert(DictScratch *s, const long long *q)
{
    const unsigned long long h = tuple_hash(q);
    for (int p = 0; p < kCap; p++) {
        if (*(volatile int *)&s->count > kDictMax) return -1;
        const int slot = (int)((h + p) & (kCap - 1));
        unsigned long long cur = *(volatile unsigned long long *)&s->keys[slot];
        if (cur == 0ull) {
            cur = atomicCAS(&s->keys[slot], 0ull, h);
            if (cur == 0ull) {
                for (int k = 0; k < 7; k++) s->q[slot][k] = q[k];
                atomicAdd(&s->count, 1);
                return slot;
            }
        }
        if (cur == h) return slot;
    }
    s->bad = 1;
    return -1;
}

// the all-zero tuple (the SELL padding slots) first
__global__ void dict_insert_zero(DictScratch *s, int *zero_slot)
{
    const long long q[7] = {0, 0, 0, 0, 0, 0, 0};
    *zero_slot = dict_insert(s, q);
}

__global__ void dict_insert_entries(int n, const int *__restrict__ up, const double *__restrict__ ux, long long nnz,
                                    const double *__restrict__ rho, DictScratch *s, int *__restrict__ slot_of)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const double rr = rho[row_of(up, n, e)];
    double v[7];
    long long q[7];
    for (int k = 0; k < 7; k++) v[k] = entry_value(ux, nnz, e, k, rr);
    quantise(s, v, q);
    slot_of[e] = dict_insert(s, q);
}

// every entry against the tuple its slot recorded (a hash collision between
// different tuples would show here)
__global__ void dict_verify(int n, const int *__restrict__ up, const double *__restrict__ ux, long long nnz,
                            const double *__restrict__ rho, DictScratch *s, const int *__restrict__ slot_of)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const double rr = rho[row_of(up, n, e)];
    double v[7];
    long long q[7];
    for (int k = 0; k < 7; k++) v[k] = entry_value(ux, nnz, e, k, rr);
    quantise(s, v, q);
    const int slot = slot_of[e];
    bool ok = slot >= 0;
    for (int k = 0; k < 7 && ok; k++) ok = s->q[slot][k] == q[k];
    if (!ok) s->bad = 1;
}

// one block: compact ids in slot order, and the tuple values
// (quantised value times the quantum, rounded to FP32): table[2 id] =
// (M_geo, K1, K2, K3), table[2 id + 1] = (K4, K5, K6, 0)
__global__ void __launch_bounds__(1024) dict_compact(DictScratch *s, float4 *table)
{
    __shared__ int warp_sum[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < kCap; c0 += blockDim.x) {
        const int slot = c0 + threadIdx.x;
        const int occ = slot < kCap && s->keys[slot] != 0ull;
        const unsigned mask = __ballot_sync(0xffffffffu, occ);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) warp_sum[w] = __popc(mask);
        __syncthreads();
        int off = 0;
        for (int k = 0; k < w; k++) off += warp_sum[k];
        const int id = base + off + __popc(mask & ((1u << lane) - 1u));
        if (occ) {
            s->ids[slot] = id;
            float t[8];
            for (int k = 0; k < 7; k++) {
                const double sc = __longlong_as_double((long long)s->scale[k]);
                t[k] = (float)((double)s->q[slot][k] * ldexp(sc, -kShift));
            }
            t[7] = 0.f;
            table[2 * id] = make_float4(t[0], t[1], t[2], t[3]);
            table[2 * id + 1] = make_float4(t[4], t[5], t[6], t[7]);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += warp_sum[k];
            base += tot;
        }
        __syncthreads();
    }
}

__global__ void dict_ids(long long nnz, const DictScratch *s, const int *__restrict__ slot_of, int *__restrict__ tid)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nnz) tid[e] = s->ids[slot_of[e]];
}

// SELL slots of rows [r0, r1) (slice pointers sp as build_sell_range): the
// float4 index blk4(column, 0, 3) of the permuted column's state record and
// twice the tuple id (the tuple's first float4 in the kernels' table);
// padding slots point at the row itself with the zero tuple
__global__ void range_sell_fill_dict(int r0, int r1, const int *__restrict__ up, const int *__restrict__ uj,
                                     const int *__restrict__ tid, int zero_id, const int *__restrict__ sp,
                                     const int *__restrict__ perm, const int *__restrict__ inv, int2 *__restrict__ sell)
{
    const int s = blockIdx.x, lane = threadIdx.x;
    const int n = r1 - r0, r = s * 32 + lane;
    const int s0 = sp[s], s1 = sp[s + 1];
    const int o = r < n ? perm[r0 + r] : 0;
    const int a0 = r < n ? up[o] : 0, len = r < n ? up[o + 1] - a0 : 0;
    for (int k = 0; k < s1 - s0; k++) {
        int2 v;
        if (k < len) v = make_int2((int)blk4(inv[uj[a0 + k]], 0, 3), 2 * tid[a0 + k]);
        else v = make_int2((int)blk4(r < n ? r0 + r : r0, 0, 3), 2 * zero_id);
        sell[(size_t)(s0 + k) * 32 + lane] = v;
    }
}

__global__ void row_density(int n, const double *__restrict__ rho, const int *__restrict__ perm, float *__restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) out[r] = (float)rho[perm[r]];
}

}  // namespace

int build_value_dict(int n, const int *d_up, const double *d_ux, long long nnz, const double *d_rho,
                     int **d_tid, float4 **d_table, int *zero_id, cudaStream_t st)
{
    *d_tid = nullptr;
    *d_table = nullptr;
    DictScratch *s = nullptr;
    int *slot_of = nullptr, *zslot = nullptr;
    int T = -1;
    cudaError_t e = cudaMallocAsync((void **)&s, sizeof(DictScratch), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&slot_of, sizeof(int) * std::max<long long>(nnz, 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&zslot, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s, 0, sizeof(DictScratch), st);
    const unsigned g = (unsigned)((nnz + 255) / 256);
    if (e == cudaSuccess && n > 0 && nnz > 0) {
        dict_scale<<<std::min(g, 148u * 8u), 256, 0, st>>>(n, d_up, d_ux, nnz, d_rho, s);
        dict_insert_zero<<<1, 1, 0, st>>>(s, zslot);
        dict_insert_entries<<<g, 256, 0, st>>>(n, d_up, d_ux, nnz, d_rho, s, slot_of);
        e = cudaGetLastError();
    }
    int count = 0, bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&count, &s->count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && n > 0 && nnz > 0 && count <= kDictMax) {
        dict_verify<<<g, 256, 0, st>>>(n, d_up, d_ux, nnz, d_rho, s, slot_of);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, &s->bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && !bad) {
            e = keep_alloc(d_table, sizeof(float4) * 2 * (size_t)count, st);
            if (e == cudaSuccess) e = keep_alloc(d_tid, sizeof(int) * std::max<long long>(nnz, 1), st);
            if (e == cudaSuccess) {
                dict_compact<<<1, 1024, 0, st>>>(s, *d_table);
                dict_ids<<<(unsigned)((nnz + 255) / 256), 256, 0, st>>>(nnz, s, slot_of, *d_tid);
                e = cudaGetLastError();
            }
            int zs = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&zs, zslot, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(zero_id, &s->ids[0] + zs, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) T = count;
        }
    }
    if (T < 0) {   // not applicable (too many tuples, a collision) or an error
        keep_free(*d_tid, st);
        keep_free(*d_table, st);
        *d_tid = nullptr;
        *d_table = nullptr;
    }
    cudaFreeAsync(s, st);
    cudaFreeAsync(slot_of, st);
    cudaFreeAsync(zslot, st);
    if (e != cudaSuccess) return -1;
    return T < 0 ? 0 : T;
}

cudaError_t build_sell_range_dict(int r0, int r1, const int *d_up, const int *d_uj, const int *d_tid, int zero_id,
                                  const int *d_perm, const int *d_inv, int2 **d_sell, int **d_slice, long long *slots,
                                  cudaStream_t st)
{
    const int n = r1 - r0, nsl = (n + 31) / 32;
    int *len = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync((void **)&len, sizeof(int) * ((size_t)nsl + 1), st)) != cudaSuccess) return e;
    if ((e = keep_alloc(d_slice, sizeof(int) * ((size_t)nsl + 1), st)) != cudaSuccess) return e;
    if ((e = launch_range_slice_len(r0, r1, d_up, d_perm, len, st)) != cudaSuccess) return e;
    if ((e = exclusive_scan_int(len, *d_slice, nsl, st)) != cudaSuccess) return e;
    int tot = 0;
    cudaMemcpyAsync(&tot, *d_slice + nsl, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    *slots = tot;
    if ((e = keep_alloc(d_sell, sizeof(int2) * 32 * std::max<size_t>(tot, 1), st)) != cudaSuccess) return e;
    if (nsl) range_sell_fill_dict<<<nsl, 32, 0, st>>>(r0, r1, d_up, d_uj, d_tid, zero_id, *d_slice, d_perm, d_inv, *d_sell);
    e = cudaGetLastError();
    cudaFreeAsync(len, st);
    return e;
}

cudaError_t build_row_density(int n, const double *d_rho, const int *d_perm, float **d_out, cudaStream_t st)
{
    cudaError_t e = keep_alloc(d_out, sizeof(float) * std::max(n, 1), st);
    if (e == cudaSuccess && n > 0) {
        row_density<<<(n + 255) / 256, 256, 0, st>>>(n, d_rho, d_perm, *d_out);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace sfg
