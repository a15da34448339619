// sfg_fno.cu -- kernels of the learned surrogate (no counterpart in the
// reference): a Fourier neural operator that maps a velocity model and a
// source position to the receiver gather the FEM would record.
//
// Everything the network computes runs here: a strided, batched BF16 GEMM on
// the tensor cores with FP32 accumulation (lifting, 1x1 convolutions,
// truncated DFTs, per-mode channel mixing, depth-to-time map, projection and
// all their gradients), and the pointwise kernels around it (complex
// recombination of the DFT stages, GELU and its derivative, casts, bias
// gradients, the relative-L2 loss, Adam).  The host (seisfem_b200/surrogate.py)
// only sequences these calls on device buffers.
#include <cuda.h>          // CUtensorMap and its enums (the encoder is looked up at run time)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "../../include/seisfem_fno.h"

namespace {

// ------------------------------------------------------------------ GEMM
//
// sfg_gemm_desc (seisfem_fno.h): C[z][m][n] = alpha * sum_k A[z][m][k] B[z][k][n]
// with an epilogue (Cin, bias, pre-activation, GELU) or atomic accumulation.
// A, B: BF16 with arbitrary element strides; C: FP32 or BF16.  The CTA tile
// is BM x BN x 32 with eight warps; both operands are staged K-contiguous in
// shared memory (row pitch 40 elements: the fragment loads are free of bank
// conflicts) and fed to mma.sync m16n8k16 (BF16 in, FP32 accumulate).
// Split-K (gridDim.z = batches x splits) accumulates FP32 partial sums.

constexpr int BK = 32;
constexpr int PITCH = BK + 8;

struct GemmArgs {
    sfg_gemm_desc d;
    int amode, bmode;          // 0: k contiguous (16-B vectors), 1: m/n contiguous (vectors), 2: scalar
    int tz1a, tz2a, tz1b, tz2b;   // TMA engine: the operand's tensor map follows batch index 1 / 2
    // fused second projection (sfg_fno_head_infer): y[z1][j][m] = b2[j] +
    // sum_n GELU(C[m][n]) w2[n][j], j < n2, instead of storing C
    const float *w2, *b2;
    float *y;
    long long ys1, ysj;
    int n2;
};

__device__ __forceinline__ float gelu_f(float x)
{
    return 0.5f * x * (1.f + erff(x * 0.70710678118654752f));
}

// Loads rows [r0, r0 + R) x k [k0, k0 + 32) of an operand whose element (r, k)
// sits at p + r * sr + k * sk into registers: each thread holds R*32/256
// elements as 16-byte groups.  `mode` picks the vector direction.
template <int R>
struct TileLoad {
    static constexpr int PER = R * BK / 256;   // elements per thread (16 or 8)
    static constexpr int VEC = 8;
    static constexpr int NV = PER / VEC;       // vectors per thread
    uint4 v[NV];

    __device__ __forceinline__ void load(const __nv_bfloat16 *p, long long sr, long long sk, int rows, int kk,
                                         int r0, int k0, int mode)
    {
        const int t = threadIdx.x;
#pragma unroll
        for (int q = 0; q < NV; q++) {
            const int idx = t + q * 256;   // vector index in the tile
            __align__(16) __nv_bfloat16 e[8];
            if (mode == 0) {               // 8 consecutive k of one row
                const int r = idx / (BK / 8), kc = (idx % (BK / 8)) * 8;
                const int gr = r0 + r, gk = k0 + kc;
                if (gr < rows && gk + 8 <= kk) {
                    v[q] = __ldg(reinterpret_cast<const uint4 *>(p + gr * sr + gk));
                    continue;
                }
#pragma unroll
                for (int u = 0; u < 8; u++)
                    e[u] = (gr < rows && gk + u < kk) ? p[gr * sr + (gk + u) * sk] : __float2bfloat16(0.f);
            } else if (mode == 1) {        // 8 consecutive rows of one k
                const int kc = idx / (R / 8), r = (idx % (R / 8)) * 8;
                const int gr = r0 + r, gk = k0 + kc;
                if (gk < kk && gr + 8 <= rows) {
                    v[q] = __ldg(reinterpret_cast<const uint4 *>(p + gr + gk * sk));
                    continue;
                }
#pragma unroll
                for (int u = 0; u < 8; u++)
                    e[u] = (gr + u < rows && gk < kk) ? p[(gr + u) * sr + gk * sk] : __float2bfloat16(0.f);
            } else {                       // scalar, same order as mode 0
                const int r = idx / (BK / 8), kc = (idx % (BK / 8)) * 8;
                const int gr = r0 + r, gk = k0 + kc;
#pragma unroll
                for (int u = 0; u < 8; u++)
                    e[u] = (gr < rows && gk + u < kk) ? p[gr * sr + (gk + u) * sk] : __float2bfloat16(0.f);
            }
            v[q] = *reinterpret_cast<const uint4 *>(e);
        }
    }

    // modes 0 and 2: s[r][k] (pitch PITCH); mode 1: s[k][r] (pitch R + 8),
    // read back with ldmatrix.trans
    __device__ __forceinline__ void store(__nv_bfloat16 *s, int mode) const
    {
        const int t = threadIdx.x;
#pragma unroll
        for (int q = 0; q < NV; q++) {
            const int idx = t + q * 256;
            if (mode == 1) {
                const int kc = idx / (R / 8), r = (idx % (R / 8)) * 8;
                *reinterpret_cast<uint4 *>(s + kc * (R + 8) + r) = v[q];
            } else {
                const int r = idx / (BK / 8), kc = (idx % (BK / 8)) * 8;
                *reinterpret_cast<uint4 *>(s + r * PITCH + kc) = v[q];
            }
        }
    }
};

__device__ __forceinline__ void mma_bf16(float *c, const uint32_t *a, const uint32_t *b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// BM x BN CTA tile, warps arranged WM x WN (WM * WN = 8); each warp owns a
// (BM/WM) x (BN/WN) sub-tile of m16 x n8 MMA tiles.
template <int BM, int BN, int WM, int WN>
__global__ void __launch_bounds__(256) gemm_bf16_kernel(const GemmArgs g)
{
    constexpr int TM = BM / WM / 16, TN = BN / WN / 8;
    constexpr int ASZ = BM * PITCH > BK * (BM + 8) ? BM * PITCH : BK * (BM + 8);
    constexpr int BSZ = BN * PITCH > BK * (BN + 8) ? BN * PITCH : BK * (BN + 8);
    __shared__ __align__(16) __nv_bfloat16 As[2][ASZ];
    __shared__ __align__(16) __nv_bfloat16 Bs[2][BSZ];
    const sfg_gemm_desc &d = g.d;
    const int nb = d.batch1 * d.batch2;
    const int bz = blockIdx.z;
    const int z = bz % nb, split = bz / nb;
    const int z1 = z / d.batch2, z2 = z % d.batch2;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int ktiles = (d.K + BK - 1) / BK;
    const int per = (ktiles + d.splits - 1) / d.splits;
    const int kt0 = split * per, kt1 = min(ktiles, kt0 + per);
    const __nv_bfloat16 *A = static_cast<const __nv_bfloat16 *>(d.A) + z1 * d.sa1 + z2 * d.sa2;
    const __nv_bfloat16 *B = static_cast<const __nv_bfloat16 *>(d.B) + z1 * d.sb1 + z2 * d.sb2;
    const long long cz = z1 * d.sc1 + z2 * d.sc2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp / WN, wn = warp % WN;
    const int gq = lane >> 2, tq = lane & 3;
    float acc[TM][TN][4];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    TileLoad<BM> la;
    TileLoad<BN> lb;
    if (kt0 < kt1) {
        la.load(A, d.sam, d.sak, d.M, d.K, m0, kt0 * BK, g.amode);
        lb.load(B, d.sbn, d.sbk, d.N, d.K, n0, kt0 * BK, g.bmode);
        la.store(As[0], g.amode);
        lb.store(Bs[0], g.bmode);
    }
    __syncthreads();
    for (int kt = kt0; kt < kt1; kt++) {
        const int cur = (kt - kt0) & 1;
        if (kt + 1 < kt1) {
            la.load(A, d.sam, d.sak, d.M, d.K, m0, (kt + 1) * BK, g.amode);
            lb.load(B, d.sbn, d.sbk, d.N, d.K, n0, (kt + 1) * BK, g.bmode);
        }
        const __nv_bfloat16 *as = As[cur], *bs = Bs[cur];
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[TM][4], bf[TN][2];
            if (g.amode == 1) {
                // As[k][m]: four 8x8 blocks (m 0-7 / 8-15, k 0-7 / 8-15) transposed by ldmatrix
                const int lm = (lane >> 3) & 1, lk = lane >> 4, lr = lane & 7;
#pragma unroll
                for (int i = 0; i < TM; i++) {
                    const int mb = wm * (BM / WM) + i * 16;
                    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(
                        as + (ks + lk * 8 + lr) * (BM + 8) + mb + lm * 8);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                                 : "=r"(af[i][0]), "=r"(af[i][1]), "=r"(af[i][2]), "=r"(af[i][3])
                                 : "r"(addr));
                }
            } else {
#pragma unroll
                for (int i = 0; i < TM; i++) {
                    const int r = wm * (BM / WM) + i * 16 + gq;
                    af[i][0] = *reinterpret_cast<const uint32_t *>(as + r * PITCH + ks + 2 * tq);
                    af[i][1] = *reinterpret_cast<const uint32_t *>(as + (r + 8) * PITCH + ks + 2 * tq);
                    af[i][2] = *reinterpret_cast<const uint32_t *>(as + r * PITCH + ks + 8 + 2 * tq);
                    af[i][3] = *reinterpret_cast<const uint32_t *>(as + (r + 8) * PITCH + ks + 8 + 2 * tq);
                }
            }
            if (g.bmode == 1) {
                // Bs[k][n]: two 8x8 blocks (k 0-7, 8-15) per n8 tile, transposed by ldmatrix
                const int lk = (lane >> 3) & 1, lr = lane & 7;
#pragma unroll
                for (int j = 0; j < TN; j++) {
                    const int nb = wn * (BN / WN) + j * 8;
                    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(bs + (ks + lk * 8 + lr) * (BN + 8) + nb);
                    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];"
                                 : "=r"(bf[j][0]), "=r"(bf[j][1])
                                 : "r"(addr));
                }
            } else {
#pragma unroll
                for (int j = 0; j < TN; j++) {
                    const int n = wn * (BN / WN) + j * 8 + gq;
                    bf[j][0] = *reinterpret_cast<const uint32_t *>(bs + n * PITCH + ks + 2 * tq);
                    bf[j][1] = *reinterpret_cast<const uint32_t *>(bs + n * PITCH + ks + 8 + 2 * tq);
                }
            }
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) mma_bf16(acc[i][j], af[i], bf[j]);
        }
        if (kt + 1 < kt1) {
            la.store(As[cur ^ 1], g.amode);
            lb.store(Bs[cur ^ 1], g.bmode);
        }
        __syncthreads();
    }
    // epilogue: a thread holds columns n, n + 1 of rows m and m + 8; with
    // unit column stride the pair is read and written as one vector
    const bool pairs = d.scn == 1 && !d.atomic;
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = m0 + wm * (BM / WM) + i * 16 + gq + h * 8;
                const int n = n0 + wn * (BN / WN) + j * 8 + 2 * tq;
                if (m >= d.M || n >= d.N) continue;
                const long long o = cz + m * d.scm + n * d.scn;
                float v0 = d.alpha * acc[i][j][2 * h], v1 = d.alpha * acc[i][j][2 * h + 1];
                if (pairs && n + 1 < d.N && (o & 1) == 0) {
                    if (d.Cin) {
                        const float2 ci = *reinterpret_cast<const float2 *>(d.Cin + o);
                        v0 += d.beta * ci.x;
                        v1 += d.beta * ci.y;
                    }
                    if (d.bias) {
                        v0 += d.bias[d.bias_on_m ? m : n];
                        v1 += d.bias[d.bias_on_m ? m : n + 1];
                    }
                    if (d.pre)
                        *reinterpret_cast<__nv_bfloat162 *>(static_cast<__nv_bfloat16 *>(d.pre) + o) =
                            __floats2bfloat162_rn(v0, v1);
                    if (d.gelu) { v0 = gelu_f(v0); v1 = gelu_f(v1); }
                    if (d.c_bf16)
                        *reinterpret_cast<__nv_bfloat162 *>(static_cast<__nv_bfloat16 *>(d.C) + o) =
                            __floats2bfloat162_rn(v0, v1);
                    else
                        *reinterpret_cast<float2 *>(static_cast<float *>(d.C) + o) = make_float2(v0, v1);
                    continue;
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int nn = n + u;
                    if (nn >= d.N) continue;
                    const long long oo = cz + m * d.scm + nn * d.scn;
                    float v = u ? v1 : v0;
                    if (d.atomic) {
                        atomicAdd(static_cast<float *>(d.C) + oo, v);
                        continue;
                    }
                    if (d.Cin) v += d.beta * d.Cin[oo];
                    if (d.bias) v += d.bias[d.bias_on_m ? m : nn];
                    if (d.pre) static_cast<__nv_bfloat16 *>(d.pre)[oo] = __float2bfloat16(v);
                    if (d.gelu) v = gelu_f(v);
                    if (d.c_bf16) static_cast<__nv_bfloat16 *>(d.C)[oo] = __float2bfloat16(v);
                    else static_cast<float *>(d.C)[oo] = v;
                }
            }
}

// ------------------------------------------------------ tcgen05 GEMM
//
// The same descriptor semantics on the 5th-generation tensor cores.  A CTA of
// 256 threads owns a 128 x BN tile of C held in tensor memory (BN FP32
// columns, one TMEM lane per row).  Each 64-deep K tile of A (128 x 64) and B
// (BN x 64) is copied by all threads with 16-byte cp.async straight into
// shared memory in a canonical no-swizzle layout: K-major when the operand is
// contiguous along K, MN-major when it is contiguous along M (or N), so
// neither case is transposed on the way.  TSTG stages rotate: while one
// elected thread issues the four tcgen05.mma.kind::f16 (BF16 x BF16 -> FP32,
// M = 128, N = BN, K = 16) of a tile and commits them to the stage's
// mbarrier, the copies of the next TSTG - 1 tiles are in flight.  The
// epilogue reads TMEM (warp w: lanes 32 (w % 4).., half the columns each),
// stages the FP32 tile in shared memory and writes C in 8-column vectors.
// Every wait is bounded: on a timeout the kernel records it in g_tc_timeouts
// and finishes without it.

constexpr int TBK = 64;
constexpr int TSTG = 3;
constexpr long long kWaitLimit = 1LL << 22;

__device__ int g_tc_timeouts;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitLimit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// shared-memory matrix descriptor: start >> 4 | LBO >> 4 << 16 | SBO >> 4 << 32
// | version 1 << 46, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void *src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Copies rows [r0, r0 + R) x k [k0, k0 + 64) of an operand, element (r, k) at
// p + r * sr + k * sk, into its canonical no-swizzle layout at shared address
// s; bytes outside the matrix are zero-filled by the copy itself.
//   mode 0 (k contiguous), K-major: (r, k) at ((r/8)*8 + k/8)*128 + (r%8)*16 +
//     (k%8)*2 -- LBO 128 B (next 8 k), SBO 1024 B (next 8 rows);
//   mode 1 (r contiguous), MN-major: (r, k) at (k/8)*R*16 + (r/8)*128 +
//     (k%8)*16 + (r%8)*2 -- SBO 128 B (next 8 rows), LBO R*16 B (next 8 k).
// Lane l of a warp takes the 16-byte group (l % 8) of a core matrix, so each
// 8-lane phase writes eight distinct bank groups, and the warp's 32 groups
// cover whole 32-byte sectors of global memory.
template <int R>
__device__ __forceinline__ void tc_fill(uint32_t s, const __nv_bfloat16 *p, long long sr, long long sk, int rows,
                                        int kk, int r0, int k0, int mode)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < R / 32; q++) {
        const int wq = (threadIdx.x >> 5) + q * 8;      // warp-group of 32 vectors, 0 .. R/4 - 1
        uint32_t dst;
        const __nv_bfloat16 *src = p;
        int bytes = 0;
        if (mode == 0) {
            const int r = (wq >> 1) * 8 + (lane & 7), kc = (wq & 1) * 4 + (lane >> 3);
            const int gr = r0 + r, gk = k0 + kc * 8;
            dst = s + ((r >> 3) * 8 + kc) * 128 + (r & 7) * 16;
            if (gr < rows && gk < kk) {
                src = p + gr * sr + gk;
                bytes = 2 * min(8, kk - gk);
            }
        } else {
            const int k = (wq & 7) * 8 + (lane & 7), rc = (wq >> 3) * 4 + (lane >> 3);
            const int gr = r0 + rc * 8, gk = k0 + k;
            dst = s + (k >> 3) * (R * 16) + rc * 128 + (k & 7) * 16;
            if (gr < rows && gk < kk) {
                src = p + gr + gk * sk;
                bytes = 2 * min(8, rows - gr);
            }
        }
        cp_async16_zfill(dst, src, bytes);
    }
}

// The accumulator of a 128 x BN tile (TMEM lanes = rows) through shared
// memory to C: 8 warps read TMEM (warp w: lanes 32 (w % 4).., half the
// columns each) into an FP32 tile, free the TMEM columns, then every thread
// writes 8-column vectors with the descriptor's epilogue (alpha, beta Cin,
// bias, pre-activation, GELU) or atomic accumulation.  `have` = the
// accumulator is complete (some K tiles, no wait gave up).
template <int BN>
__device__ __forceinline__ void tc_tile_to_smem(uint32_t tmem, float *tile, bool have)
{
    constexpr int TP = BN + 4;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (have) {
        const int row = (warp & 3) * 32 + lane;
        const int cb = (warp >> 2) * (BN / 2);
#pragma unroll 1
        for (int c0 = cb; c0 < cb + BN / 2; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float4 *t4 = reinterpret_cast<float4 *>(tile + row * TP + c0);
#pragma unroll
            for (int j = 0; j < 4; j++)
                t4[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                    __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

template <int BN>
__device__ __forceinline__ void tc_epilogue(const sfg_gemm_desc &d, uint32_t tmem, float *tile, int m0, int n0,
                                            long long cz, bool have)
{
    constexpr int BM = 128;
    constexpr int TP = BN + 4;
    tc_tile_to_smem<BN>(tmem, tile, have);
    if (!have) return;
    // C in vectors of 8 columns: consecutive threads take consecutive vectors
    // of a row
    constexpr int VPR = BN / 8;
    for (int v = threadIdx.x; v < BM * VPR; v += 256) {
        const int rr = v / VPR, cc = (v % VPR) * 8;
        const int m = m0 + rr, nbase = n0 + cc;
        if (m >= d.M || nbase >= d.N) continue;
        const int cnt = min(8, d.N - nbase);
        const float4 *t4 = reinterpret_cast<const float4 *>(tile + rr * TP + cc);
        const float4 q0 = t4[0], q1 = t4[1];
        float x[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        const long long o = cz + m * d.scm + (long long)nbase * d.scn;
        if (d.atomic) {
            for (int j = 0; j < cnt; j++) atomicAdd(static_cast<float *>(d.C) + o + j * d.scn, d.alpha * x[j]);
            continue;
        }
        const bool vec = cnt == 8 && d.scn == 1 && (o & 7) == 0;
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] *= d.alpha;
        if (d.Cin) {
            if (vec && (reinterpret_cast<uintptr_t>(d.Cin) & 15) == 0) {
                const float4 a0 = *reinterpret_cast<const float4 *>(d.Cin + o);
                const float4 a1 = *reinterpret_cast<const float4 *>(d.Cin + o + 4);
                const float cin[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
                for (int j = 0; j < 8; j++) x[j] += d.beta * cin[j];
            } else {
                for (int j = 0; j < cnt; j++) x[j] += d.beta * d.Cin[o + j * d.scn];
            }
        }
        if (d.bias) {
            if (d.bias_on_m) {
                const float b = d.bias[m];
#pragma unroll
                for (int j = 0; j < 8; j++) x[j] += b;
            } else {
                for (int j = 0; j < cnt; j++) x[j] += d.bias[nbase + j];
            }
        }
        if (d.pre) {
            __nv_bfloat16 *pp = static_cast<__nv_bfloat16 *>(d.pre) + o;
            if (vec && (reinterpret_cast<uintptr_t>(d.pre) & 15) == 0) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int j = 0; j < 8; j++) h[j] = __float2bfloat16(x[j]);
                *reinterpret_cast<uint4 *>(pp) = *reinterpret_cast<const uint4 *>(h);
            } else {
                for (int j = 0; j < cnt; j++) pp[j * d.scn] = __float2bfloat16(x[j]);
            }
        }
        if (d.gelu) {
#pragma unroll
            for (int j = 0; j < 8; j++) x[j] = gelu_f(x[j]);
        }
        if (d.c_bf16) {
            __nv_bfloat16 *cp = static_cast<__nv_bfloat16 *>(d.C) + o;
            if (vec && (reinterpret_cast<uintptr_t>(d.C) & 15) == 0) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int j = 0; j < 8; j++) h[j] = __float2bfloat16(x[j]);
                *reinterpret_cast<uint4 *>(cp) = *reinterpret_cast<const uint4 *>(h);
            } else {
                for (int j = 0; j < cnt; j++) cp[j * d.scn] = __float2bfloat16(x[j]);
            }
        } else {
            float *cp = static_cast<float *>(d.C) + o;
            if (vec && (reinterpret_cast<uintptr_t>(d.C) & 15) == 0) {
                *reinterpret_cast<float4 *>(cp) = make_float4(x[0], x[1], x[2], x[3]);
                *reinterpret_cast<float4 *>(cp + 4) = make_float4(x[4], x[5], x[6], x[7]);
            } else {
                for (int j = 0; j < cnt; j++) cp[j * d.scn] = x[j];
            }
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(256) gemm_tc_kernel(const GemmArgs g)
{
    constexpr int BM = 128;
    constexpr int ASTG = BM * TBK * 2, BSTG = BN * TBK * 2;     // bytes of one stage
    constexpr int TP = BN + 4;                                   // epilogue tile pitch (floats)
    static_assert(BM * TP * 4 <= TSTG * (ASTG + BSTG), "epilogue tile must fit the stages");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[TSTG];
    __shared__ uint32_t tmem_base;
    const sfg_gemm_desc &d = g.d;
    const int nb = d.batch1 * d.batch2;
    const int z = blockIdx.z % nb, split = blockIdx.z / nb;
    const int z1 = z / d.batch2, z2 = z % d.batch2;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int ktiles = (d.K + TBK - 1) / TBK;
    const int per = (ktiles + d.splits - 1) / d.splits;
    const int kt0 = split * per, kt1 = min(ktiles, kt0 + per);
    const int nt = max(0, kt1 - kt0);
    const __nv_bfloat16 *A = static_cast<const __nv_bfloat16 *>(d.A) + z1 * d.sa1 + z2 * d.sa2;
    const __nv_bfloat16 *B = static_cast<const __nv_bfloat16 *>(d.B) + z1 * d.sb1 + z2 * d.sb2;
    const long long cz = z1 * d.sc1 + z2 * d.sc2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t sA = smem_u32(smem), sB = sA + TSTG * ASTG;
    // A: K-major (LBO 128, SBO 1024; K = 16 is 256 B on) or MN-major (SBO 128,
    // LBO 128 * 16; K = 16 is 2 LBO on); B likewise with BN rows
    const uint32_t a_lbo = g.amode == 1 ? BM * 16 : 128, a_sbo = g.amode == 1 ? 128 : 1024;
    const uint32_t b_lbo = g.bmode == 1 ? BN * 16 : 128, b_sbo = g.bmode == 1 ? 128 : 1024;
    const uint32_t a_step = g.amode == 1 ? 2 * BM * 16 : 256, b_step = g.bmode == 1 ? 2 * BN * 16 : 256;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(g.amode == 1) << 15) |
                           ((uint32_t)(g.bmode == 1) << 16) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < TSTG; s++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    bool ok = true;
    // prologue: the first TSTG - 1 tiles in flight (one commit group each)
#pragma unroll
    for (int s = 0; s < TSTG - 1; s++) {
        if (s < nt) {
            const int k0 = (kt0 + s) * TBK;
            tc_fill<BM>(sA + s * ASTG, A, d.sam, d.sak, d.M, d.K, m0, k0, g.amode);
            tc_fill<BN>(sB + s * BSTG, B, d.sbn, d.sbk, d.N, d.K, n0, k0, g.bmode);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int it = 0; it < nt; it++) {
        const int st = it % TSTG;
        asm volatile("cp.async.wait_group %0;" ::"n"(TSTG - 2) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = sA + st * ASTG, b0 = sB + st * BSTG;
#pragma unroll
            for (int ks = 0; ks < TBK / 16; ks++) {
                const uint64_t da = umma_desc(a0 + ks * a_step, a_lbo, a_sbo);
                const uint64_t db = umma_desc(b0 + ks * b_step, b_lbo, b_sbo);
                const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&bars[st])));
        }
        // refill the stage the previous tile used, once its MMAs have read it
        const int nxt = it + TSTG - 1;
        if (nxt < nt) {
            const int sn = nxt % TSTG;
            if (it >= 1) ok = mbar_wait(smem_u32(&bars[sn]), ((it - 1) / TSTG) & 1) && ok;
            const int k0 = (kt0 + nxt) * TBK;
            tc_fill<BM>(sA + sn * ASTG, A, d.sam, d.sak, d.M, d.K, m0, k0, g.amode);
            tc_fill<BN>(sB + sn * BSTG, B, d.sbn, d.sbk, d.N, d.K, n0, k0, g.bmode);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (nt > 0) ok = mbar_wait(smem_u32(&bars[(nt - 1) % TSTG]), ((nt - 1) / TSTG) & 1) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok && lane == 0) atomicAdd(&g_tc_timeouts, 1);
    // all threads agree on whether the accumulator is complete
    const int good = __syncthreads_and(ok ? 1 : 0);
    tc_epilogue<BN>(d, tmem, reinterpret_cast<float *>(smem), m0, n0, cz, nt > 0 && good);
}

// ------------------------------------------------ tcgen05 GEMM with TMA
//
// The same tile and epilogue, with the operand tiles brought in by the
// Tensor Memory Accelerator: one thread issues, per stage, the bulk tensor
// copies of the A and B tiles (cp.async.bulk.tensor, completion counted in
// bytes on the stage's mbarrier) and then the stage's four
// tcgen05.mma.kind::f16, committed to a second mbarrier that frees the stage
// for the copies TSTG tiles later.  The tiles land in shared memory in the
// canonical 128-byte-swizzled layouts: K-major for a k-contiguous operand
// (one box of 64 k x R rows, rows 128 B apart, 8-row groups 1024 B apart),
// MN-major for an m/n-contiguous one (R / 64 boxes of 64 m/n x 64 k, k rows
// 128 B apart, 8-row groups 1024 B apart, 64-element blocks 8 KB apart).
// The copies zero-fill outside the matrix, so ragged M, N and K need no
// special case.  The other 255 threads wait for the last commit and run the
// epilogue.  Every wait is bounded (g_tc_timeouts).

// shared-memory descriptor with the 128-byte swizzle (layout type 2)
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return umma_desc(saddr, lbo, sbo) | (2ull << 61);
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// the k-tile at k0 of rows [r0, r0 + R) of one operand (MODE 0: k
// contiguous, MODE 1: rows contiguous) into the stage at dst
template <int MODE, int R>
__device__ __forceinline__ void tma_operand(uint32_t dst, const CUtensorMap *map, int k0, int r0, int z2, int z1,
                                            uint32_t bar)
{
    if (MODE == 0) {
        tma_load_4d(dst, map, k0, r0, z2, z1, bar);
    } else {
#pragma unroll
        for (int j = 0; j < R / 64; j++) tma_load_4d(dst + j * 8192, map, r0 + 64 * j, k0, z2, z1, bar);
    }
}

// The fused head of the surrogate's inference, straight from TMEM: warp w
// reads rows 32 (w % 4).. and half the columns (tcgen05.ld, 16 at a time),
// applies alpha, bias and GELU in registers and accumulates the n2 dot
// products with w2 (bias and w2 staged in shared memory, read as
// broadcasts); the two column halves of a row meet in shared memory and the
// lower half writes y.  The hidden layer never leaves the SM.
template <int BN>
__device__ __forceinline__ void head_from_tmem(const GemmArgs &g, uint32_t tmem, float *scratch, int m0, int z1,
                                               bool have)
{
    const sfg_gemm_desc &d = g.d;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *sb = scratch;                    // [BN] bias
    float *sw = scratch + BN;               // [BN][4] w2 (zero past N and n2)
    float *part = scratch + 5 * BN;         // [128][4] sums of the upper column half
    for (int c = threadIdx.x; c < BN; c += 256) {
        sb[c] = (c < d.N && d.bias) ? d.bias[c] : 0.f;
#pragma unroll
        for (int j = 0; j < 4; j++) sw[4 * c + j] = (c < d.N && j < g.n2) ? g.w2[c * g.n2 + j] : 0.f;
    }
    __syncthreads();
    const int row = (warp & 3) * 32 + lane;
    const int cb = (warp >> 2) * (BN / 2);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (have) {
#pragma unroll 1
        for (int c0 = cb; c0 < cb + BN / 2; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (c0 >= d.N) continue;
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int c = c0 + j;
                const float v = gelu_f(d.alpha * __uint_as_float(r[j]) + sb[c]);
                const float4 w = *reinterpret_cast<const float4 *>(sw + 4 * c);
                acc[0] += v * w.x; acc[1] += v * w.y; acc[2] += v * w.z; acc[3] += v * w.w;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    if (warp >= 4) {
#pragma unroll
        for (int j = 0; j < 4; j++) part[4 * row + j] = acc[j];
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
    const int m = m0 + row;
    if (have && warp < 4 && m < d.M)
        for (int j = 0; j < g.n2; j++)
            g.y[z1 * g.ys1 + j * g.ysj + m] = acc[j] + part[4 * row + j] + (g.b2 ? g.b2[j] : 0.f);
}

template <int BN, int AMODE, int BMODE, bool HEAD = false>
__global__ void __launch_bounds__(256) gemm_tma_kernel(const __grid_constant__ GemmArgs g,
                                                        const __grid_constant__ CUtensorMap ta,
                                                        const __grid_constant__ CUtensorMap tb)
{
    constexpr int BM = 128;
    constexpr int ASTG = BM * TBK * 2, BSTG = BN * TBK * 2;     // bytes of one stage
    static_assert(BM * (BN + 4) * 4 <= TSTG * (ASTG + BSTG), "epilogue tile must fit the stages");
    static_assert(BMODE == 0 || BN % 64 == 0, "MN-major tiles come in 64-element blocks");
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[TSTG], empty[TSTG];
    __shared__ uint32_t tmem_base;
    const sfg_gemm_desc &d = g.d;
    const int nb = d.batch1 * d.batch2;
    const int z = blockIdx.z % nb, split = blockIdx.z / nb;
    const int z1 = z / d.batch2, z2 = z % d.batch2;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int ktiles = (d.K + TBK - 1) / TBK;
    const int per = (ktiles + d.splits - 1) / d.splits;
    const int kt0 = split * per, kt1 = min(ktiles, kt0 + per);
    const int nt = max(0, kt1 - kt0);
    const long long cz = z1 * d.sc1 + z2 * d.sc2;
    const int warp = threadIdx.x >> 5;
    // stages on a 1024-byte boundary (the swizzle atom); the launch adds the slack
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sA = (raw + 1023u) & ~1023u, sB = sA + TSTG * ASTG;
    unsigned char *stages = smem_raw + (sA - raw);
    const int az1 = g.tz1a ? z1 : 0, az2 = g.tz2a ? z2 : 0, bz1 = g.tz1b ? z1 : 0, bz2 = g.tz2b ? z2 : 0;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)AMODE << 15) |
                               ((uint32_t)BMODE << 16) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    // K = 16 steps: 32 bytes along a K-major row, two 8-row groups of an MN-major tile
    constexpr uint32_t A_STEP = AMODE ? 2048 : 32, B_STEP = BMODE ? 2048 : 32;
    constexpr uint32_t A_LBO = AMODE ? 8192 : 16, B_LBO = BMODE ? 8192 : 16;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < TSTG; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    bool ok = true;
    if (threadIdx.x == 0) {
        auto issue = [&](int s, int t) {
            const uint32_t bar = smem_u32(&full[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(ASTG + BSTG)
                         : "memory");
            const int k0 = (kt0 + t) * TBK;
            tma_operand<AMODE, BM>(sA + s * ASTG, &ta, k0, m0, az2, az1, bar);
            tma_operand<BMODE, BN>(sB + s * BSTG, &tb, k0, n0, bz2, bz1, bar);
        };
        int issued = 0, used = 0;
        for (; issued < min(TSTG, nt); issued++) issue(issued, issued);
        for (int it = 0; it < nt; it++) {
            const int st = it % TSTG;
            if (!mbar_wait(smem_u32(&full[st]), (it / TSTG) & 1)) { ok = false; break; }
            used = it + 1;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = sA + st * ASTG, b0 = sB + st * BSTG;
#pragma unroll
            for (int ks = 0; ks < TBK / 16; ks++) {
                const uint64_t da = umma_desc_sw128(a0 + ks * A_STEP, A_LBO, 1024);
                const uint64_t db = umma_desc_sw128(b0 + ks * B_STEP, B_LBO, 1024);
                const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(IDESC), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&empty[st])));
            // refill the stage the previous tile used, once its MMAs have read it
            const int prev = it - 1;
            if (prev >= 0 && prev + TSTG < nt) {
                if (!mbar_wait(smem_u32(&empty[prev % TSTG]), (prev / TSTG) & 1)) { ok = false; break; }
                issue(prev % TSTG, prev + TSTG);
                issued++;
            }
        }
        // after a wait gave up: let the copies already issued land before the block exits
        for (int t = used; !ok && t < issued; t++) mbar_wait(smem_u32(&full[t % TSTG]), (t / TSTG) & 1);
    }
    if (nt > 0) ok = mbar_wait(smem_u32(&empty[(nt - 1) % TSTG]), ((nt - 1) / TSTG) & 1) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok && (threadIdx.x & 31) == 0) atomicAdd(&g_tc_timeouts, 1);
    const int good = __syncthreads_and(ok ? 1 : 0);
    if constexpr (HEAD) {
        head_from_tmem<BN>(g, tmem, reinterpret_cast<float *>(stages), m0, z1, nt > 0 && good);
    } else {
        tc_epilogue<BN>(d, tmem, reinterpret_cast<float *>(stages), m0, n0, cz, nt > 0 && good);
    }
}

// ------------------------------------- persistent tcgen05 GEMM (TMA tiles)
//
// One CTA per SM walks a list of output tiles (batch, split, 128-row tile,
// BN-column tile; consecutive tiles share their A rows).  Three roles run
// side by side on their own mbarriers:
//   warp 0 (one thread)  TMA producer: the A and B k-tiles of every tile in
//                        turn into a ring of PSTG stages;
//   warp 1 (one thread)  MMA issuer: tcgen05.mma into one of two TMEM
//                        accumulators, a commit per stage (frees it for the
//                        producer) and one per tile (hands the accumulator to
//                        the epilogue);
//   warps 4-7            epilogue: tcgen05.ld of the accumulator (warp w:
//                        TMEM lanes 32 (w % 4)..), the descriptor's epilogue
//                        in registers, 16-column stores per row, then the
//                        accumulator back to the MMA issuer.
// So the loads of tile i + 1 and its MMAs overlap the epilogue of tile i,
// and TMEM allocation, barrier set-up and tensor-map prefetch happen once per
// CTA instead of once per tile.  Every wait is bounded; the first one that
// gives up sets a flag that ends every other wait of the CTA at once.

constexpr int PSTG = 4;

__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, volatile int *abort)
{
    for (long long i = 0; i < kWaitLimit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63) == 63 && *abort) return false;
    }
    *abort = 1;
    return false;
}

struct TileCoord {
    int z1, z2, m0, n0, kt0, nt;
    long long cz;
};

__device__ __forceinline__ TileCoord tile_coord(const sfg_gemm_desc &d, int item, int tm, int tn, int BN)
{
    TileCoord c;
    const int per_z = tm * tn;
    const int zs = item / per_z, rem = item % per_z;
    const int nb = d.batch1 * d.batch2;
    const int z = zs % nb, split = zs / nb;
    c.z1 = z / d.batch2;
    c.z2 = z % d.batch2;
    c.m0 = (rem / tn) * 128;
    c.n0 = (rem % tn) * BN;
    const int ktiles = (d.K + TBK - 1) / TBK;
    const int per = (ktiles + d.splits - 1) / d.splits;
    c.kt0 = split * per;
    c.nt = max(0, min(ktiles, c.kt0 + per) - c.kt0);
    c.cz = c.z1 * d.sc1 + c.z2 * d.sc2;
    return c;
}

// Columns n0 .. n0 + 15 of row m with the descriptor's epilogue.
__device__ __forceinline__ void store_row16(const sfg_gemm_desc &d, const uint32_t *r, int m, int n0, long long cz)
{
    if (m >= d.M || n0 >= d.N) return;
    const int cnt = min(16, d.N - n0);
    const long long o = cz + m * d.scm + (long long)n0 * d.scn;
    float x[16];
#pragma unroll
    for (int j = 0; j < 16; j++) x[j] = d.alpha * __uint_as_float(r[j]);
    if (d.atomic) {
        for (int j = 0; j < cnt; j++) atomicAdd(static_cast<float *>(d.C) + o + j * d.scn, x[j]);
        return;
    }
    const bool vec = cnt == 16 && d.scn == 1 && (o & 7) == 0;
    if (d.Cin) {
        if (vec && (reinterpret_cast<uintptr_t>(d.Cin) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 a = *reinterpret_cast<const float4 *>(d.Cin + o + 4 * q);
                x[4 * q] += d.beta * a.x; x[4 * q + 1] += d.beta * a.y;
                x[4 * q + 2] += d.beta * a.z; x[4 * q + 3] += d.beta * a.w;
            }
        } else {
            for (int j = 0; j < cnt; j++) x[j] += d.beta * d.Cin[o + j * d.scn];
        }
    }
    if (d.bias) {
        if (d.bias_on_m) {
            const float b = d.bias[m];
#pragma unroll
            for (int j = 0; j < 16; j++) x[j] += b;
        } else {
            for (int j = 0; j < cnt; j++) x[j] += d.bias[n0 + j];
        }
    }
    if (d.pre) {
        __nv_bfloat16 *pp = static_cast<__nv_bfloat16 *>(d.pre) + o;
        if (vec && (reinterpret_cast<uintptr_t>(d.pre) & 15) == 0) {
            __align__(16) __nv_bfloat16 h[16];
#pragma unroll
            for (int j = 0; j < 16; j++) h[j] = __float2bfloat16(x[j]);
            reinterpret_cast<uint4 *>(pp)[0] = reinterpret_cast<const uint4 *>(h)[0];
            reinterpret_cast<uint4 *>(pp)[1] = reinterpret_cast<const uint4 *>(h)[1];
        } else {
            for (int j = 0; j < cnt; j++) pp[j * d.scn] = __float2bfloat16(x[j]);
        }
    }
    if (d.gelu) {
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = gelu_f(x[j]);
    }
    if (d.c_bf16) {
        __nv_bfloat16 *cp = static_cast<__nv_bfloat16 *>(d.C) + o;
        if (vec && (reinterpret_cast<uintptr_t>(d.C) & 15) == 0) {
            __align__(16) __nv_bfloat16 h[16];
#pragma unroll
            for (int j = 0; j < 16; j++) h[j] = __float2bfloat16(x[j]);
            reinterpret_cast<uint4 *>(cp)[0] = reinterpret_cast<const uint4 *>(h)[0];
            reinterpret_cast<uint4 *>(cp)[1] = reinterpret_cast<const uint4 *>(h)[1];
        } else {
            for (int j = 0; j < cnt; j++) cp[j * d.scn] = __float2bfloat16(x[j]);
        }
    } else {
        float *cp = static_cast<float *>(d.C) + o;
        if (vec && (reinterpret_cast<uintptr_t>(d.C) & 15) == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++)
                reinterpret_cast<float4 *>(cp)[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
        } else {
            for (int j = 0; j < cnt; j++) cp[j * d.scn] = x[j];
        }
    }
}

template <int BN, int AMODE, int BMODE>
__global__ void __launch_bounds__(256, 1) gemm_persist_kernel(const __grid_constant__ GemmArgs g,
                                                               const __grid_constant__ CUtensorMap ta,
                                                               const __grid_constant__ CUtensorMap tb, int items)
{
    constexpr int BM = 128;
    constexpr int ASTG = BM * TBK * 2, BSTG = BN * TBK * 2;
    static_assert(BMODE == 0 || BN % 64 == 0, "MN-major tiles come in 64-element blocks");
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[PSTG], empty[PSTG], tfull[2], tempty[2];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const sfg_gemm_desc &d = g.d;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tm = (d.M + BM - 1) / BM, tn = (d.N + BN - 1) / BN;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sA = (raw + 1023u) & ~1023u, sB = sA + PSTG * ASTG;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)AMODE << 15) |
                               ((uint32_t)BMODE << 16) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    constexpr uint32_t A_STEP = AMODE ? 2048 : 32, B_STEP = BMODE ? 2048 : 32;
    constexpr uint32_t A_LBO = AMODE ? 8192 : 16, B_LBO = BMODE ? 8192 : 16;
    volatile int *abort = &abort_flag;
    if (threadIdx.x == 0) {
        abort_flag = 0;
#pragma unroll
        for (int s = 0; s < PSTG; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
        }
#pragma unroll
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tfull[b])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&tempty[b])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(2 * BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    bool ok = true;
    if (warp == 0 && lane == 0) {
        // TMA producer
        long long gk = 0;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const TileCoord tc = tile_coord(d, item, tm, tn, BN);
            const int az1 = g.tz1a ? tc.z1 : 0, az2 = g.tz2a ? tc.z2 : 0;
            const int bz1 = g.tz1b ? tc.z1 : 0, bz2 = g.tz2b ? tc.z2 : 0;
            for (int t = 0; t < tc.nt; t++, gk++) {
                const int s = (int)(gk % PSTG);
                if (gk >= PSTG && !mbar_wait_or_abort(smem_u32(&empty[s]), (uint32_t)(((gk / PSTG) - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                const uint32_t bar = smem_u32(&full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(ASTG + BSTG)
                             : "memory");
                const int k0 = (tc.kt0 + t) * TBK;
                tma_operand<AMODE, BM>(sA + s * ASTG, &ta, k0, tc.m0, az2, az1, bar);
                tma_operand<BMODE, BN>(sB + s * BSTG, &tb, k0, tc.n0, bz2, bz1, bar);
            }
        }
        // on an abort, let the copies already issued land before the CTA ends
        if (!ok)
            for (long long q = (gk > PSTG ? gk - PSTG : 0); q < gk; q++)
                mbar_wait(smem_u32(&full[q % PSTG]), (uint32_t)((q / PSTG) & 1));
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        long long gk = 0;
        int j = 0;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x, j++) {
            const TileCoord tc = tile_coord(d, item, tm, tn, BN);
            const int ab = j & 1, use = j >> 1;
            if (use >= 1 && !mbar_wait_or_abort(smem_u32(&tempty[ab]), (uint32_t)((use - 1) & 1), abort)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t acc_addr = tmem + (uint32_t)(ab * BN);
            for (int t = 0; t < tc.nt; t++, gk++) {
                const int s = (int)(gk % PSTG);
                if (!mbar_wait_or_abort(smem_u32(&full[s]), (uint32_t)((gk / PSTG) & 1), abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = sA + s * ASTG, b0 = sB + s * BSTG;
#pragma unroll
                for (int ks = 0; ks < TBK / 16; ks++) {
                    const uint64_t da = umma_desc_sw128(a0 + ks * A_STEP, A_LBO, 1024);
                    const uint64_t db = umma_desc_sw128(b0 + ks * B_STEP, B_LBO, 1024);
                    const uint32_t acc = (t > 0 || ks > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(acc_addr),
                        "l"(da), "l"(db), "r"(IDESC), "r"(acc));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&empty[s])));
            }
            if (!ok) break;
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&tfull[ab])));
        }
    } else if (warp >= 4) {
        // epilogue
        const int row = (warp & 3) * 32 + lane;
        int j = 0;
        for (int item = blockIdx.x; item < items; item += gridDim.x, j++) {
            const TileCoord tc = tile_coord(d, item, tm, tn, BN);
            const int ab = j & 1, use = j >> 1;
            if (!mbar_wait_or_abort(smem_u32(&tfull[ab]), (uint32_t)(use & 1), abort)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t r[16];
                __syncwarp();   // tcgen05.ld is .aligned: the warp converges after the stores' branches
                const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(ab * BN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (tc.nt > 0) store_row16(d, r, tc.m0 + row, tc.n0 + c0, tc.cz);
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[ab])) : "memory");
        }
    }
    if (!ok && (threadIdx.x & 31) == 0) atomicAdd(&g_tc_timeouts, 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    __syncwarp();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
}

// Vector loads need 16-byte aligned groups of 8 elements: the base pointer
// and every stride other than the contiguous one must keep that alignment.
int pick_mode(long long s_row, long long s_k, long long s1, long long s2, const void *p)
{
    const bool al = (reinterpret_cast<uintptr_t>(p) & 15) == 0 && s1 % 8 == 0 && s2 % 8 == 0;
    if (s_k == 1 && s_row % 8 == 0 && al) return 0;
    if (s_row == 1 && s_k % 8 == 0 && al) return 1;
    return 2;
}

// ------------------------------------------------------- pointwise kernels

constexpr int KC = 16, KD = 32;    // kept W modes, kept D modes (16 + 16)

// P[z][64][32]: rows 0-31 = cos-rows times [Yre | Yim], rows 32-63 sin-rows.
// Z = sum_d e^{-i theta} Y:  Zre = C.Yre + S.Yim,  Zim = C.Yim - S.Yre.
__global__ void dft_combine_kernel(const float *__restrict__ P, __nv_bfloat16 *__restrict__ Z, int B, int C)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)B * C * KD * KC;
    if (t >= total) return;
    const int k2 = (int)(t % KC);
    const int k1 = (int)((t / KC) % KD);
    const long long zz = t / (KC * KD);            // b * C + c
    const int c = (int)(zz % C), b = (int)(zz / C);
    const float *p = P + zz * 64 * 32;
    const float re = p[k1 * 32 + k2] + p[(32 + k1) * 32 + 16 + k2];
    const float im = p[k1 * 32 + 16 + k2] - p[(32 + k1) * 32 + k2];
    const long long mode = k1 * KC + k2;
    __nv_bfloat16 *o = Z + (mode * B + b) * 2 * C;
    o[c] = __float2bfloat16(re);
    o[C + c] = __float2bfloat16(im);
}

__global__ void dft_combine_bwd_kernel(const __nv_bfloat16 *__restrict__ dZ, __nv_bfloat16 *__restrict__ dP, int B,
                                       int C)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)B * C * KD * KC;
    if (t >= total) return;
    const int k2 = (int)(t % KC);
    const int k1 = (int)((t / KC) % KD);
    const long long zz = t / (KC * KD);
    const int c = (int)(zz % C), b = (int)(zz / C);
    const long long mode = k1 * KC + k2;
    const __nv_bfloat16 *g = dZ + (mode * B + b) * 2 * C;
    const __nv_bfloat16 re = g[c], im = g[C + c];
    __nv_bfloat16 *p = dP + zz * 64 * 32;
    p[k1 * 32 + k2] = re;
    p[(32 + k1) * 32 + 16 + k2] = re;
    p[k1 * 32 + 16 + k2] = im;
    p[(32 + k1) * 32 + k2] = __float2bfloat16(-__bfloat162float(im));
}

// Tiled versions for C a multiple of 16: a block takes 16 channels of one
// shot and 128 modes and turns the transpose between the per-plane P layout
// and the per-mode Zmix layout through shared memory, so both sides move
// whole 32-byte sectors (the one-thread-per-element versions above write or
// read Zmix two bytes at a time).
constexpr int CMB_C = 16, CMB_M = 128;

__global__ void __launch_bounds__(256) dft_combine_tiled(const float *__restrict__ P, __nv_bfloat16 *__restrict__ Z,
                                                         int B, int C)
{
    __shared__ __align__(16) __nv_bfloat16 s[CMB_M][2][CMB_C];
    const int b = blockIdx.z, c0 = blockIdx.y * CMB_C, mode0 = blockIdx.x * CMB_M;
    for (int idx = threadIdx.x; idx < CMB_C * CMB_M; idx += 256) {
        const int cl = idx / CMB_M, ml = idx % CMB_M, mode = mode0 + ml;
        const int k1 = mode / KC, k2 = mode % KC;
        const float *p = P + ((long long)b * C + c0 + cl) * 64 * 32;
        s[ml][0][cl] = __float2bfloat16(p[k1 * 32 + k2] + p[(32 + k1) * 32 + 16 + k2]);
        s[ml][1][cl] = __float2bfloat16(p[k1 * 32 + 16 + k2] - p[(32 + k1) * 32 + k2]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < CMB_M * 2 * 2; idx += 256) {
        const int ml = idx >> 2, part = (idx >> 1) & 1, h = idx & 1;
        __nv_bfloat16 *o = Z + ((long long)(mode0 + ml) * B + b) * 2 * C + part * C + c0 + h * 8;
        *reinterpret_cast<uint4 *>(o) = *reinterpret_cast<const uint4 *>(&s[ml][part][h * 8]);
    }
}

__global__ void __launch_bounds__(256) dft_combine_bwd_tiled(const __nv_bfloat16 *__restrict__ dZ,
                                                             __nv_bfloat16 *__restrict__ dP, int B, int C)
{
    __shared__ __align__(16) __nv_bfloat16 s[CMB_M][2][CMB_C];
    const int b = blockIdx.z, c0 = blockIdx.y * CMB_C, mode0 = blockIdx.x * CMB_M;
    for (int idx = threadIdx.x; idx < CMB_M * 2 * 2; idx += 256) {
        const int ml = idx >> 2, part = (idx >> 1) & 1, h = idx & 1;
        const __nv_bfloat16 *g = dZ + ((long long)(mode0 + ml) * B + b) * 2 * C + part * C + c0 + h * 8;
        *reinterpret_cast<uint4 *>(&s[ml][part][h * 8]) = *reinterpret_cast<const uint4 *>(g);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < CMB_C * CMB_M; idx += 256) {
        const int cl = idx / CMB_M, ml = idx % CMB_M, mode = mode0 + ml;
        const int k1 = mode / KC, k2 = mode % KC;
        const __nv_bfloat16 re = s[ml][0][cl], im = s[ml][1][cl];
        __nv_bfloat16 *p = dP + ((long long)b * C + c0 + cl) * 64 * 32;
        p[k1 * 32 + k2] = re;
        p[(32 + k1) * 32 + 16 + k2] = re;
        p[k1 * 32 + 16 + k2] = im;
        p[(32 + k1) * 32 + k2] = __float2bfloat16(-__bfloat162float(im));
    }
}

__global__ void expand_weights_kernel(const float *__restrict__ Wr, const float *__restrict__ Wi,
                                      __nv_bfloat16 *__restrict__ Wb, int modes, int C)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)modes * C * C) return;
    const int o = (int)(t % C), i = (int)((t / C) % C);
    const long long mode = t / ((long long)C * C);
    const float r = Wr[t], im = Wi[t];
    __nv_bfloat16 *w = Wb + mode * 4 * C * C;
    const int C2 = 2 * C;
    w[i * C2 + o] = __float2bfloat16(r);
    w[i * C2 + C + o] = __float2bfloat16(im);
    w[(C + i) * C2 + o] = __float2bfloat16(-im);
    w[(C + i) * C2 + C + o] = __float2bfloat16(r);
}

__global__ void fold_weights_kernel(const float *__restrict__ dWb, float *__restrict__ dWr, float *__restrict__ dWi,
                                    int modes, int C)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)modes * C * C) return;
    const int o = (int)(t % C), i = (int)((t / C) % C);
    const long long mode = t / ((long long)C * C);
    const float *w = dWb + mode * 4 * C * C;
    const int C2 = 2 * C;
    dWr[t] += w[i * C2 + o] + w[(C + i) * C2 + C + o];
    dWi[t] += w[i * C2 + C + o] - w[(C + i) * C2 + o];
}

__global__ void gelu_bwd_kernel(const void *__restrict__ dy, int dy_bf16, const __nv_bfloat16 *__restrict__ pre,
                                __nv_bfloat16 *__restrict__ dx, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float x = __bfloat162float(pre[t]);
    const float g = dy_bf16 ? __bfloat162float(static_cast<const __nv_bfloat16 *>(dy)[t])
                            : static_cast<const float *>(dy)[t];
    // d/dx [x Phi(x)] = Phi(x) + x phi(x)
    const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    dx[t] = __float2bfloat16(g * (cdf + x * pdf));
}

__global__ void cast_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = __float2bfloat16(x[t]);
}

// Block (c, slice): the sum over one slice of the outer index and all of the
// inner index of channel c, added to db[c].
__global__ void bias_grad_kernel(const __nv_bfloat16 *__restrict__ dy, float *__restrict__ db, int outer, int C,
                                 long long inner)
{
    const int c = blockIdx.x;
    const long long per = (outer + gridDim.y - 1) / gridDim.y;
    const long long o0 = blockIdx.y * per, o1 = min((long long)outer, o0 + per);
    const long long cnt = (o1 > o0 ? o1 - o0 : 0) * inner;
    float s = 0.f;
    for (long long q = threadIdx.x; q < cnt; q += blockDim.x) {
        const long long o = o0 + q / inner, i = q % inner;
        s += __bfloat162float(dy[(o * C + c) * inner + i]);
    }
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0 && red[0] != 0.f) atomicAdd(db + c, red[0]);
}

// y[j][i][k] = x[i][j][k] (BF16)
__global__ void swap01_kernel(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ y, int n0, int n1,
                              long long n2)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)n0 * n1 * n2;
    if (t >= total) return;
    const long long k = t % n2;
    const long long i = (t / n2) % n0;
    const long long j = t / (n2 * n0);
    y[t] = x[(i * n1 + j) * n2 + k];
}

__global__ void zero_kernel(float *__restrict__ p, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) p[t] = 0.f;
}

__global__ void scale_kernel(float *__restrict__ p, long long n, float a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) p[t] *= a;
}

// per shot: scratch[2b] = |pred-target|^2, scratch[2b+1] = |target|^2
__global__ void rel_loss_sums(const float *__restrict__ pred, const __nv_bfloat16 *__restrict__ tgt, float *scratch,
                              long long n)
{
    const int b = blockIdx.y;
    const float *p = pred + b * n;
    const __nv_bfloat16 *q = tgt + b * n;
    float e = 0.f, r = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float tv = __bfloat162float(q[i]), d = p[i] - tv;
        e += d * d;
        r += tv * tv;
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(scratch + 2 * b, e);
        atomicAdd(scratch + 2 * b + 1, r);
    }
}

__global__ void rel_loss_grad(const float *__restrict__ pred, const __nv_bfloat16 *__restrict__ tgt,
                              const float *__restrict__ scratch, float *loss, __nv_bfloat16 *__restrict__ dpred, int B,
                              long long n)
{
    const int b = blockIdx.y;
    const float den = fmaxf(scratch[2 * b + 1], 1e-30f);
    if (blockIdx.x == 0 && threadIdx.x == 0 && loss) loss[b] = scratch[2 * b] / den;
    if (!dpred) return;
    const float s = 2.f / ((float)B * den);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dpred[b * n + i] = __float2bfloat16(s * (pred[b * n + i] - __bfloat162float(tgt[b * n + i])));
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

unsigned grid_of(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int launched() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

}  // namespace

// The automatic engine choice: tcgen05 tiles for GEMMs with at least half a
// 128-row tile, 32 columns and 64-deep K (the surrogate's depth-to-time map,
// M = 64, runs 1.9x faster on half-filled tcgen05 tiles than on mma.sync);
// mma.sync tiles otherwise.
bool tc_auto(const sfg_gemm_desc &d) { return d.M >= 64 && d.N >= 32 && d.K >= 64; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver the runtime loaded (no link-time
// dependency on libcuda); null when unavailable
EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// Tensor map of one BF16 operand of `rows` x K (element (r, k) at
// base + r * s_row + k * s_k, batches at s1 / s2), boxes as gemm_tma_kernel
// loads them with the 128-byte swizzle: mode 0 (s_k = 1) dims {K, rows, b2,
// b1}, box {64, R}; mode 1 (s_row = 1) dims {rows, K, b2, b1}, box {64, 64}.
// A batch dimension with stride 0 (an operand shared by every batch) or a
// single batch is kept at extent 1 and coordinate 0 (t1 / t2 = 0).
bool operand_map(CUtensorMap *map, const void *base, int mode, int rows, int K, long long s_row, long long s_k,
                 long long s1, long long s2, int b1, int b2, int R, int &t1, int &t2)
{
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    cuuint64_t dim[4], str[3];
    cuuint32_t box[4], es[4] = {1, 1, 1, 1};
    if (mode == 0) {
        dim[0] = (cuuint64_t)K; dim[1] = (cuuint64_t)rows; str[0] = (cuuint64_t)s_row * 2;
        box[0] = 64; box[1] = (cuuint32_t)R;
    } else {
        dim[0] = (cuuint64_t)rows; dim[1] = (cuuint64_t)K; str[0] = (cuuint64_t)s_k * 2;
        box[0] = 64; box[1] = 64;
    }
    auto up16 = [](cuuint64_t v) { return (v + 15) / 16 * 16; };
    t2 = (b2 > 1 && s2 != 0) ? 1 : 0;
    t1 = (b1 > 1 && s1 != 0) ? 1 : 0;
    dim[2] = t2 ? (cuuint64_t)b2 : 1;
    str[1] = t2 ? (cuuint64_t)s2 * 2 : up16(str[0] * dim[1]);
    dim[3] = t1 ? (cuuint64_t)b1 : 1;
    str[2] = t1 ? (cuuint64_t)s1 * 2 : up16(str[1] * dim[2]);
    box[2] = box[3] = 1;
    for (int i = 0; i < 3; i++)
        if (str[i] == 0 || str[i] % 16 != 0 || str[i] >= (1ull << 40)) return false;
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dim, str, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int AM, int BMD, bool HEAD = false>
int launch_tma_shape(const GemmArgs &g, const CUtensorMap &ta, const CUtensorMap &tb, long long nb, cudaStream_t st)
{
    const sfg_gemm_desc &d = g.d;
    const int smem = TSTG * (128 + BN) * TBK * 2 + 1024;
    if (cudaFuncSetAttribute(gemm_tma_kernel<BN, AM, BMD, HEAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return 2;
    dim3 grid((d.N + BN - 1) / BN, (d.M + 127) / 128, (unsigned)nb);
    if (grid.y > 65535) return 1;
    gemm_tma_kernel<BN, AM, BMD, HEAD><<<grid, 256, smem, st>>>(g, ta, tb);
    return launched();
}

template <int BN, int AM, int BMD>
int launch_persist_shape(const GemmArgs &g, const CUtensorMap &ta, const CUtensorMap &tb, long long nb,
                         cudaStream_t st)
{
    const sfg_gemm_desc &d = g.d;
    const int smem = PSTG * (128 + BN) * TBK * 2 + 1024;
    if (cudaFuncSetAttribute(gemm_persist_kernel<BN, AM, BMD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
        return 2;
    const long long items = nb * (long long)((d.M + 127) / 128) * ((d.N + BN - 1) / BN);
    if (items > 0x7fffffffLL) return 1;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::min<long long>(items, sms);
    gemm_persist_kernel<BN, AM, BMD><<<grid, 256, smem, st>>>(g, ta, tb, (int)items);
    return launched();
}

// tcgen05 with TMA operand tiles (persistent, or one tile per CTA); -1 when
// the operands do not allow it (the caller then takes the cp.async engine)
template <int BN>
int launch_tma(GemmArgs g, long long nb, cudaStream_t st, bool persistent)
{
    const sfg_gemm_desc &d = g.d;
    if (g.bmode == 1 && BN % 64 != 0) return -1;
    CUtensorMap ta, tb;
    if (!operand_map(&ta, d.A, g.amode, d.M, d.K, d.sam, d.sak, d.sa1, d.sa2, d.batch1, d.batch2, 128, g.tz1a,
                     g.tz2a) ||
        !operand_map(&tb, d.B, g.bmode, d.N, d.K, d.sbn, d.sbk, d.sb1, d.sb2, d.batch1, d.batch2, BN, g.tz1b,
                     g.tz2b))
        return -1;
    if (persistent) {
        if (g.amode == 0 && g.bmode == 0) return launch_persist_shape<BN, 0, 0>(g, ta, tb, nb, st);
        if (g.amode == 1 && g.bmode == 0) return launch_persist_shape<BN, 1, 0>(g, ta, tb, nb, st);
        if constexpr (BN % 64 == 0) {
            if (g.amode == 0) return launch_persist_shape<BN, 0, 1>(g, ta, tb, nb, st);
            return launch_persist_shape<BN, 1, 1>(g, ta, tb, nb, st);
        }
        return -1;
    }
    if (g.amode == 0 && g.bmode == 0) return launch_tma_shape<BN, 0, 0>(g, ta, tb, nb, st);
    if (g.amode == 1 && g.bmode == 0) return launch_tma_shape<BN, 1, 0>(g, ta, tb, nb, st);
    if constexpr (BN % 64 == 0) {
        if (g.amode == 0) return launch_tma_shape<BN, 0, 1>(g, ta, tb, nb, st);
        return launch_tma_shape<BN, 1, 1>(g, ta, tb, nb, st);
    }
    return -1;
}

template <int BN>
int launch_tc(const GemmArgs &g, long long nb, cudaStream_t st)
{
    const sfg_gemm_desc &d = g.d;
    const int smem = TSTG * (128 + BN) * TBK * 2;
    if (cudaFuncSetAttribute(gemm_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return 2;
    dim3 grid((d.N + BN - 1) / BN, (d.M + 127) / 128, (unsigned)nb);
    if (grid.y > 65535) return 1;
    gemm_tc_kernel<BN><<<grid, 256, smem, st>>>(g);
    return launched();
}

extern "C" {

int sfg_fno_tc_timeouts(int *count, int reset)
{
    if (!count) return 1;
    if (cudaMemcpyFromSymbol(count, g_tc_timeouts, sizeof(int)) != cudaSuccess) return 2;
    if (reset) {
        const int zero = 0;
        if (cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof(int)) != cudaSuccess) return 2;
    }
    return 0;
}

int sfg_fno_gemm(const sfg_gemm_desc *dp, void *stream)
{
    if (!dp) return 1;
    const sfg_gemm_desc &d = *dp;
    if (!d.A || !d.B || !d.C || d.M <= 0 || d.N <= 0 || d.K <= 0 || d.batch1 <= 0 || d.batch2 <= 0 ||
        d.splits <= 0)
        return 1;
    if ((d.splits > 1 || d.atomic) && (d.c_bf16 || d.Cin || d.bias || d.gelu || d.pre)) return 1;
    if (d.splits > 1 && !d.atomic) return 1;
    const long long nb = (long long)d.batch1 * d.batch2 * d.splits;
    if (nb > 65535) return 1;
    GemmArgs g;
    g.d = d;
    g.tz1a = g.tz2a = g.tz1b = g.tz2b = 0;
    g.w2 = g.b2 = nullptr;
    g.y = nullptr;
    g.ys1 = g.ysj = 0;
    g.n2 = 0;
    g.amode = pick_mode(d.sam, d.sak, d.sa1, d.sa2, d.A);
    g.bmode = pick_mode(d.sbn, d.sbk, d.sb1, d.sb2, d.B);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool tc = d.engine == 2 || d.engine == 3 || d.engine == 4 || (d.engine == 0 && tc_auto(d));
    if (tc && d.N >= 32 && g.amode != 2 && g.bmode != 2) {   // copies move 16-byte groups
        if (d.engine != 3) {   // TMA operand tiles where the operands allow them
            // persistent CTAs where the main loop dominates (at least 8 k-tiles
            // per output tile); where a tile has only a few k-tiles, one tile
            // per CTA with the 256-thread staged epilogue is faster (measured:
            // head GEMM, K = 64, 161 vs 205 us; 8192^2 x 1024, 202 vs 187 us)
            const int kt = (d.K + TBK - 1) / TBK, per = (kt + d.splits - 1) / d.splits;
            const bool pers = d.engine == 2 || (d.engine == 0 && per >= 8);
            const int r = d.N >= 128 ? launch_tma<128>(g, nb, st, pers)
                          : d.N >= 64 ? launch_tma<64>(g, nb, st, pers)
                                      : launch_tma<32>(g, nb, st, pers);
            if (r >= 0) return r;
        }
        if (d.N >= 128) return launch_tc<128>(g, nb, st);
        if (d.N >= 64) return launch_tc<64>(g, nb, st);
        return launch_tc<32>(g, nb, st);
    }
    if (d.M >= 128 && d.N >= 128) {
        dim3 grid((d.N + 127) / 128, (d.M + 127) / 128, (unsigned)nb);
        if (grid.y > 65535) return 1;
        gemm_bf16_kernel<128, 128, 2, 4><<<grid, 256, 0, st>>>(g);
    } else if (d.M >= d.N) {
        dim3 grid((d.N + 63) / 64, (d.M + 127) / 128, (unsigned)nb);
        if (grid.y > 65535) return 1;
        gemm_bf16_kernel<128, 64, 4, 2><<<grid, 256, 0, st>>>(g);
    } else {
        dim3 grid((d.N + 127) / 128, (d.M + 63) / 64, (unsigned)nb);
        if (grid.y > 65535) return 1;
        gemm_bf16_kernel<64, 128, 2, 4><<<grid, 256, 0, st>>>(g);
    }
    return launched();
}

int sfg_fno_head_infer(const sfg_gemm_desc *dp, const float *w2, const float *b2, float *y, long long y_batch,
                       long long y_ch, int n2, void *stream)
{
    if (!dp || !w2 || !y || n2 < 1 || n2 > 4) return 1;
    const sfg_gemm_desc &d = *dp;
    if (!d.A || !d.B || d.M <= 0 || d.N <= 0 || d.N > 128 || d.K <= 0 || d.batch1 <= 0 || d.batch1 > 65535 ||
        d.batch2 != 1 || d.splits != 1 || d.atomic || d.Cin || d.pre || d.bias_on_m)
        return 1;
    GemmArgs g;
    g.d = d;
    g.tz1a = g.tz2a = g.tz1b = g.tz2b = 0;
    g.amode = pick_mode(d.sam, d.sak, d.sa1, d.sa2, d.A);
    g.bmode = pick_mode(d.sbn, d.sbk, d.sb1, d.sb2, d.B);
    g.w2 = w2; g.b2 = b2; g.y = y; g.ys1 = y_batch; g.ysj = y_ch; g.n2 = n2;
    if (g.amode != 1 || g.bmode != 1) return 3;   // the one layout the surrogate's head has
    CUtensorMap ta, tb;
    if (!operand_map(&ta, d.A, 1, d.M, d.K, d.sam, d.sak, d.sa1, d.sa2, d.batch1, 1, 128, g.tz1a, g.tz2a) ||
        !operand_map(&tb, d.B, 1, d.N, d.K, d.sbn, d.sbk, d.sb1, d.sb2, d.batch1, 1, 128, g.tz1b, g.tz2b))
        return 3;
    return launch_tma_shape<128, 1, 1, true>(g, ta, tb, d.batch1, static_cast<cudaStream_t>(stream));
}

int sfg_fno_dft_combine(const float *P, void *Zmix, int B, int C, void *stream)
{
    if (!P || !Zmix || B <= 0 || C <= 0) return 1;
    const long long n = (long long)B * C * KD * KC;
    const bool aligned = (reinterpret_cast<uintptr_t>(Zmix) & 15) == 0;
    if (C % CMB_C == 0 && aligned && B <= 65535) {
        dft_combine_tiled<<<dim3(KD * KC / CMB_M, C / CMB_C, B), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            P, static_cast<__nv_bfloat16 *>(Zmix), B, C);
        return launched();
    }
    dft_combine_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        P, static_cast<__nv_bfloat16 *>(Zmix), B, C);
    return launched();
}

int sfg_fno_dft_combine_bwd(const void *dZmix, void *dP, int B, int C, void *stream)
{
    if (!dZmix || !dP || B <= 0 || C <= 0) return 1;
    const long long n = (long long)B * C * KD * KC;
    const bool aligned = (reinterpret_cast<uintptr_t>(dZmix) & 15) == 0;
    if (C % CMB_C == 0 && aligned && B <= 65535) {
        dft_combine_bwd_tiled<<<dim3(KD * KC / CMB_M, C / CMB_C, B), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const __nv_bfloat16 *>(dZmix), static_cast<__nv_bfloat16 *>(dP), B, C);
        return launched();
    }
    dft_combine_bwd_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(dZmix), static_cast<__nv_bfloat16 *>(dP), B, C);
    return launched();
}

int sfg_fno_expand_weights(const float *Wr, const float *Wi, void *Wblk, int modes, int C, void *stream)
{
    if (!Wr || !Wi || !Wblk || modes <= 0 || C <= 0) return 1;
    const long long n = (long long)modes * C * C;
    expand_weights_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        Wr, Wi, static_cast<__nv_bfloat16 *>(Wblk), modes, C);
    return launched();
}

int sfg_fno_fold_weights(const float *dWblk, float *dWr, float *dWi, int modes, int C, void *stream)
{
    if (!dWblk || !dWr || !dWi || modes <= 0 || C <= 0) return 1;
    const long long n = (long long)modes * C * C;
    fold_weights_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(dWblk, dWr, dWi, modes, C);
    return launched();
}

int sfg_fno_gelu_bwd(const void *dy, int dy_bf16, const void *pre, void *dx, long long n, void *stream)
{
    if (!dy || !pre || !dx || n < 0) return 1;
    if (n) gelu_bwd_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        dy, dy_bf16, static_cast<const __nv_bfloat16 *>(pre), static_cast<__nv_bfloat16 *>(dx), n);
    return launched();
}

int sfg_fno_cast_bf16(const float *x, void *y, long long n, void *stream)
{
    if (!x || !y || n < 0) return 1;
    if (n) cast_bf16_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, static_cast<__nv_bfloat16 *>(y), n);
    return launched();
}

int sfg_fno_bias_grad(const void *dy, float *db, int outer, int C, long long inner, void *stream)
{
    if (!dy || !db || outer <= 0 || C <= 0 || C > 65535 || inner <= 0) return 1;
    const dim3 grid((unsigned)C, (unsigned)std::min(outer, 64));
    bias_grad_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16 *>(dy), db,
                                                                           outer, C, inner);
    return launched();
}

int sfg_fno_swap01(const void *x, void *y, int n0, int n1, long long n2, void *stream)
{
    if (!x || !y || n0 <= 0 || n1 <= 0 || n2 <= 0) return 1;
    const long long n = (long long)n0 * n1 * n2;
    swap01_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16 *>(x), static_cast<__nv_bfloat16 *>(y), n0, n1, n2);
    return launched();
}

int sfg_fno_zero(float *p, long long n, void *stream)
{
    if (!p || n < 0) return 1;
    if (n) zero_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, n);
    return launched();
}

int sfg_fno_scale(float *p, long long n, float a, void *stream)
{
    if (!p || n < 0) return 1;
    if (n) scale_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, n, a);
    return launched();
}

int sfg_fno_rel_loss(const float *pred, const void *target, float *loss, void *dpred, float *scratch, int B,
                     long long n, void *stream)
{
    if (!pred || !target || !scratch || B <= 0 || B > 65535 || n <= 0) return 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(scratch, 0, sizeof(float) * 2 * B, st) != cudaSuccess) return 2;
    const unsigned gx = (unsigned)std::min<long long>(grid_of(n, 256), 256);
    rel_loss_sums<<<dim3(gx, B), 256, 0, st>>>(pred, static_cast<const __nv_bfloat16 *>(target), scratch, n);
    rel_loss_grad<<<dim3(gx, B), 256, 0, st>>>(pred, static_cast<const __nv_bfloat16 *>(target), scratch, loss,
                                              static_cast<__nv_bfloat16 *>(dpred), B, n);
    return launched();
}

int sfg_fno_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float beta1, float beta2,
                 float eps, int step, void *stream)
{
    if (!p || !g || !m || !v || n < 0 || step < 1) return 1;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    if (n) adam_kernel<<<grid_of(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, g, m, v, n, lr, beta1,
                                                                                       beta2, eps, c1, c2);
    return launched();
}

}  // extern "C"
