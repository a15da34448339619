/*
 * seisfem_fno.h -- C ABI of the learned surrogate's kernels in
 * libseisfem_b200.so.  No counterpart in the reference: a Fourier neural
 * operator maps a velocity model plus a source position to the receiver
 * gather, trained on shots this library's FEM computes; the FEM stays its
 * fallback and the judge of its error.
 *
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Calls are asynchronous and return SFG_OK (0) or an
 * SFG_ERR_* code of seisfem_b200.h (SFG_ERR_ARG for bad shapes, SFG_ERR_CUDA
 * for a launch error).  BF16 is `__nv_bfloat16` (2 bytes).
 */
#ifndef SEISFEM_FNO_H
#define SEISFEM_FNO_H

#ifdef __cplusplus
extern "C" {
#endif

/* C[z][m][n] = alpha * sum_k A[z][m][k] * B[z][k][n] (+ beta * Cin) (+ bias)
 * then optionally GELU; z = z1 * batch2 + z2 runs over batch1 x batch2
 * problems (element strides per level).  A and B are BF16, the tensor cores
 * accumulate in FP32.  Epilogue order: v = alpha*acc; v += beta*Cin[c];
 * v += bias[n] (bias_on_m: bias[m]); pre[c] = v (BF16, if pre); v = gelu(v)
 * (if gelu); C[c] = v (FP32 or BF16).  atomic != 0 adds alpha*acc to an FP32
 * C with atomics instead (no Cin/bias/gelu/pre): for split-K (splits > 1) and
 * for summing the batch into one output (C strides 0 over the batch). */
typedef struct {
    const void *A, *B;
    void *C;
    const float *Cin;
    void *pre;
    const float *bias;
    long long sa1, sa2, sam, sak;  /* A: batch level 1, batch level 2, m, k */
    long long sb1, sb2, sbk, sbn;  /* B */
    long long sc1, sc2, scm, scn;  /* C (Cin and pre use the same strides) */
    int M, N, K, batch1, batch2, splits;
    float alpha, beta;
    int c_bf16, gelu, bias_on_m, atomic;
    int engine;                    /* 0: automatic, 1: mma.sync tiles, 2: tcgen05 with TMEM accumulators,
                                      persistent CTAs (TMA operand tiles where the strides allow, else
                                      cp.async), 3: tcgen05 with cp.async operand tiles, 4: tcgen05 with
                                      TMA tiles, one output tile per CTA.  Automatic: tcgen05 for
                                      M >= 64, N >= 32, K >= 64, persistent from 8 k-tiles per tile */
} sfg_gemm_desc;

int sfg_fno_gemm(const sfg_gemm_desc *d, void *stream);
/* waits of the tcgen05 GEMM that gave up (bounded mbarrier waits) since the
 * last reset; a non-zero count means some outputs were not written */
int sfg_fno_tc_timeouts(int *count, int reset);

/* forward DFT recombination: P[z][64][32] (FP32; rows 0-31 cos, 32-63 sin
 * times [Yre | Yim]) -> Zmix[mode = k1*16+k2][b][ri][c] (BF16), z = b*C + c */
int sfg_fno_dft_combine(const float *P, void *Zmix, int B, int C, void *stream);
/* its adjoint: dZmix (BF16) -> dP[z][64][32] (BF16) */
int sfg_fno_dft_combine_bwd(const void *dZmix, void *dP, int B, int C, void *stream);
/* mixing weights (FP32 Wr, Wi [mode][C][C]) -> BF16 blocks [mode][2C][2C] =
 * [[Wr, Wi], [-Wi, Wr]] */
int sfg_fno_expand_weights(const float *Wr, const float *Wi, void *Wblk, int modes, int C, void *stream);
/* gradient of the blocks (FP32 [mode][2C][2C]) folded back onto Wr, Wi (added) */
int sfg_fno_fold_weights(const float *dWblk, float *dWr, float *dWi, int modes, int C, void *stream);
/* dx = dy * gelu'(pre) (dy FP32 or BF16, pre BF16, dx BF16) */
int sfg_fno_gelu_bwd(const void *dy, int dy_bf16, const void *pre, void *dx, long long n, void *stream);
/* The surrogate's head for inference in one kernel: y[b][j][m] = b2[j] +
 * sum_n GELU(alpha (A B)[b][m][n] + bias[n]) w2[n][j] for j < n2, with the
 * first GEMM given by *d (A and B contiguous along M and N, N <= 128, one
 * batch level, d->C unused) and y at y + b * y_batch + j * y_ch + m; the
 * hidden activations never reach memory.  Returns 1 for a bad argument, 3
 * when the operands' layout does not fit (the caller then runs the two
 * GEMMs). */
int sfg_fno_head_infer(const sfg_gemm_desc *d, const float *w2, const float *b2, float *y, long long y_batch,
                       long long y_ch, int n2, void *stream);
/* FP32 -> BF16 */
int sfg_fno_cast_bf16(const float *x, void *y, long long n, void *stream);
/* bias gradient of a [outer][C][inner] tensor (BF16): db[c] += sum over outer, inner */
int sfg_fno_bias_grad(const void *dy, float *db, int outer, int C, long long inner, void *stream);
/* y[j][i][k] = x[i][j][k] for x[n0][n1][n2] (BF16) */
int sfg_fno_swap01(const void *x, void *y, int n0, int n1, long long n2, void *stream);
/* p[0..n) = 0 (FP32) */
int sfg_fno_zero(float *p, long long n, void *stream);
/* p[0..n) *= a (FP32): the 1/ranks of gradients summed over data-parallel ranks */
int sfg_fno_scale(float *p, long long n, float a, void *stream);
/* relative-L2 loss of a batch: pred (FP32) vs target (BF16), [B][n] each;
 * loss[b] = |pred-target|^2 / |target|^2 and dpred = 2 (pred-target) /
 * (B |target|^2) (BF16); scratch: 2*B floats */
int sfg_fno_rel_loss(const float *pred, const void *target, float *loss, void *dpred, float *scratch, int B,
                     long long n, void *stream);
/* Adam (decoupled weight decay 0): p -= lr * mhat / (sqrt(vhat) + eps) */
int sfg_fno_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float beta1, float beta2,
                 float eps, int step, void *stream);

#ifdef __cplusplus
}
#endif
#endif
