/*
 * sasb200_mlp.h -- C-ABI of libsasb200_mlp.so (the learned I(q) surrogate)
 * and of libsasb200_peaks.so (the pipe-throughput probes used as roofline
 * denominators).
 *
 * No counterpart in the reference: sasmodels has no learned surrogate and
 * no throughput probes.  The network is 16 (7 used) -> 4 x 256 SiLU -> 1
 * with BF16 operands, compensated (hi + lo) BF16 activations and FP32
 * accumulation in tensor memory (tcgen05).  All pointers are device
 * pointers; bf16 tensors are passed as void*.  Every function returns 0 on
 * success, -1 for a bad argument, -3 for a CUDA launch error;
 * sasb200_mlp_last_error() describes the last failure on the calling host
 * thread.  Kernels with pipeline waits write a nonzero value to *err when a
 * bounded wait runs out (the kernel then unwinds instead of hanging).
 * n_pad is n rounded up to a multiple of 128 (one tile of rows).
 */
#ifndef SASB200_MLP_H
#define SASB200_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char *sasb200_mlp_last_error(void);

/* features: the compensated BF16 pair x + x_lo [n_pad x 16] from float64
 * per-point inputs (radius, length, radius pd, length pd, contrast, q,
 * orientation flag); rows >= n are zero. */
int32_t sasb200_mlp_features(int32_t n, int32_t n_pad, const double *radius,
                             const double *length, const double *rpd, const double *lpd,
                             const double *drho, const double *q, const double *flag,
                             void *x, void *x_lo, void *stream);

/* pipelined forward: the weights packed once by sasb200_mlp_pack into an
 * image of sasb200_mlp_image_bytes() bytes (16-byte aligned); out[n], and
 * for training the z/h planes [4][n_pad x 256] bf16 (both NULL for
 * inference); persistent grid of at most `blocks` CTAs (0 = one per SM). */
int32_t sasb200_mlp_image_bytes(void);
int32_t sasb200_mlp_pack(const void *w0, const void *w1, const void *w2, const void *w3,
                         void *img, void *stream);
int32_t sasb200_mlp_infer(int32_t n, int32_t n_pad, const void *x, const void *x_lo,
                          const void *img, const float *const *b, const float *w_out,
                          const float *b_out, float *out, void *z_save, void *h_save,
                          int32_t *err, int32_t blocks, void *stream);

/* the same forward through the overlapped kernel (a dedicated MMA warp, two
 * TMEM accumulators, layer l+1's MMAs running under layer l's epilogue chunk
 * by chunk), same image and arguments.  Hidden activations and the z/h
 * planes bitwise those of sasb200_mlp_infer; out differs only by the order
 * of the output dot's sums.  Used for inference (planes NULL) and for the
 * training forward. */
int32_t sasb200_mlp_serve(int32_t n, int32_t n_pad, const void *x, const void *x_lo,
                          const void *img, const float *const *b, const float *w_out,
                          const float *b_out, float *out, void *z_save, void *h_save,
                          int32_t *err, int32_t blocks, void *stream);

/* pipelined backward (training): W3^T, W2^T, W1^T packed once per weight
 * update by sasb200_mlp_pack_t into sasb200_mlp_image_t_bytes() bytes; dZ
 * planes [4][n_pad x 256] bf16 from dout and the saved pre-activations. */
int32_t sasb200_mlp_image_t_bytes(void);
int32_t sasb200_mlp_pack_t(const void *wt1, const void *wt2, const void *wt3, void *img_t,
                           void *stream);
int32_t sasb200_mlp_backward_p(int32_t n, int32_t n_pad, const void *img_t, const float *w_out,
                               const float *dout, const void *z_save, void *dz_save,
                               int32_t *err, int32_t blocks, void *stream);

/* training: forward with saved pre-activations and activations
 * (z_save, h_save: [4][n_pad x 256] bf16 each, or both NULL), backward
 * through the hidden layers (wt: transposed bf16 weights), weight
 * gradients as split-K partial GEMMs C[splits][M x nb] = A[M x K] B[nb x K]^T,
 * Huber loss gradient, Adam (also refreshing the bf16
 * copies w and, if non-NULL, the transposed wt). */
int32_t sasb200_mlp_forward(int32_t n, int32_t n_pad, const void *x, const void *x_lo,
                            const void *const *w, const float *const *b, const float *w_out,
                            const float *b_out, float *out, void *z_save, void *h_save,
                            int32_t *err, void *stream);
int32_t sasb200_mlp_backward(int32_t n, int32_t n_pad, const void *const *wt,
                             const float *w_out, const float *dout, const void *z_save,
                             void *dz_save, int32_t *err, void *stream);
int32_t sasb200_gemm_nt(int32_t M, int32_t nb, int32_t K, int32_t lda, int32_t ldb,
                        const void *A, const void *B, int32_t splits, float *C, int32_t *err,
                        void *stream);
int32_t sasb200_transpose_bf16(int32_t rows, int32_t cols, const void *src, void *dst,
                               void *stream);
int32_t sasb200_loss_grad(int32_t n, int32_t n_pad, const float *out, const float *y,
                          float delta, float *dout, float *loss, void *stream);
int32_t sasb200_adam(int32_t size, int32_t splits, const float *grad, float *p, float *m,
                     float *v, float lr, float b1, float b2, float eps, int32_t step, void *w,
                     void *wt, int32_t rows, int32_t cols, void *stream);

/* the learning rate and Adam bias corrections of a training step, on the
 * device: counters = {schedule step s, Adam step count t} (int32), sched =
 * {lr, 1 - b1^t, 1 - b2^t} with lr = lr0 min(1, (s + 1)/warmup)
 * (1 + cos(pi s/total))/2, then s and t advance by one.  A CUDA graph of a
 * whole training step replays with these. */
int32_t sasb200_lr_schedule(int32_t *counters, float *sched, int32_t total, int32_t warmup,
                            float lr0, float b1, float b2, void *stream);

/* Adam for all n (<= 16) parameter tensors in one launch, lr and bias
 * corrections from sched (sasb200_lr_schedule): host arrays of n entries
 * (device pointers; w[k], wt[k] may be NULL), each tensor updated as by
 * sasb200_adam */
int32_t sasb200_adam_multi(int32_t n, const int32_t *sizes, const int32_t *splits,
                           const float *const *grads, float *const *p, float *const *m,
                           float *const *v, void *const *w, void *const *wt, const int32_t *rows,
                           const int32_t *cols, const float *sched, float b1, float b2, float eps,
                           void *stream);

/* out[c] = sum over r of M[r][c] (times v[r] when v is non-NULL) for a
 * row-major bf16 [rows x cols] matrix, in a fixed order: partial sums of
 * 64-row blocks into part (sasb200_col_sum_parts(rows) x cols floats), then
 * each column's partials combined in a fixed order (one warp per column). */
int32_t sasb200_col_sums(int32_t rows, int32_t cols, const void *M, const float *v, float *part,
                         float *out, void *stream);
int32_t sasb200_col_sum_parts(int32_t rows);

/* libsasb200_peaks.so: dependent-chain throughput probes (FP64 FMA, FP32
 * FMA, MUFU sine) whose measured rates are the roofline peaks of the
 * FP64 and FP32-compensated kernels. */
int32_t sasb200_probe_fp64_fma(double *out, int32_t blocks, int32_t iters, void *stream);
int32_t sasb200_probe_fp32_fma(float *out, int32_t blocks, int32_t iters, void *stream);
int32_t sasb200_probe_mufu_sin(float *out, int32_t blocks, int32_t iters, void *stream);
int32_t sasb200_probe_threads_per_block(void);
int32_t sasb200_probe_chains(void);

#ifdef __cplusplus
}
#endif

#endif /* SASB200_MLP_H */
