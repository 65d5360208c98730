/*
 * stfwi_nn.h -- C ABI of the learned preconditioner's network kernels
 * (libstfwi.so, sm_100a).
 *
 * The reference has no counterpart: its inversion is plain
 * illumination-preconditioned L-BFGS (fwi/optim_lbfgsb.py:137-473,
 * preconditioner fwi/illumination.py:18-48 and fwi/preconditioning.py:65-139).
 * These entry points run a U-Net that maps [gradient, illumination, Vp, Vs]
 * to a Vs update direction, with BF16 operands and FP32 accumulation on the
 * tcgen05 tensor cores; the inversion driver keeps plain L-BFGS as its
 * fallback and accepts a learned step only if it lowers the misfit.
 *
 * Conventions: activations are BF16 NHWC ([n][h][w][c], c contiguous);
 * 3x3 weights are BF16 [9][cout][cin] with tap = 3*(dy+1) + (dx+1)
 * (output pixel p reads input pixel p + (dy, dx)); convolutions are
 * stride 1 with zero padding 1; channel counts are multiples of 16. All
 * tensor pointers are device memory, 16-byte aligned (scale4 of
 * stfwi_nn_pack_input is host memory); every call is asynchronous
 * on `stream` (a cudaStream_t, NULL = default stream). Status codes are
 * those of stfwi.h; stfwi_nn_last_error() gives the message of the last
 * failing call of this thread. stfwi_nn_check() synchronises the stream and
 * reports a tensor-core pipeline wait that gave up.
 */
#ifndef STFWI_NN_H
#define STFWI_NN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char *stfwi_nn_last_error(void);
int stfwi_nn_check(void *stream);

/* y[.., y_coff + co] (channel stride y_cstride) = act(b[co] + sum_{tap,ci} x[p + tap][ci] w[tap][co][ci]),
   act = ReLU when relu != 0.  The height and width must tile into 128-pixel boxes
   (w a multiple of 128, or w in {16, 32, 64} with h a multiple of 128 / w). */
int stfwi_nn_conv3x3(const void *x, int n, int h, int w, int cin, const void *wt, int cout, const float *bias,
                     int relu, void *y, int y_cstride, int y_coff, void *stream);

/* input gradient: dx[p][ci] = [mask[p][m_coff + ci] > 0] * sum_{tap,co} dz[p - tap][co] w[tap][co][ci],
   with wt_t = the weights packed as [8 - tap][ci][co] (stfwi_nn_pack_weights); mask may be NULL. */
int stfwi_nn_conv3x3_dgrad(const void *dz, int n, int h, int w, int cout, const void *wt_t, int cin,
                           const void *mask, int m_cstride, int m_coff, void *dx, void *stream);

/* weight gradient: dw[tap][co][ci] += sum_p dz[p][co] x[p + tap][ci] (FP32; w a multiple of 64) */
int stfwi_nn_conv3x3_wgrad(const void *x, const void *dz, int n, int h, int w, int cin, int cout, float *dw,
                           void *stream);

/* features [n][4][hd][wd] FP32 times scale4[c] (4 floats, host) -> x [n][h][w][16] BF16, zero outside
   hd x wd and in channels 4-15 */
int stfwi_nn_pack_input(const float *feat, int n, int hd, int wd, int h, int w, const float *scale4, void *x,
                        void *stream);

/* 2x2 average pool of channels [in_coff, in_coff + c) of in [n][h][w][in_cstride] -> out [n][h/2][w/2][c] */
int stfwi_nn_avgpool2(const void *in, int n, int h, int w, int c, int in_cstride, int in_coff, void *out,
                      void *stream);

/* gradient into a ReLU output y kept in a concatenation slice (channel stride cstride, offset coff) that
   also feeds a 2x2 average pool: dz = (dcat[slice] + dpool[parent] / 4) * [y > 0]; dcat may be NULL */
int stfwi_nn_skip_grad(const void *dcat, const void *ycat, int cstride, int coff, const void *dpool, int n, int h,
                       int w, int c, void *dz, void *stream);

/* nearest 2x upsampling of low [n][h][w][c] into channels [0, c) of out [n][2h][2w][out_cstride] */
int stfwi_nn_upsample2(const void *low, int n, int h, int w, int c, int out_cstride, void *out, void *stream);

/* dz[n][h][w][c] = [low > 0] * sum over the 2x2 children of dcat[.., 0:c] (channel stride cstride) */
int stfwi_nn_upsample2_grad(const void *dcat, int cstride, const void *low, int n, int h, int w, int c, void *dz,
                            void *stream);

/* 1x1 output head: out[p] = b + sum_c wt[c] y[p][c] (FP32 out, c a multiple of 16, <= 64) */
int stfwi_nn_head(const void *y, size_t npix, int c, const float *wt, const float *b, float *out, void *stream);

/* loss += sum_p wgt[p] (out[p] - target[p])^2 * inv_norm (FP64); dz = dloss/dy masked by [y > 0] (BF16);
   dwt[c], db += their gradients (FP32) */
int stfwi_nn_head_loss_grad(const void *y, size_t npix, int c, const float *wt, const float *out,
                            const float *target, const float *wgt, float inv_norm, void *dz, float *dwt, float *db,
                            double *loss, void *stream);

/* db[c] += sum_p dz[p][c] (c <= 1024) */
int stfwi_nn_bias_grad(const void *dz, size_t npix, int c, float *db, void *stream);

/* FP32 master weights [9][cout][cin] -> BF16 wf (same layout) and wt ([8 - tap][cin][cout]; may be NULL) */
int stfwi_nn_pack_weights(const float *w32, int cout, int cin, void *wf, void *wt, void *stream);

/* Adam in the efficient form of Kingma and Ba: m, v moments; p -= lr_t m / (sqrt(v) + eps) with lr_t the
   bias-corrected rate; g is scaled by grad_scale on read and cleared */
int stfwi_nn_adam(float *p, float *g, float *m, float *v, size_t n, float lr_t, float b1, float b2, float eps,
                  float grad_scale, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* STFWI_NN_H */
