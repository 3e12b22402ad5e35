/*
 * fvnet.h -- C-ABI of the learned coarse-grid correction (BF16 tensor-core convolutions on sm_100a,
 * FP64 conservative projection, AdamW).
 *
 * The reference has no such component: its learned models are JAX/Equinox surrogates that replace
 * the solver (surrogate/models.py), and a coarse solver + learned correction is listed as future work
 * (README.md:20).  The pieces follow the reference's semantics where they exist:
 *   PeriodicConv (surrogate/models.py:16-29): wrap-pad by k//2, VALID cross-correlation, weight
 *     (c_out, c_in, k, k) + bias;  GELU = jax.nn.gelu default (tanh approximation, models.py:43-44);
 *   zero-initialised last layer (models.py:67-69);
 *   loss = MSE in normalised units (train.py:74-75), pushforward unroll (train.py:107-111);
 *   optimiser = clip_by_global_norm(1.0) + adamw(weight_decay=1e-4) (train.py:209-211).
 *
 * Conventions: all pointers are DEVICE pointers; work is queued on `stream` (a cudaStream_t, or
 * NULL); nothing here allocates.  Activations are NHWC BF16 with channels padded to 16 or 32.
 * Status codes are those of fv.h (0 = OK); fv_last_error() gives the message.  `err` arguments
 * point to a device int set to 1 if a bounded device-side wait gave up (the kernel then returns
 * without writing its outputs).
 */
#ifndef FVNET_H
#define FVNET_H

#ifdef __cplusplus
extern "C" {
#endif

#define FVNET_OK 0
#define FVNET_ERR_ARG 1
#define FVNET_ERR_CUDA 2

/* convolution modes */
#define FVNET_CONV_HIDDEN 0    /* Z = conv(X) + bias; A = gelu(Z)           (hidden layers) */
#define FVNET_CONV_OUTPUT 1    /* out4 = conv(X)[:, :4] + bias[:4] in FP32  (projection layer) */
#define FVNET_CONV_BWD_GELU 2  /* A = conv_T(X) * gelu'(Zprev)              (backward data through a hidden layer) */
#define FVNET_CONV_BWD_PLAIN 3 /* A = conv_T(X)                              (backward data, no activation) */

/* Periodic 3x3 convolution on the tensor cores.  X: [B][H][W][cin_pad] BF16; Wpacked: weights packed
 * by fvnet_pack_weights (forward pack for the forward modes, backward pack for the backward modes,
 * where cin_pad/cout_pad are the backward conv's: the layer's cout_pad/cin_pad).  W in {32, 64, 128,
 * 256}, H a multiple of 256/W.  Supported (cin_pad, cout_pad): HIDDEN (16,32),(32,32); OUTPUT (32,16);
 * BWD_GELU (16,32),(32,32); BWD_PLAIN (16,32),(32,32),(32,16). */
int fvnet_conv3x3(int mode, int cin_pad, int cout_pad, int B, int H, int W, const void* X, const void* Wpacked,
                  const float* bias, const void* Zprev, void* Z, void* A, float* out4, int* err, void* stream);

/* Weight and bias gradients of a layer (cin -> cout, padded cin_pad -> cout_pad) from its input X
 * [B][H][W][cin_pad] and output gradient dZ [B][H][W][cout_pad], both BF16, on the tensor cores
 * (per x-shift: M = 3*cin rows (ky, ci), N = cout, K = pixels).  dW: [cout][cin][3][3] FP32, db: [cout]
 * FP32.  Workspace: partial >= fvnet_wgrad_parts(B, H) * 9 * cin_pad * cout_pad floats,
 * db_part >= fvnet_wgrad_parts(B, H) * cout_pad floats.
 * W in {32, 64, 128}. */
int fvnet_conv3x3_wgrad(int cin_pad, int cout_pad, int cin, int cout, int B, int H, int W, const void* X, const void* dZ,
                        float* partial, float* dW, float* db, float* db_part, int* err, void* stream);
int fvnet_wgrad_parts(int B, int H);

/* Canonical FP32 weights [cout][cin][3][3] -> BF16 forward pack [9][cin_pad/8][cout_pad][8] and
 * backward-data pack [9][cout_pad/8][cin_pad][8] (transposed, spatially flipped); each 9*cin_pad*cout_pad. */
int fvnet_pack_weights(int cout, int cin, int cout_pad, int cin_pad, const float* W, void* Wfwd, void* Wbwd,
                       void* stream);

/* Network input: X16[p][c] = bf16((U[p][c] - stats[c]) * stats[4+c]) for the 4 conserved fields of
 * the FP64 state U [npix][4], channels 4..15 zero.  stats = {mean[4], 1/std[4]} (FP64). */
int fvnet_prep_input(const double* U, long long npix, const double* stats, void* X16, void* stream);

/* The correction step, FP64: per sample b (npix cells each), D = out4 * dscale * w with the coarse
 * cell's weights w = (rho, rho, rho, E) (corrections relative to the cell, so that rarefied cells get
 * proportionally small ones), D -= mean(D) per field (zero-mean projection: the totals of mass,
 * momentum and energy are unchanged), then
 *   FVNET_CORR_STRICT: Unext = Uc + D; a sample with any cell !(rho > 0) || !(p > 0) falls back to the
 *                      plain coarse step Unext = Uc (theta 0);
 *   FVNET_CORR_KEEP:   Unext = Uc + D always (the trained step of a training iteration: the loss then
 *                      sees an unphysical correction instead of ignoring it); fallback flags it;
 *   FVNET_CORR_SCALE:  Unext = Uc + theta D with the largest theta in [0,1] keeping every cell's rho
 *                      and p above a tenth of their coarse values (theta = 0 is the plain coarse step);
 *                      theta is uniform over the sample, so theta D is still zero-mean.  With
 *                      max_speed_ratio > 0 theta is then halved (up to 6 times, else 0) until the
 *                      sample's signal speed max(|u| + a) + max(|v| + a) is at most max_speed_ratio
 *                      times that of Uc: the next coarse step's CFL dt shrinks at most by that factor.
 * max_speed_ratio: <= 0 (no bound) or >= 1; used by FVNET_CORR_SCALE only.
 * fallback[b] = 1 when sample b did not receive its full correction; theta (may be NULL) receives
 * the fraction applied. */
#define FVNET_CORR_STRICT 0
#define FVNET_CORR_KEEP 1
#define FVNET_CORR_SCALE 2
int fvnet_apply_correction(const double* Uc, const float* out4, int B, int npix, const double* dscale, double* Unext,
                           int* fallback, double* theta, int mode, double max_speed_ratio, void* stream);

/* Loss and gradient: loss_part[b] = sum over the sample of ((Unext - Y) / std)^2 (the loss is the
 * sum of loss_part over b divided by B*npix*4); dout16 [B][npix][16] BF16 = d loss / d out4 through
 * the projection, the fraction theta[b] applied (held constant; NULL = 1) and the scaling by dscale
 * and the weights of the coarse state Uc (channels 4..15 zero). */
int fvnet_loss_grad(const double* Unext, const double* Y, const double* Uc, int B, int npix, const double* stats,
                    const double* dscale, const double* theta, double* loss_part, void* dout16, void* stream);

/* One AdamW step on n FP32 parameters with clipping of the gradient by its global norm (max_norm);
 * step is 1-based (bias correction).  norm_part: fvnet_norm_partials() doubles of workspace;
 * norm_out (may be NULL) receives the gradient norm before clipping. */
int fvnet_adamw(float* params, const float* grads, float* m, float* v, long long n, double* norm_part, float lr, float b1,
                float b2, float eps, float weight_decay, float max_norm, int step, double* norm_out, void* stream);
int fvnet_norm_partials(void);

#ifdef __cplusplus
}
#endif

#endif /* FVNET_H */
