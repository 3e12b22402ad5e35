// Elementwise and reduction kernels of the learned correction (everything around the convolutions):
//  * input normalisation of the coarse FP64 state to the network's BF16 input,
//  * the FP64 correction step: de-normalise the network output, project each conserved field of each
//    sample to zero mean (so total mass, momentum and energy are unchanged to FP64 roundoff), add it
//    to the coarse state, and fall back to the plain coarse state when the result is non-physical,
//  * the loss (MSE in normalised units, surrogate/train.py:74-75) and its gradient through the
//    projection, and
//  * AdamW with clipping by global norm (surrogate/train.py:209-211: optax.clip_by_global_norm(1.0)
//    then optax.adamw(lr, weight_decay=1e-4), defaults b1 0.9, b2 0.999, eps 1e-8).
// Reductions use fixed-order trees (one CTA per sample, or per-block partials summed in order), so
// every result is deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "../../include/fvnet.h"
#include "fv_physics.cuh"

int fv_internal_set_error(int code, const char* msg);

namespace {

constexpr int RT = 256;  // threads of the per-sample reduction CTAs

__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = RT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// X16[p][c] = bf16((U[p][c] - mean[c]) * inv_std[c]) for c < 4, 0 for c = 4..15
__global__ void prep_input_kernel(const double* __restrict__ U, long long npix, const double* __restrict__ stats,
                                  __nv_bfloat16* __restrict__ X16) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        __nv_bfloat16 v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.0f);
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = __float2bfloat16_rn((float)((U[p * 4 + c] - stats[c]) * stats[4 + c]));
        uint4* dst = reinterpret_cast<uint4*>(X16 + p * 16);
        dst[0] = *reinterpret_cast<uint4*>(v);
        dst[1] = *reinterpret_cast<uint4*>(v + 8);
    }
}

__device__ __forceinline__ double block_min(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = RT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_max(double v, double* sh) { return -block_min(-v, sh); }

// The network predicts corrections relative to the coarse cell: the density and momentum corrections
// in units of the cell's density, the energy correction in units of its energy (the reference's
// Positive wrapper, models.py:254-306, works in log-primitive variables for the same reason: an
// absolute correction sized for dense, energetic regions breaks positivity in rarefied ones).
// raw correction of field c at cell p: out * dscale[c] * (rho, rho, rho, E)[c] of the coarse state.
__device__ __forceinline__ double corr_weight(const double* uc, int p, int c) { return uc[p * 4 + (c == 3 ? 3 : 0)]; }
__device__ __forceinline__ double raw_correction(const float* o, const double* uc, const double* dscale, int p, int c) {
    return (double)o[p * 4 + c] * dscale[c] * corr_weight(uc, p, c);
}

// Largest theta in [0, 1] with rho(theta) >= 0.1 rho and p(theta) >= 0.1 p for U(theta) = U + theta D,
// U physical.  rho is linear in theta; with k = 0.1 p / (gamma - 1), p(theta) >= 0.1 p <=> g(theta) =
// rho(theta) E(theta) - |m(theta)|^2 / 2 - k rho(theta) >= 0, a quadratic with g(0) = 0.9 rho p/(gamma-1)
// > 0, so the admissible thetas form an interval [0, first positive root).
__device__ __forceinline__ double admissible_theta(const double* u, const double* d) {
    const double rho = u[0], mx = u[1], my = u[2], E = u[3];
    const double dr = d[0], dmx = d[1], dmy = d[2], dE = d[3];
    double th = 1.0;
    if (dr < 0.0) th = fmin(th, 0.9 * rho / (-dr));
    const double p = fv::GM1 * (E - 0.5 * (mx * mx + my * my) / rho);
    const double k = 0.1 * p / fv::GM1;
    const double a = dr * dE - 0.5 * (dmx * dmx + dmy * dmy);
    const double b = rho * dE + E * dr - (mx * dmx + my * dmy) - k * dr;
    const double c = rho * E - 0.5 * (mx * mx + my * my) - k * rho;
    double root = 1e300;  // smallest positive root of a t^2 + b t + c
    if (a == 0.0) {
        if (b < 0.0) root = -c / b;
    } else {
        const double disc = b * b - 4.0 * a * c;
        if (disc >= 0.0) {
            const double q = -0.5 * (b + copysign(sqrt(disc), b));
            const double r1 = q / a, r2 = (q != 0.0) ? c / q : 1e300;
            if (r1 > 0.0) root = fmin(root, r1);
            if (r2 > 0.0) root = fmin(root, r2);
        }
    }
    return fmax(0.0, fmin(th, root));
}

// Signal speed of a sample's state Uc + theta D, as the CFL step sees it on square cells:
// max(|u| + a) + max(|v| + a) over the cells (solver2d.hpp:67-83 with dx = dy), a = sqrt(gamma p / rho);
// infinite if a cell is not physical.  Every thread of the CTA calls it and gets the result.
__device__ __forceinline__ double signal_speed(const double* uc, const float* o, const double* dscale,
                                               const double* mean, double theta, int npix, double* sh) {
    double sx = 0.0, sy = 0.0;
    for (int p = threadIdx.x; p < npix; p += RT) {
        fv::Q4 u{uc[p * 4 + 0] + theta * (raw_correction(o, uc, dscale, p, 0) - mean[0]),
                 uc[p * 4 + 1] + theta * (raw_correction(o, uc, dscale, p, 1) - mean[1]),
                 uc[p * 4 + 2] + theta * (raw_correction(o, uc, dscale, p, 2) - mean[2]),
                 uc[p * 4 + 3] + theta * (raw_correction(o, uc, dscale, p, 3) - mean[3])};
        const fv::Q4 w = fv::to_primitive(u);
        if (!(w.a > 0.0) || !(w.d > 0.0)) {
            sx = INFINITY;
            continue;
        }
        const double a = sqrt(fv::GAMMA * w.d / w.a);
        sx = fmax(sx, fabs(w.b) + a);
        sy = fmax(sy, fabs(w.c) + a);
    }
    sx = block_max(sx, sh);
    sy = block_max(sy, sh);
    return sx + sy;
}

// One CTA per sample.  D = out4 * dscale (FP64), D -= mean(D) per field (zero-mean projection), then
//   mode STRICT: Unext = Uc + D, or Uc if any cell of it has !(rho > 0) || !(p > 0)  (theta 1 or 0)
//   mode KEEP:   Unext = Uc + D always; theta = 1, fallback flags the non-physical samples
//   mode SCALE:  Unext = Uc + theta D with the largest theta in [0,1] keeping every cell's rho and p
//                above a tenth of their coarse values (theta = 0 is the plain coarse step); with
//                max_speed_ratio > 0, theta is then halved (up to 6 times, else 0) until the signal
//                speed of Uc + theta D is at most max_speed_ratio times that of Uc
// fallback[b] = 1 when the sample did not get its full correction (or, in KEEP mode, would not have).
__global__ void __launch_bounds__(RT) apply_correction_kernel(const double* __restrict__ Uc, const float* __restrict__ out4,
                                                              int npix, const double* __restrict__ dscale,
                                                              double* __restrict__ Unext, int* __restrict__ fallback,
                                                              double* __restrict__ theta_out, int mode,
                                                              double max_speed_ratio) {
    __shared__ double sh[RT];
    __shared__ int sbad;
    const int b = blockIdx.x;
    const double* uc = Uc + (size_t)b * npix * 4;
    const float* o = out4 + (size_t)b * npix * 4;
    double* un = Unext + (size_t)b * npix * 4;
    double mean[4];
    for (int c = 0; c < 4; ++c) {
        double s = 0.0;
        for (int p = threadIdx.x; p < npix; p += RT) s += raw_correction(o, uc, dscale, p, c);
        mean[c] = block_sum(s, sh) / npix;
    }
    double theta = 1.0;
    if (mode == FVNET_CORR_SCALE) {
        double tmin = 1.0;
        for (int p = threadIdx.x; p < npix; p += RT) {
            double d[4];
            for (int c = 0; c < 4; ++c) d[c] = raw_correction(o, uc, dscale, p, c) - mean[c];
            tmin = fmin(tmin, admissible_theta(uc + (size_t)p * 4, d));
        }
        theta = block_min(tmin, sh);
        if (max_speed_ratio > 0.0 && theta > 0.0) {
            // the coarse step's CFL dt must not shrink by more than the ratio: a correction that
            // raises the signal speed (a near-vacuum cell, a fast spurious jet) would make the next
            // coarse step take that many more sub-steps
            const double limit = max_speed_ratio * signal_speed(uc, o, dscale, mean, 0.0, npix, sh);
            double th = theta;
            int k = 0;
            for (; k <= 6 && signal_speed(uc, o, dscale, mean, th, npix, sh) > limit; ++k) th *= 0.5;
            theta = (k <= 6) ? th : 0.0;
        }
    }
    if (threadIdx.x == 0) sbad = 0;
    __syncthreads();
    int bad = 0;
    for (int p = threadIdx.x; p < npix; p += RT) {
        fv::Q4 u{uc[p * 4 + 0] + theta * (raw_correction(o, uc, dscale, p, 0) - mean[0]),
                 uc[p * 4 + 1] + theta * (raw_correction(o, uc, dscale, p, 1) - mean[1]),
                 uc[p * 4 + 2] + theta * (raw_correction(o, uc, dscale, p, 2) - mean[2]),
                 uc[p * 4 + 3] + theta * (raw_correction(o, uc, dscale, p, 3) - mean[3])};
        const fv::Q4 w = fv::to_primitive(u);
        if (!(w.a > 0.0) || !(w.d > 0.0)) bad = 1;
        un[p * 4 + 0] = u.a; un[p * 4 + 1] = u.b; un[p * 4 + 2] = u.c; un[p * 4 + 3] = u.d;
    }
    if (bad) atomicOr(&sbad, 1);
    __syncthreads();
    if (sbad && mode != FVNET_CORR_KEEP) {  // the plain coarse step
        for (int e = threadIdx.x; e < npix * 4; e += RT) un[e] = uc[e];
        theta = 0.0;
    }
    if (threadIdx.x == 0) {
        fallback[b] = (sbad || theta < 1.0) ? 1 : 0;
        if (theta_out) theta_out[b] = theta;
    }
}

// One CTA per sample.  r = (Unext - Y) * inv_std; loss_part[b] = sum r^2.  Gradient of
// L = sum_b loss_part[b] / (B * npix * 4) with respect to the network output through the projection:
// g = 2 r inv_std / N; g -= mean(g) per field (the projection is its own adjoint); dout = theta g
// dscale, where theta is the fraction of the correction the sample received (held constant: 0 for a
// sample that fell back to the coarse step).  dout is BF16 with 16 channels.
__global__ void __launch_bounds__(RT) loss_grad_kernel(const double* __restrict__ Unext, const double* __restrict__ Y,
                                                       const double* __restrict__ Uc, int npix,
                                                       const double* __restrict__ stats,
                                                       const double* __restrict__ dscale, const double* __restrict__ theta,
                                                       double inv_total, double* __restrict__ loss_part,
                                                       __nv_bfloat16* __restrict__ dout16) {
    __shared__ double sh[RT];
    const int b = blockIdx.x;
    const double* un = Unext + (size_t)b * npix * 4;
    const double* y = Y + (size_t)b * npix * 4;
    const double* uc = Uc + (size_t)b * npix * 4;
    __nv_bfloat16* d = dout16 + (size_t)b * npix * 16;
    double l = 0.0, gmean[4];
    for (int c = 0; c < 4; ++c) {
        double s = 0.0;
        for (int p = threadIdx.x; p < npix; p += RT) {
            const double r = (un[p * 4 + c] - y[p * 4 + c]) * stats[4 + c];
            l += r * r;
            s += 2.0 * r * stats[4 + c] * inv_total;
        }
        gmean[c] = block_sum(s, sh) / npix;
    }
    const double ltot = block_sum(l, sh);
    if (threadIdx.x == 0) loss_part[b] = ltot;
    const double th = theta ? theta[b] : 1.0;
    for (int p = threadIdx.x; p < npix; p += RT) {
        __nv_bfloat16 v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.0f);
        if (th != 0.0) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double r = (un[p * 4 + c] - y[p * 4 + c]) * stats[4 + c];
                const double g = 2.0 * r * stats[4 + c] * inv_total - gmean[c];
                v[c] = __float2bfloat16_rn((float)(th * g * dscale[c] * corr_weight(uc, p, c)));
            }
        }
        uint4* dst = reinterpret_cast<uint4*>(d + (size_t)p * 16);
        dst[0] = *reinterpret_cast<uint4*>(v);
        dst[1] = *reinterpret_cast<uint4*>(v + 8);
    }
}

constexpr int AT = 256, AB = 120;  // AdamW: threads, blocks (fixed so the norm is summed in a fixed order)

__global__ void __launch_bounds__(AT) sq_partial_kernel(const float* __restrict__ g, long long n, double* __restrict__ part) {
    __shared__ double sh[AT];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)AT + threadIdx.x; i < n; i += (long long)AB * AT) s += (double)g[i] * g[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = AT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(AT) adamw_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                                   float* __restrict__ v, long long n, const double* __restrict__ part,
                                                   float lr, float b1, float b2, float eps, float wd, float max_norm,
                                                   int step, double* __restrict__ norm_out) {
    double ss = 0.0;
    for (int k = 0; k < AB; ++k) ss += part[k];
    const double norm = sqrt(ss);
    if (blockIdx.x == 0 && threadIdx.x == 0 && norm_out) *norm_out = norm;
    const float scale = (float)(norm > max_norm ? max_norm / norm : 1.0);  // clip_by_global_norm
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    for (long long i = blockIdx.x * (long long)AT + threadIdx.x; i < n; i += (long long)gridDim.x * AT) {
        const float gi = g[i] * scale;
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float upd = (mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i];
        p[i] -= lr * upd;
    }
}

}  // namespace

extern "C" {

int fvnet_prep_input(const double* U, long long npix, const double* stats, void* X16, void* stream) {
    if (!U || !stats || !X16 || npix <= 0) return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_prep_input: bad arguments");
    const int blocks = (int)std::min<long long>((npix + 255) / 256, 148 * 16);
    prep_input_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(U, npix, stats,
                                                                             static_cast<__nv_bfloat16*>(X16));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FVNET_OK : fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
}

int fvnet_apply_correction(const double* Uc, const float* out4, int B, int npix, const double* dscale, double* Unext,
                           int* fallback, double* theta, int mode, double max_speed_ratio, void* stream) {
    if (!Uc || !out4 || !dscale || !Unext || !fallback || B <= 0 || npix <= 0 || mode < FVNET_CORR_STRICT ||
        mode > FVNET_CORR_SCALE || !(max_speed_ratio <= 0.0 || max_speed_ratio >= 1.0))
        return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_apply_correction: bad arguments");
    apply_correction_kernel<<<B, RT, 0, static_cast<cudaStream_t>(stream)>>>(Uc, out4, npix, dscale, Unext, fallback,
                                                                             theta, mode, max_speed_ratio);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FVNET_OK : fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
}

int fvnet_loss_grad(const double* Unext, const double* Y, const double* Uc, int B, int npix, const double* stats,
                    const double* dscale, const double* theta, double* loss_part, void* dout16, void* stream) {
    if (!Unext || !Y || !Uc || !stats || !dscale || !loss_part || !dout16 || B <= 0 || npix <= 0)
        return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_loss_grad: bad arguments");
    const double inv_total = 1.0 / (double(B) * npix * 4);
    loss_grad_kernel<<<B, RT, 0, static_cast<cudaStream_t>(stream)>>>(Unext, Y, Uc, npix, stats, dscale, theta, inv_total,
                                                                      loss_part, static_cast<__nv_bfloat16*>(dout16));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FVNET_OK : fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
}

int fvnet_adamw(float* params, const float* grads, float* m, float* v, long long n, double* norm_part, float lr, float b1,
                float b2, float eps, float weight_decay, float max_norm, int step, double* norm_out, void* stream) {
    if (!params || !grads || !m || !v || !norm_part || n <= 0 || step < 1)
        return fv_internal_set_error(FVNET_ERR_ARG, "fvnet_adamw: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    sq_partial_kernel<<<AB, AT, 0, st>>>(grads, n, norm_part);
    const int blocks = (int)std::min<long long>((n + AT - 1) / AT, 1024);
    adamw_kernel<<<blocks, AT, 0, st>>>(params, grads, m, v, n, norm_part, lr, b1, b2, eps, weight_decay, max_norm, step,
                                        norm_out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FVNET_OK : fv_internal_set_error(FVNET_ERR_CUDA, cudaGetErrorString(e));
}

int fvnet_norm_partials(void) { return AB; }

}  // extern "C"
